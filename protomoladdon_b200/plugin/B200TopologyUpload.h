/* -*- c++ -*- */
// Copies the parts of a periodic ProtoMol topology that the B200 forces read
// into a libpmb200 context: the arrays OneAtomPairTwo::doOneAtomPair and
// NonbondedFullEwaldSystemForce::realTerm use per pair
// (protomol/src/protomol/force/OneAtomPairTwo.h:57-125,
// .../force/nonbonded/NonbondedFullEwaldSystemForce.h:776-851): type,
// scaledCharge, molecule, scaledMass, the LJ table, the exclusion table and
// coulombScalingFactor, then the box.  C++98, like the reference.
#ifndef PMB200_B200TOPOLOGYUPLOAD_H
#define PMB200_B200TOPOLOGYUPLOAD_H

#include <protomol/topology/Topology.h>
#include <protomol/topology/PeriodicBoundaryConditions.h>
#include <protomol/topology/CubicCellManager.h>
#include <protomol/parallel/Parallel.h>

#include <vector>

#include "pmb200.h"

namespace ProtoMol {

// The atoms, LJ table, exclusions and coulombScalingFactor of any topology
// with the cubic cell manager.  Returns the first non-zero libpmb200 status,
// or PMB200_OK.
template <class TBC>
int b200UploadAtoms(pmb200_ctx *ctx, const Topology<TBC, CubicCellManager> &t) {
  const int n = (int)t.atoms.size();
  const int nt = t.lennardJonesParameters.size();
  std::vector<int> type(n > 0 ? n : 1), mol(n > 0 ? n : 1);
  std::vector<double> q(n > 0 ? n : 1), mass(n > 0 ? n : 1), lj(4 * nt * nt > 0 ? 4 * nt * nt : 4);
  for (int i = 0; i < n; i++) {
    type[i] = t.atoms[i].type;
    q[i] = t.atoms[i].scaledCharge;
    mol[i] = t.atoms[i].molecule;
    mass[i] = t.atoms[i].scaledMass;
  }
  for (int a = 0; a < nt; a++)
    for (int b = 0; b < nt; b++) {
      const LennardJonesParameters &l = t.lennardJonesParameters(a, b);
      double *o = &lj[4 * (a * nt + b)];
      o[0] = l.A; o[1] = l.B; o[2] = l.A14; o[3] = l.B14;
    }
  const std::vector<ExclusionPair> &table = t.exclusions.getTable();
  std::vector<int> ex(3 * table.size() + 3);
  for (size_t k = 0; k < table.size(); k++) {
    ex[3 * k] = table[k].a1;
    ex[3 * k + 1] = table[k].a2;
    ex[3 * k + 2] = (int)table[k].excl;
  }
  return pmb200_set_topology(ctx, n, &type[0], &q[0], &mol[0], &mass[0], nt > 0 ? nt : 1,
                             &lj[0], (int)table.size(), &ex[0], t.coulombScalingFactor);
}

// The same and the periodic box.
inline int b200UploadTopology(pmb200_ctx *ctx,
                              const Topology<PeriodicBoundaryConditions, CubicCellManager> &t) {
  int rc = b200UploadAtoms(ctx, t);
  if (rc) return rc;
  const PeriodicBoundaryConditions &bc = t.boundaryConditions;
  return pmb200_set_box(ctx, bc.e1().c, bc.e2().c, bc.e3().c, bc.origin().c);
}

// Force::numberOfBlocks for the B200 forces: the cells of the device grid,
// grouped as Parallel::getNumberOfPackages groups the reference's cells
// (NonbondedCutoffForce::numberOfBlocks,
// protomol/src/protomol/force/nonbonded/NonbondedCutoffForce.h:60-65).
inline unsigned int b200NumberOfBlocks(pmb200_ctx *ctx) {
  int dims[3];
  double edge[3];
  if (pmb200_grid(ctx, dims, edge) != PMB200_OK) return 1;
  return Parallel::getNumberOfPackages((unsigned int)(dims[0] * dims[1] * dims[2]));
}

// SystemForce::parallelEvaluate's share of one rank, as
// NonbondedCutoffSystemForce::parallelEvaluate splits it
// (protomol/src/protomol/force/nonbonded/NonbondedCutoffSystemForce.h:57-77):
// block i of count = b200NumberOfBlocks covers the cells
// [n i / count, n (i + 1) / count), Parallel::next() is called once per
// block in order, and the blocks it grants are evaluated (runs of adjacent
// blocks in one pmb200_eval_cells call).  Forces and e/vir/mvir are
// accumulated into; Parallel::reduce then sums the ranks' shares
// (force/ForceGroup.cpp:116).  Returns the first non-zero libpmb200 status
// (every next() call is still made).
inline int b200ParallelEval(pmb200_ctx *ctx, const double *pos, double *forces, double *e,
                            double *vir, double *mvir, unsigned flags) {
  int dims[3];
  double edge[3];
  int rc = pmb200_grid(ctx, dims, edge);
  if (rc) return rc;
  const unsigned long long n = (unsigned long long)dims[0] * dims[1] * dims[2];
  const unsigned int count = Parallel::getNumberOfPackages((unsigned int)n);
  int lo = -1, hi = -1;
  for (unsigned int i = 0; i < count; i++) {
    const int a = (int)(n * i / count), b = (int)(n * (i + 1) / count);
    if (!Parallel::next()) continue;
    if (lo >= 0 && a == hi) {
      hi = b;
      continue;
    }
    if (lo >= 0 && !rc) rc = pmb200_eval_cells(ctx, pos, forces, e, vir, mvir, flags, lo, hi);
    lo = a;
    hi = b;
  }
  if (lo >= 0 && !rc) rc = pmb200_eval_cells(ctx, pos, forces, e, vir, mvir, flags, lo, hi);
  return rc;
}

}  // namespace ProtoMol

#endif  // PMB200_B200TOPOLOGYUPLOAD_H
