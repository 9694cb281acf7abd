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

}  // namespace ProtoMol

#endif  // PMB200_B200TOPOLOGYUPLOAD_H
