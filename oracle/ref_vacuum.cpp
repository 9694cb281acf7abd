// Test infrastructure only: the reference's vacuum cutoff force,
//   NonbondedCutoffSystemForce<CubicCellManager,
//     OneAtomPairTwo<VacuumBoundaryConditions, C2SwitchingFunction,
//                    LennardJonesForce, C1SwitchingFunction, CoulombForce>>
// (protomol/src/protomol/module/NonbondedCutoffForceModule.cpp:114-115), and
// its tabulated LJ registrations
//   OneAtomPair<VacuumBoundaryConditions, UniversalSwitchingFunction,
//               LennardJonesTableForce<S, 7, Real>>, S = C2, Cn, ComplimentCnCn
// (NonbondedCutoffForceModule.cpp:121-126), on a
// Topology<VacuumBoundaryConditions, CubicCellManager> built from flat
// arrays like pmref_create's periodic one.  Nothing in the product links
// this.
#include <protomol/force/nonbonded/NonbondedCutoffSystemForce.h>
#include <protomol/force/OneAtomPairTwo.h>
#include <protomol/force/LennardJonesForce.h>
#include <protomol/force/CoulombForce.h>
#include <protomol/force/OneAtomPair.h>
#include <protomol/force/table/LennardJonesTableForce.h>
#include <protomol/switch/UniversalSwitchingFunction.h>
#include <protomol/switch/CnSwitchingFunction.h>
#include <protomol/switch/CmpCnCnSwitchingFunction.h>
#include <protomol/switch/C1SwitchingFunction.h>
#include <protomol/switch/C2SwitchingFunction.h>
#include <protomol/topology/VacuumBoundaryConditions.h>
#include <protomol/topology/CubicCellManager.h>
#include <protomol/topology/CellListEnumeratorStandard.h>
#include <protomol/topology/Topology.h>
#include <protomol/topology/TopologyUtilities.h>
#include <protomol/type/ScalarStructure.h>
#include <protomol/type/Vector3DBlock.h>
#include <protomol/base/Report.h>

#include <cstring>

using namespace ProtoMol;

typedef Topology<VacuumBoundaryConditions, CubicCellManager> VTopo;
typedef OneAtomPairTwo<VacuumBoundaryConditions, C2SwitchingFunction, LennardJonesForce,
                       C1SwitchingFunction, CoulombForce>
  VPair;
typedef NonbondedCutoffSystemForce<CubicCellManager, VPair> VForce;

namespace {

void fill_topology(VTopo &t, int n, const int *type, const double *qscaled, const int *mol,
                   const double *mass, int ntypes, const double *lj, int nexcl,
                   const int *excl) {
  t.atoms.resize(n);
  int nmol = 0;
  for (int i = 0; i < n; i++) {
    t.atoms[i].type = type[i];
    t.atoms[i].scaledCharge = qscaled[i];
    t.atoms[i].molecule = mol[i];
    t.atoms[i].scaledMass = mass ? mass[i] : 1.0;
    t.atoms[i].cellListNext = -1;
    if (mol[i] + 1 > nmol) nmol = mol[i] + 1;
  }
  t.atomTypes.resize(ntypes);
  t.lennardJonesParameters.resize(ntypes);
  for (int a = 0; a < ntypes; a++)
    for (int b = 0; b < ntypes; b++) {
      const double *p = lj + 4 * (a * ntypes + b);
      t.lennardJonesParameters.set(a, b, LennardJonesParameters(p[0], p[1], p[2], p[3]));
    }
  t.molecules.resize(nmol);
  for (int m = 0; m < nmol; m++) t.molecules[m].mass = 0.0;
  for (int i = 0; i < n; i++) {
    t.molecules[mol[i]].atoms.push_back(i);
    t.molecules[mol[i]].mass += t.atoms[i].scaledMass;
  }
  t.exclusions.resize(n);
  for (int e = 0; e < nexcl; e++)
    t.exclusions.add(excl[3 * e], excl[3 * e + 1],
                     excl[3 * e + 2] == 1 ? EXCLUSION_MODIFIED : EXCLUSION_FULL);
  t.exclusions.optimize();
}

int run(SystemForce &force, VTopo &t, int n, const double *pos, double *forces,
        double *energies, double *virial, double *molvirial, int mode) {
  Vector3DBlock p(n), f(n);
  std::memcpy(p.c, pos, sizeof(double) * 3 * n);
  std::memcpy(f.c, forces, sizeof(double) * 3 * n);
  ScalarStructure e;
  e.clear();
  e.virial(mode >= 1);
  e.molecularVirial(mode >= 2);
  if (mode >= 2) buildMolecularCenterOfMass(&p, &t);
  force.evaluate(&t, &p, &f, &e);
  std::memcpy(forces, f.c, sizeof(double) * 3 * n);
  energies[0] = e[ScalarStructure::COULOMB];
  energies[1] = e[ScalarStructure::LENNARDJONES];
  if (virial)
    for (int k = 0; k < 9; k++)
      virial[k] = e[(ScalarStructure::Index)(ScalarStructure::VIRIALXX + k)];
  if (molvirial)
    for (int k = 0; k < 9; k++)
      molvirial[k] = e[(ScalarStructure::Index)(ScalarStructure::MOLVIRIALXX + k)];
  return 0;
}

template <class S>
int run_table(const S &swf, VTopo &t, int n, double rc_alg, const double *pos, double *forces,
              double *energies, double *virial, double *molvirial, int mode) {
  typedef LennardJonesTableForce<S, 7, Real> T;
  typedef OneAtomPair<VacuumBoundaryConditions, UniversalSwitchingFunction, T> P;
  NonbondedCutoffSystemForce<CubicCellManager, P> force(rc_alg,
                                                       P(T(swf), UniversalSwitchingFunction()));
  return run(force, t, n, pos, forces, energies, virial, molvirial, mode);
}

}  // namespace

extern "C" {

// One evaluation: arrays as pmref_create takes them; forces accumulated
// into; energies {COULOMB, LENNARDJONES}; mode 0/1/2 as pmref_eval.
int pmref_vacuum_eval(int n, const int *type, const double *qscaled, const int *mol,
                      const double *mass, int ntypes, const double *lj, int nexcl,
                      const int *excl, double coulomb_scaling, double cellsize, double ron,
                      double rc_lj, double rc_coul, double rc_alg, const double *pos,
                      double *forces, double *energies, double *virial, double *molvirial,
                      int mode) {
  Report::report << Report::reportlevel(-4);
  VTopo t(coulomb_scaling, ExclusionType(ExclusionType::ONE2), VacuumBoundaryConditions(),
          CubicCellManager(cellsize), 16.0f);
  fill_topology(t, n, type, qscaled, mol, mass, ntypes, lj, nexcl, excl);
  VForce force(rc_alg, VPair(LennardJonesForce(), C2SwitchingFunction(ron, rc_lj),
                             CoulombForce(), C1SwitchingFunction(rc_coul)));
  return run(force, t, n, pos, forces, energies, virial, molvirial, mode);
}

// The tabulated LJ in vacuum: kind 2 C2, 3 Cn, 4 ComplimentCnCn; p =
// {switchon, cutoff, order, switchoff}.  Returns 1 for another kind.
int pmref_vacuum_table_eval(int n, const int *type, const double *qscaled, const int *mol,
                            const double *mass, int ntypes, const double *lj, int nexcl,
                            const int *excl, double coulomb_scaling, double cellsize, int kind,
                            const double *p, double rc_alg, const double *pos, double *forces,
                            double *energies, double *virial, double *molvirial, int mode) {
  Report::report << Report::reportlevel(-4);
  VTopo t(coulomb_scaling, ExclusionType(ExclusionType::ONE2), VacuumBoundaryConditions(),
          CubicCellManager(cellsize), 16.0f);
  fill_topology(t, n, type, qscaled, mol, mass, ntypes, lj, nexcl, excl);
  if (kind == 2)
    return run_table(C2SwitchingFunction(p[0], p[1]), t, n, rc_alg, pos, forces, energies,
                     virial, molvirial, mode);
  if (kind == 3)
    return run_table(CnSwitchingFunction(p[2], p[0], p[3], p[1]), t, n, rc_alg, pos, forces,
                     energies, virial, molvirial, mode);
  if (kind == 4)
    return run_table(CmpCnCnSwitchingFunction(p[0], p[1], p[3], p[2]), t, n, rc_alg, pos,
                     forces, energies, virial, molvirial, mode);
  return 1;
}

}  // extern "C"
