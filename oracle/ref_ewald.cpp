// Test infrastructure only: a C entry into the reference's own Ewald
// real-space force,
//   NonbondedFullEwaldSystemForce<PeriodicBoundaryConditions,
//     CubicCellManager, real = true, reciprocal = false, correction = false,
//     CutoffSwitchingFunction>
// (protomol/src/protomol/module/NonbondedFullElectrostaticForceModule.cpp:34,
// "Coulomb -algorithm FullEwald -real"), evaluated on the topology that
// pmref_create (ref_driver.cpp) built.  oracle/Makefile compiles this file
// twice: as the reference ships it (erfc by the Abramowitz & Stegun
// polynomial) into libpmref.so, and with USE_EWALD_EXACT_ERF (libm erfc,
// protomol/src/protomol/force/nonbonded/NonbondedFullEwaldSystemForce.h:30)
// into libpmref_exacterf.so.  Nothing in the product links either.
#include <protomol/force/nonbonded/NonbondedFullEwaldSystemForce.h>
#include <protomol/switch/CutoffSwitchingFunction.h>
#include <protomol/topology/PeriodicBoundaryConditions.h>
#include <protomol/topology/CubicCellManager.h>
#include <protomol/topology/Topology.h>
#include <protomol/topology/TopologyUtilities.h>
#include <protomol/type/ScalarStructure.h>
#include <protomol/type/Vector3DBlock.h>
#include <protomol/base/Report.h>

#include <cstring>

using namespace ProtoMol;

typedef Topology<PeriodicBoundaryConditions, CubicCellManager> PTopo;
typedef NonbondedFullEwaldSystemForce<PeriodicBoundaryConditions, CubicCellManager, true,
                                      false, false, CutoffSwitchingFunction>
  EwaldReal;

extern "C" {

void *pmref_topology(void *h);

// 1 when this library's Ewald force uses libm erfc, 0 for the polynomial.
int pmref_ewald_exact_erfc(void) {
#ifdef USE_EWALD_EXACT_ERF
  return 1;
#else
  return 0;
#endif
}

// One SystemForce::evaluate of a fresh real-space Ewald force (alpha <= 0:
// the reference's default).  forces (3n, AoS) are accumulated into;
// energies[0] = the Coulomb term it adds; virial/molvirial (9 each) written
// per virial_mode (0 none, 1 atomic, 2 atomic + molecular).
int pmref_ewald_eval(void *h, double alpha, double accuracy, const double *pos,
                     double *forces, double *energies, double *virial, double *molvirial,
                     int virial_mode) {
  Report::report << Report::reportlevel(-4);
  PTopo *t = (PTopo *)pmref_topology(h);
  const int n = (int)t->atoms.size();
  Vector3DBlock p(n), f(n);
  memcpy(p.c, pos, sizeof(double) * 3 * n);
  memcpy(f.c, forces, sizeof(double) * 3 * n);
  ScalarStructure e;
  e.clear();
  e.virial(virial_mode >= 1);
  e.molecularVirial(virial_mode >= 2);
  if (virial_mode >= 2) buildMolecularCenterOfMass(&p, t);
  t->uncacheCellList();
  EwaldReal force(alpha, accuracy, 3.0);
  force.evaluate(t, &p, &f, &e);
  memcpy(forces, f.c, sizeof(double) * 3 * n);
  energies[0] = e[ScalarStructure::COULOMB];
  if (virial)
    for (int k = 0; k < 9; k++)
      virial[k] = e[(ScalarStructure::Index)(ScalarStructure::VIRIALXX + k)];
  if (molvirial)
    for (int k = 0; k < 9; k++)
      molvirial[k] = e[(ScalarStructure::Index)(ScalarStructure::MOLVIRIALXX + k)];
  return 0;
}

}  // extern "C"
