// Test infrastructure only: the reference's own analytic Hessian of the
// nonbonded energy, Hessian::findForces + Hessian::evaluate
// (protomol/src/protomol/integrator/hessian/Hessian.cpp:116-568, pair
// blocks 581-691 with ReducedHessLennardJones, ReducedHessCoulomb and the
// C1/C2 switch Hessians), on the topology pmref_create built.  The Hessian
// reads its switches from the force ids in a ForceGroup, and parses a
// combined "LennardJones Coulomb" force as Lennard-Jones alone, so the group
// holds the two terms as the separate forces it understands:
//   LennardJones -algorithm NonbondedCutoff -switchingFunction C2 ...
//   Coulomb -algorithm NonbondedCutoff -switchingFunction C1 ...
// (NonbondedCutoffForceModule.cpp:61, 55), whose sum is the combined force.
// Nothing in the product links this.
#include <protomol/integrator/hessian/Hessian.h>
#include <protomol/force/ForceGroup.h>
#include <protomol/force/nonbonded/NonbondedCutoffSystemForce.h>
#include <protomol/force/OneAtomPair.h>
#include <protomol/force/LennardJonesForce.h>
#include <protomol/force/CoulombForce.h>
#include <protomol/switch/C1SwitchingFunction.h>
#include <protomol/switch/C2SwitchingFunction.h>
#include <protomol/topology/PeriodicBoundaryConditions.h>
#include <protomol/topology/CubicCellManager.h>
#include <protomol/topology/CellListEnumeratorPeriodicBoundaries.h>
#include <protomol/topology/Topology.h>
#include <protomol/type/Vector3DBlock.h>
#include <protomol/base/Report.h>

#include <cstring>

using namespace ProtoMol;

typedef Topology<PeriodicBoundaryConditions, CubicCellManager> PTopo;
typedef NonbondedCutoffSystemForce<
    CubicCellManager, OneAtomPair<PeriodicBoundaryConditions, C2SwitchingFunction,
                                  LennardJonesForce> >
    LJForce;
typedef NonbondedCutoffSystemForce<
    CubicCellManager, OneAtomPair<PeriodicBoundaryConditions, C1SwitchingFunction,
                                  CoulombForce> >
    CoulForce;

extern "C" {

void *pmref_topology(void *h);

// hess: (3n)^2 doubles, column-major as Hessian::hessM, overwritten (not
// mass-weighted).  Returns 0.
int pmref_hessian(void *h, const double *pos, double *hess, double ron, double rc_lj,
                  double rc_coul, double rc_alg) {
  Report::report << Report::reportlevel(-4);
  PTopo *t = (PTopo *)pmref_topology(h);
  const int n = (int)t->atoms.size();
  Vector3DBlock p(n);
  std::memcpy(p.c, pos, sizeof(double) * 3 * n);
  ForceGroup group;
  group.addSystemForce(new LJForce(rc_alg, OneAtomPair<PeriodicBoundaryConditions,
                                                       C2SwitchingFunction, LennardJonesForce>(
                                               LennardJonesForce(),
                                               C2SwitchingFunction(ron, rc_lj))));
  group.addSystemForce(new CoulForce(rc_alg, OneAtomPair<PeriodicBoundaryConditions,
                                                         C1SwitchingFunction, CoulombForce>(
                                                 CoulombForce(), C1SwitchingFunction(rc_coul))));
  Hessian hs;
  hs.findForces(&group);
  hs.initialData(3 * n);
  hs.clear();
  hs.evaluate(&p, t, false);
  std::memcpy(hess, hs.hessM, sizeof(double) * 9 * (size_t)n * n);
  return 0;
}

}  // extern "C"
