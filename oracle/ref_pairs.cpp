// Test infrastructure only: the reference's other periodic cutoff
// registrations (protomol/src/protomol/module/NonbondedCutoffForceModule.cpp:
// 53-82) -- NonbondedCutoffSystemForce<CubicCellManager, P> with
//   P = OneAtomPair<PBC, S, LennardJonesForce>, OneAtomPair<PBC, S, CoulombForce>,
//       OneAtomPairTwo<PBC, S1, LennardJonesForce, S2, CoulombForce>,
//       OneAtomPair<PBC, UniversalSwitchingFunction, LennardJonesTableForce<S, 7, Real>>
// and S, S1, S2 among C1, C2, Cn and ComplimentCnCn -- evaluated on the topology pmref_create
// built.  Nothing in the product links this.
#include <protomol/force/nonbonded/NonbondedCutoffSystemForce.h>
#include <protomol/force/OneAtomPair.h>
#include <protomol/force/OneAtomPairTwo.h>
#include <protomol/force/LennardJonesForce.h>
#include <protomol/force/CoulombForce.h>
#include <protomol/force/table/LennardJonesTableForce.h>
#include <protomol/switch/UniversalSwitchingFunction.h>
#include <protomol/switch/C1SwitchingFunction.h>
#include <protomol/switch/C2SwitchingFunction.h>
#include <protomol/switch/CnSwitchingFunction.h>
#include <protomol/switch/CmpCnCnSwitchingFunction.h>
#include <protomol/topology/PeriodicBoundaryConditions.h>
#include <protomol/topology/CubicCellManager.h>
#include <protomol/topology/CellListEnumeratorPeriodicBoundaries.h>
#include <protomol/topology/Topology.h>
#include <protomol/topology/TopologyUtilities.h>
#include <protomol/type/ScalarStructure.h>
#include <protomol/type/Vector3DBlock.h>
#include <protomol/base/Report.h>

#include <cstring>

using namespace ProtoMol;

typedef Topology<PeriodicBoundaryConditions, CubicCellManager> PTopo;
typedef PeriodicBoundaryConditions PBC;

namespace {

// switch kinds as in include/pmb200.h: 1 C1, 2 C2, 3 Cn, 4 ComplimentCnCn;
// p = {switchon, cutoff, order, switchoff}
C1SwitchingFunction sw(const C1SwitchingFunction *, const double *p) {
  return C1SwitchingFunction(p[1]);
}
C2SwitchingFunction sw(const C2SwitchingFunction *, const double *p) {
  return C2SwitchingFunction(p[0], p[1]);
}
CnSwitchingFunction sw(const CnSwitchingFunction *, const double *p) {
  return CnSwitchingFunction(p[2], p[0], p[3], p[1]);
}
CmpCnCnSwitchingFunction sw(const CmpCnCnSwitchingFunction *, const double *p) {
  return CmpCnCnSwitchingFunction(p[0], p[1], p[3], p[2]);
}

int run(SystemForce *force, PTopo *t, const double *pos, double *forces, double *energies,
        double *virial, double *molvirial, int mode) {
  const int n = (int)t->atoms.size();
  Vector3DBlock p(n), f(n);
  std::memcpy(p.c, pos, sizeof(double) * 3 * n);
  std::memcpy(f.c, forces, sizeof(double) * 3 * n);
  ScalarStructure e;
  e.clear();
  e.virial(mode >= 1);
  e.molecularVirial(mode >= 2);
  if (mode >= 2) buildMolecularCenterOfMass(&p, t);
  t->uncacheCellList();
  force->evaluate(t, &p, &f, &e);
  std::memcpy(forces, f.c, sizeof(double) * 3 * n);
  energies[0] = e[ScalarStructure::COULOMB];
  energies[1] = e[ScalarStructure::LENNARDJONES];
  if (virial)
    for (int k = 0; k < 9; k++)
      virial[k] = e[(ScalarStructure::Index)(ScalarStructure::VIRIALXX + k)];
  if (molvirial)
    for (int k = 0; k < 9; k++)
      molvirial[k] = e[(ScalarStructure::Index)(ScalarStructure::MOLVIRIALXX + k)];
  delete force;
  return 0;
}

template <class S>
SystemForce *single_lj(const double *p, double rc) {
  typedef OneAtomPair<PBC, S, LennardJonesForce> P;
  return new NonbondedCutoffSystemForce<CubicCellManager, P>(
      rc, P(LennardJonesForce(), sw((S *)0, p)));
}
template <class S>
SystemForce *single_coul(const double *p, double rc) {
  typedef OneAtomPair<PBC, S, CoulombForce> P;
  return new NonbondedCutoffSystemForce<CubicCellManager, P>(rc,
                                                             P(CoulombForce(), sw((S *)0, p)));
}
template <class S1, class S2>
SystemForce *two(const double *p1, const double *p2, double rc) {
  typedef OneAtomPairTwo<PBC, S1, LennardJonesForce, S2, CoulombForce> P;
  return new NonbondedCutoffSystemForce<CubicCellManager, P>(
      rc, P(LennardJonesForce(), sw((S1 *)0, p1), CoulombForce(), sw((S2 *)0, p2)));
}
template <class S>
SystemForce *table_lj(const double *p, double rc) {
  typedef LennardJonesTableForce<S, 7, Real> T;
  typedef OneAtomPair<PBC, UniversalSwitchingFunction, T> P;
  return new NonbondedCutoffSystemForce<CubicCellManager, P>(
      rc, P(T(sw((S *)0, p)), UniversalSwitchingFunction()));
}
template <class S1>
SystemForce *two_any(int k2, const double *p1, const double *p2, double rc) {
  if (k2 == 1) return two<S1, C1SwitchingFunction>(p1, p2, rc);
  if (k2 == 2) return two<S1, C2SwitchingFunction>(p1, p2, rc);
  if (k2 == 4) return two<S1, CmpCnCnSwitchingFunction>(p1, p2, rc);
  return two<S1, CnSwitchingFunction>(p1, p2, rc);
}

}  // namespace

extern "C" {

void *pmref_topology(void *h);

// lj_kind / coul_kind: 0 none, 1 C1, 2 C2, 3 Cn, 4 ComplimentCnCn (at least
// one non-zero); lj_kind 16 + S: the tabulated LJ with switch S (2, 3, 4),
// alone;
// forces accumulated into; energies {COULOMB, LENNARDJONES}; mode 0/1/2 as
// pmref_eval.  Returns 0, or 1 for an unknown kind.
int pmref_pair_eval(void *h, int lj_kind, const double *ljp, int coul_kind, const double *cop,
                    double rc_alg, const double *pos, double *forces, double *energies,
                    double *virial, double *molvirial, int mode) {
  Report::report << Report::reportlevel(-4);
  PTopo *t = (PTopo *)pmref_topology(h);
  SystemForce *f = 0;
  if (lj_kind & 16) {
    if (coul_kind) return 1;
    if (lj_kind == 18) f = table_lj<C2SwitchingFunction>(ljp, rc_alg);
    else if (lj_kind == 19) f = table_lj<CnSwitchingFunction>(ljp, rc_alg);
    else if (lj_kind == 20) f = table_lj<CmpCnCnSwitchingFunction>(ljp, rc_alg);
  } else if (lj_kind && coul_kind) {
    if (lj_kind == 1) f = two_any<C1SwitchingFunction>(coul_kind, ljp, cop, rc_alg);
    else if (lj_kind == 2) f = two_any<C2SwitchingFunction>(coul_kind, ljp, cop, rc_alg);
    else if (lj_kind == 4) f = two_any<CmpCnCnSwitchingFunction>(coul_kind, ljp, cop, rc_alg);
    else f = two_any<CnSwitchingFunction>(coul_kind, ljp, cop, rc_alg);
  } else if (lj_kind) {
    if (lj_kind == 1) f = single_lj<C1SwitchingFunction>(ljp, rc_alg);
    else if (lj_kind == 2) f = single_lj<C2SwitchingFunction>(ljp, rc_alg);
    else if (lj_kind == 4) f = single_lj<CmpCnCnSwitchingFunction>(ljp, rc_alg);
    else f = single_lj<CnSwitchingFunction>(ljp, rc_alg);
  } else if (coul_kind) {
    if (coul_kind == 1) f = single_coul<C1SwitchingFunction>(cop, rc_alg);
    else if (coul_kind == 2) f = single_coul<C2SwitchingFunction>(cop, rc_alg);
    else if (coul_kind == 4) f = single_coul<CmpCnCnSwitchingFunction>(cop, rc_alg);
    else f = single_coul<CnSwitchingFunction>(cop, rc_alg);
  }
  if (!f) return 1;
  return run(f, t, pos, forces, energies, virial, molvirial, mode);
}

}  // extern "C"
