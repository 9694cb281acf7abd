// Test harness: the B200 plugin force inside the reference's own
// ForceFactory, next to the reference prototype, on a reference-built
// Topology.  Built by tests/plugin/Makefile against the reference library
// compiled under oracle/_ref; used only by tests/test_plugin_gpu.py.
#include "B200CutoffSystemForce.h"
#include "B200EwaldRealSystemForce.h"
#include "B200PairSystemForce.h"
#include "B200ForceModule.h"

#include <protomol/factory/ForceFactory.h>
#include <protomol/force/nonbonded/NonbondedCutoffSystemForce.h>
#include <protomol/force/nonbonded/NonbondedFullEwaldSystemForce.h>
#include <protomol/switch/CutoffSwitchingFunction.h>
#include <protomol/force/OneAtomPairTwo.h>
#include <protomol/force/LennardJonesForce.h>
#include <protomol/force/CoulombForce.h>
#include <protomol/switch/C1SwitchingFunction.h>
#include <protomol/switch/C2SwitchingFunction.h>
#include <protomol/topology/CellListEnumeratorPeriodicBoundaries.h>
#include <protomol/topology/CellListEnumeratorStandard.h>
#include <protomol/topology/VacuumBoundaryConditions.h>
#include <protomol/switch/CnSwitchingFunction.h>
#include <protomol/force/OneAtomPair.h>
#include <protomol/topology/TopologyUtilities.h>
#include <protomol/config/Value.h>
#include <protomol/parallel/Parallel.h>

#include <cstring>
#include <exception>
#include <string>

using namespace ProtoMol;

extern "C" void *pmref_topology(void *h);

typedef Topology<PeriodicBoundaryConditions, CubicCellManager> PTopo;
typedef NonbondedCutoffSystemForce<
    CubicCellManager, OneAtomPairTwo<PeriodicBoundaryConditions, C2SwitchingFunction,
                                     LennardJonesForce, C1SwitchingFunction, CoulombForce> >
    RefForce;
typedef NonbondedFullEwaldSystemForce<PeriodicBoundaryConditions, CubicCellManager, true, false,
                                      false, CutoffSwitchingFunction>
    RefEwaldReal;

static char g_msg[1024];
// parallel mode: forces are called through SystemForce::parallelEvaluate
// (with Force::numberOfBlocks asked first, as ForceGroup does) instead of
// evaluate; without MPI, Parallel::next() grants every block
static int g_parallel = 0;
static unsigned int g_blocks = 0;

extern "C" const char *harness_message() { return g_msg; }
extern "C" void harness_set_parallel(int on) { g_parallel = on; }
extern "C" unsigned int harness_last_blocks() { return g_blocks; }

template <class TTopo>
static void call_force(Force *force, TTopo *t, Vector3DBlock *p, Vector3DBlock *fr,
                       ScalarStructure *en) {
  SystemForce *sf = dynamic_cast<SystemForce *>(force);
  if (g_parallel) {
    Parallel::resetNext();
    g_blocks = sf->numberOfBlocks(t, p);
    sf->parallelEvaluate(t, p, fr, en);
  } else {
    sf->evaluate(t, p, fr, en);
  }
}

static Force *make_force(ForceFactory &f, const std::string &id, double ron, double rclj,
                         double rcc, double rc) {
  std::vector<Value> v;
  v.push_back(Value(ron));
  v.push_back(Value(rclj));
  v.push_back(Value(rcc));
  v.push_back(Value(rc));
  return f.make(id, v);
}

static void eval_force(Force *force, PTopo *t, const double *pos, int n, double *f, double *e,
                       double *vir, double *mvir) {
  Vector3DBlock p(n), fr(n);
  std::memcpy(p.c, pos, sizeof(double) * 3 * n);
  fr.zero();
  ScalarStructure en;
  en.clear();
  en.virial(true);
  en.molecularVirial(true);
  buildMolecularCenterOfMass(&p, t);
  call_force(force, t, &p, &fr, &en);
  std::memcpy(f, fr.c, sizeof(double) * 3 * n);
  e[0] = en[ScalarStructure::COULOMB];
  e[1] = en[ScalarStructure::LENNARDJONES];
  for (int k = 0; k < 9; k++) {
    vir[k] = en[(ScalarStructure::Index)(ScalarStructure::VIRIALXX + k)];
    mvir[k] = en[(ScalarStructure::Index)(ScalarStructure::MOLVIRIALXX + k)];
  }
}

// which: 0 = the reference prototype, 1 = the B200 plugin, 2 = the B200
// plugin through the reference's "time" decorator.  Forces are made by the
// factory from the config-file id and the four parameter values.
// Returns 0, or 1 with harness_message() set (factory / plugin exceptions).
extern "C" int harness_eval(void *ref_handle, int which, int n, const double *pos, double ron,
                            double rclj, double rcc, double rc, double *forces,
                            double *energies, double *virial, double *molvirial) {
  g_msg[0] = 0;
  try {
    PTopo *t = (PTopo *)pmref_topology(ref_handle);
    ForceFactory factory;
    factory.reg(new RefForce());
    registerB200CutoffForce(factory);
    const char *base = "LennardJones Coulomb -switchingFunction C2 -switchingFunction C1 -algorithm ";
    std::string id = std::string(base) + (which == 0 ? "NonbondedCutoff" : "NonbondedCutoffB200");
    if (which == 2) id = "time " + id;
    Force *force = make_force(factory, id, ron, rclj, rcc, rc);
    if (!force) {
      std::strncpy(g_msg, ("factory could not make '" + id + "'").c_str(), sizeof(g_msg) - 1);
      return 1;
    }
    std::strncpy(g_msg, force->getId().c_str(), sizeof(g_msg) - 1);
    eval_force(force, t, pos, n, forces, energies, virial, molvirial);
    delete force;
    return 0;
  } catch (const std::exception &e) {
    std::strncpy(g_msg, e.what(), sizeof(g_msg) - 1);
  } catch (...) {
    std::strncpy(g_msg, "unknown exception", sizeof(g_msg) - 1);
  }
  return 1;
}

// The Ewald real-space term: which 0 = the reference prototype
// ("Coulomb -algorithm FullEwald -real"), 1 = the B200 plugin
// ("Coulomb -algorithm FullEwaldB200 -real"); made by the factory from the id
// and the values {alpha, accuracy}.
extern "C" int harness_ewald_eval(void *ref_handle, int which, int n, const double *pos,
                                  double alpha, double accuracy, double *forces,
                                  double *energies, double *virial, double *molvirial) {
  g_msg[0] = 0;
  try {
    PTopo *t = (PTopo *)pmref_topology(ref_handle);
    ForceFactory factory;
    factory.reg(new RefEwaldReal());
    registerB200EwaldRealForce(factory);
    std::string id = which == 0 ? "Coulomb -algorithm FullEwald -real"
                                : "Coulomb -algorithm FullEwaldB200 -real";
    std::vector<Value> v;
    v.push_back(Value(alpha));
    v.push_back(Value(accuracy));
    Force *force = factory.make(id, v);
    if (!force) {
      std::strncpy(g_msg, ("factory could not make '" + id + "'").c_str(), sizeof(g_msg) - 1);
      return 1;
    }
    std::strncpy(g_msg, force->getId().c_str(), sizeof(g_msg) - 1);
    eval_force(force, t, pos, n, forces, energies, virial, molvirial);
    delete force;
    return 0;
  } catch (const std::exception &e) {
    std::strncpy(g_msg, e.what(), sizeof(g_msg) - 1);
  } catch (...) {
    std::strncpy(g_msg, "unknown exception", sizeof(g_msg) - 1);
  }
  return 1;
}

// The other switch combinations through the factory: the id (e.g.
// "LennardJones Coulomb -switchingFunction C2 -switchingFunction Cn
// -algorithm NonbondedCutoffB200") and its parameter values in order.
// vacuum = 0: on the periodic topology of ref_handle; 1: on a vacuum
// topology built here from that topology's atoms and tables.
template <class TBC>
static int pair_eval_on(Topology<TBC, CubicCellManager> *t, bool vacuum, const char *id,
                        int nvalues, const double *values, const double *pos, int n,
                        double *forces, double *energies, double *virial, double *molvirial) {
  ForceFactory factory;
  registerB200PairForces(factory, vacuum);
  std::vector<Value> v;
  for (int k = 0; k < nvalues; k++) v.push_back(Value(values[k]));
  Force *force = factory.make(id, v);
  if (!force) {
    std::strncpy(g_msg, (std::string("factory could not make '") + id + "'").c_str(),
                 sizeof(g_msg) - 1);
    return 1;
  }
  std::strncpy(g_msg, force->getId().c_str(), sizeof(g_msg) - 1);
  Vector3DBlock p(n), fr(n);
  std::memcpy(p.c, pos, sizeof(double) * 3 * n);
  fr.zero();
  ScalarStructure en;
  en.clear();
  en.virial(true);
  en.molecularVirial(true);
  buildMolecularCenterOfMass(&p, t);
  call_force(force, t, &p, &fr, &en);
  std::memcpy(forces, fr.c, sizeof(double) * 3 * n);
  energies[0] = en[ScalarStructure::COULOMB];
  energies[1] = en[ScalarStructure::LENNARDJONES];
  for (int k = 0; k < 9; k++) {
    virial[k] = en[(ScalarStructure::Index)(ScalarStructure::VIRIALXX + k)];
    molvirial[k] = en[(ScalarStructure::Index)(ScalarStructure::MOLVIRIALXX + k)];
  }
  delete force;
  return 0;
}

extern "C" int harness_pair_eval(void *ref_handle, int vacuum, const char *id, int nvalues,
                                 const double *values, int n, const double *pos, double *forces,
                                 double *energies, double *virial, double *molvirial) {
  g_msg[0] = 0;
  try {
    PTopo *t = (PTopo *)pmref_topology(ref_handle);
    if (!vacuum)
      return pair_eval_on(t, false, id, nvalues, values, pos, n, forces, energies, virial,
                          molvirial);
    typedef Topology<VacuumBoundaryConditions, CubicCellManager> VTopo;
    VTopo v(t->coulombScalingFactor, ExclusionType(ExclusionType::ONE2),
            VacuumBoundaryConditions(), CubicCellManager(4.0), 16.0f);
    // element-wise copies: the LJ and exclusion tables own raw arrays
    v.atoms = t->atoms;
    v.atomTypes = t->atomTypes;
    v.molecules = t->molecules;
    const int nt = (int)t->lennardJonesParameters.size();
    v.lennardJonesParameters.resize(nt);
    for (int a = 0; a < nt; a++)
      for (int b = 0; b < nt; b++)
        v.lennardJonesParameters.set(a, b, t->lennardJonesParameters(a, b));
    v.exclusions.resize(n);
    const std::vector<ExclusionPair> &tab = t->exclusions.getTable();
    for (size_t k = 0; k < tab.size(); k++) v.exclusions.add(tab[k].a1, tab[k].a2, tab[k].excl);
    v.exclusions.optimize();
    return pair_eval_on(&v, true, id, nvalues, values, pos, n, forces, energies, virial,
                        molvirial);
  } catch (const std::exception &e) {
    std::strncpy(g_msg, e.what(), sizeof(g_msg) - 1);
  } catch (...) {
    std::strncpy(g_msg, "unknown exception", sizeof(g_msg) - 1);
  }
  return 1;
}
