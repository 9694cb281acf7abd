// Registration of the B200 forces (see B200ForceModule.h).
#include "B200ForceModule.h"
#include "B200CutoffSystemForce.h"
#include "B200EwaldRealSystemForce.h"
#include "B200PairSystemForce.h"

#include <protomol/ProtoMolApp.h>
#include <protomol/factory/ForceFactory.h>
#include <protomol/module/TopologyModule.h>
#include <protomol/base/StringUtilities.h>

using namespace ProtoMol;

void ProtoMol::registerB200CutoffForce(ForceFactory &factory) {
  factory.reg(new B200CutoffSystemForce());
}

void ProtoMol::registerB200EwaldRealForce(ForceFactory &factory) {
  factory.reg(new B200EwaldRealSystemForce());
}

// The switch combinations NonbondedCutoffForceModule registers for the
// plain and tabulated LJ / Coulomb potentials (NonbondedCutoffForceModule.cpp:
// 55-82 and 98-141); the periodic (C2, C1) pair has its own class.
template <class TBC>
static void registerPairs(ForceFactory &f, bool vacuum) {
  const int C1 = PMB200_SW_C1, C2 = PMB200_SW_C2, CN = PMB200_SW_CN, NO = PMB200_SW_NONE,
            CM = PMB200_SW_CMPCNCN;
  const int common[][2] = {{NO, C1}, {NO, C2}, {NO, CN}, {NO, CM}, {C1, NO}, {C2, NO},
                           {CN, NO}, {CM, NO}, {C2, C2}, {C2, CN}, {CN, CN}};
  for (int k = 0; k < (int)(sizeof(common) / sizeof(common[0])); k++)
    f.reg(new B200PairSystemForce<TBC>(common[k][0], common[k][1]));
  // OneAtomPair<BC, Universal, LennardJonesTableForce<S, 7, Real>>
  // (NonbondedCutoffForceModule.cpp:67-72, 121-126)
  const int TB = PMB200_SW_TABLE;
  f.reg(new B200PairSystemForce<TBC>(TB | C2, NO));
  f.reg(new B200PairSystemForce<TBC>(TB | CN, NO));
  f.reg(new B200PairSystemForce<TBC>(TB | CM, NO));
  if (vacuum) {
    f.reg(new B200PairSystemForce<TBC>(C2, C1));
    f.reg(new B200PairSystemForce<TBC>(CM, C1));
  } else {
    f.reg(new B200PairSystemForce<TBC>(CM, CM));
  }
}

void ProtoMol::registerB200PairForces(ForceFactory &factory, bool vacuum) {
  if (vacuum) registerPairs<VacuumBoundaryConditions>(factory, true);
  else registerPairs<PeriodicBoundaryConditions>(factory, false);
}

void B200ForceModule::registerForces(ProtoMolApp *app) {
  // the same split by boundary conditions as the CPU prototypes they stand
  // beside (NonbondedCutoffForceModule.cpp:53, 96;
  // NonbondedFullElectrostaticForceModule.cpp:31)
  const std::string bc = app->config[InputBoundaryConditions::keyword];
  if (equalNocase(bc, PeriodicBoundaryConditions::keyword)) {
    registerB200CutoffForce(app->forceFactory);
    registerB200EwaldRealForce(app->forceFactory);
    registerB200PairForces(app->forceFactory, false);
  } else if (equalNocase(bc, VacuumBoundaryConditions::keyword)) {
    registerB200PairForces(app->forceFactory, true);
  }
}
