// Registration of the B200 forces (see B200ForceModule.h).
#include "B200ForceModule.h"
#include "B200CutoffSystemForce.h"
#include "B200EwaldRealSystemForce.h"

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

void B200ForceModule::registerForces(ProtoMolApp *app) {
  // periodic boundaries only, like the CPU prototypes they stand beside
  // (NonbondedCutoffForceModule.cpp:54, NonbondedFullElectrostaticForceModule.cpp:31)
  const std::string bc = app->config[InputBoundaryConditions::keyword];
  if (equalNocase(bc, PeriodicBoundaryConditions::keyword)) {
    registerB200CutoffForce(app->forceFactory);
    registerB200EwaldRealForce(app->forceFactory);
  }
}
