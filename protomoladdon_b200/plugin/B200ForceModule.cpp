// Registration of the B200 cutoff force (see B200ForceModule.h).
#include "B200ForceModule.h"
#include "B200CutoffSystemForce.h"

#include <protomol/ProtoMolApp.h>
#include <protomol/factory/ForceFactory.h>
#include <protomol/module/TopologyModule.h>
#include <protomol/base/StringUtilities.h>

using namespace ProtoMol;

void ProtoMol::registerB200CutoffForce(ForceFactory &factory) {
  factory.reg(new B200CutoffSystemForce());
}

void B200ForceModule::registerForces(ProtoMolApp *app) {
  // periodic boundaries only, like the CPU prototype it stands beside
  const std::string bc = app->config[InputBoundaryConditions::keyword];
  if (equalNocase(bc, PeriodicBoundaryConditions::keyword))
    registerB200CutoffForce(app->forceFactory);
}
