/* -*- c++ -*- */
// ProtoMol module that registers the B200 forces (the cutoff LJ + Coulomb
// force and the Ewald real-space term) with the app's ForceFactory, following the module hooks of
// protomol/src/protomol/base/Module.h (registerForces) and the periodic-only
// registration of NonbondedCutoffForceModule::registerForces
// (protomol/src/protomol/module/NonbondedCutoffForceModule.cpp:38-76).
// Add it to the module list in moduleInitFunction
// (protomol/src/protomol/modules.cpp:29-56):
//   app->modManager->add(new ProtoMol::B200ForceModule);
#ifndef PMB200_B200FORCEMODULE_H
#define PMB200_B200FORCEMODULE_H

#include <protomol/base/Module.h>

namespace ProtoMol {
class ForceFactory;

class B200ForceModule : public Module {
public:
  const std::string getName() const { return "B200Forces"; }
  void registerForces(ProtoMolApp *app);
};

// Register the prototypes with a factory directly (what registerForces does
// for a periodic configuration); for hosts that build their own factory.
void registerB200CutoffForce(ForceFactory &factory);
void registerB200EwaldRealForce(ForceFactory &factory);
// The other switch combinations (B200PairSystemForce), periodic or vacuum.
void registerB200PairForces(ForceFactory &factory, bool vacuum);
}  // namespace ProtoMol

#endif
