/* -*- c++ -*- */
// ProtoMol SystemForce that evaluates the periodic cutoff LJ(C2) +
// Coulomb(C1) force on a B200 through libpmb200 (include/pmb200.h).
//
// It stands where ProtoMol registers
//   NonbondedCutoffSystemForce<CubicCellManager,
//     OneAtomPairTwo<PeriodicBoundaryConditions, C2SwitchingFunction,
//                    LennardJonesForce, C1SwitchingFunction, CoulombForce>>
// (protomol/src/protomol/module/NonbondedCutoffForceModule.cpp:75-76) under
// its own algorithm keyword, NonbondedCutoffB200, because duplicate ids throw
// (protomol/src/protomol/base/Factory.h:50-58).  Parameters come in the
// reference's order (OneAtomPairTwo::getParameters then
// NonbondedCutoffForce::getParameters): C2 -switchon, C2 -cutoff, C1 -cutoff,
// algorithm -cutoff.  Written in the C++98 dialect the reference builds with.
#ifndef PMB200_B200CUTOFFSYSTEMFORCE_H
#define PMB200_B200CUTOFFSYSTEMFORCE_H

#include <protomol/force/system/SystemForce.h>
#include <protomol/topology/Topology.h>
#include <protomol/topology/PeriodicBoundaryConditions.h>
#include <protomol/topology/CubicCellManager.h>
#include <protomol/type/ScalarStructure.h>
#include <protomol/type/Vector3DBlock.h>
#include <protomol/base/Exception.h>
#include <protomol/base/StringUtilities.h>

#include <string>
#include <vector>

#include "pmb200.h"
#include "B200TopologyUpload.h"

namespace ProtoMol {

class B200CutoffSystemForce : public SystemForce {
  typedef Topology<PeriodicBoundaryConditions, CubicCellManager> RealTopologyType;

public:
  // Prototype for the factory (no device context).
  B200CutoffSystemForce() : myCtx(0), myCached(0) { setParams(0.0, 0.0, 0.0, 0.0); }

  // A working force; the parameters are checked like
  // C2SwitchingFunction::make (0 <= switchon < cutoff).
  B200CutoffSystemForce(Real switchon, Real cutoffLJ, Real cutoffCoulomb, Real cutoff,
                        int precision = PMB200_MIXED, int device = 0)
      : myCtx(0), myCached(0) {
    setParams(switchon, cutoffLJ, cutoffCoulomb, cutoff);
    myParams.precision = precision;
    myParams.device = device;
    const int rc = pmb200_create(&myParams, &myCtx);
    if (rc == PMB200_ECUDA)
      THROW("B200 cutoff force: no usable CUDA device " + toString(device) + ".");
    if (rc)
      THROW("B200 cutoff force: parameters rejected (status " + toString(rc) +
            "); need 0 <= switchon < C2 cutoff and algorithm cutoff >= both switch cutoffs.");
  }

  virtual ~B200CutoffSystemForce() { pmb200_destroy(myCtx); }

  // SystemForce::evaluate (protomol/src/protomol/force/system/SystemForce.h:
  // 32-35): forces and energies are accumulated into; the virial and the
  // molecular virial are added when the ScalarStructure asks for them.
  virtual void evaluate(const GenericTopology *topo, const Vector3DBlock *positions,
                        Vector3DBlock *forces, ScalarStructure *energies) {
    run(topo, positions, forces, energies, false);
  }

  // SystemForce::parallelEvaluate (the default evaluates everything on every
  // rank, force/system/SystemForce.h:91-96, which Parallel::reduce would then
  // count once per rank): this rank's blocks of cells only, as
  // NonbondedCutoffSystemForce::parallelEvaluate does.
  virtual void parallelEvaluate(const GenericTopology *topo, const Vector3DBlock *positions,
                                Vector3DBlock *forces, ScalarStructure *energies) {
    run(topo, positions, forces, energies, true);
  }

  // Force::numberOfBlocks: the Parallel::next() calls parallelEvaluate makes.
  virtual unsigned int numberOfBlocks(const GenericTopology *topo, const Vector3DBlock *) {
    prepare(topo);
    return b200NumberOfBlocks(myCtx);
  }

private:
  void prepare(const GenericTopology *topo) {
    if (!myCtx) THROW("B200 cutoff force: evaluate called on the factory prototype.");
    const RealTopologyType *t = dynamic_cast<const RealTopologyType *>(topo);
    if (!t) THROW("B200 cutoff force: needs periodic boundaries and the cubic cell manager.");
    if (myCached != topo) upload(*t);
  }

  void run(const GenericTopology *topo, const Vector3DBlock *positions, Vector3DBlock *forces,
           ScalarStructure *energies, bool parallel) {
    prepare(topo);
    unsigned flags = PMB200_ENERGY;
    if (energies->virial()) flags |= PMB200_VIRIAL;
    if (energies->molecularVirial()) flags |= PMB200_MOLVIRIAL;
    double e[2] = {0.0, 0.0};
    double vir[9], mvir[9];
    for (int k = 0; k < 9; k++) vir[k] = mvir[k] = 0.0;
    if (parallel)
      check(b200ParallelEval(myCtx, positions->c, forces->c, e, vir, mvir, flags));
    else
      check(pmb200_eval(myCtx, positions->c, forces->c, e, vir, mvir, flags));
    (*energies)[ScalarStructure::COULOMB] += e[0];
    (*energies)[ScalarStructure::LENNARDJONES] += e[1];
    for (int k = 0; k < 9; k++) {
      if (flags & PMB200_VIRIAL)
        (*energies)[(ScalarStructure::Index)(ScalarStructure::VIRIALXX + k)] += vir[k];
      if (flags & PMB200_MOLVIRIAL)
        (*energies)[(ScalarStructure::Index)(ScalarStructure::MOLVIRIALXX + k)] += mvir[k];
    }
  }

public:
  // The topology (types, charges, exclusions, box) is re-read after this.
  virtual void uncache() { myCached = 0; }

  virtual std::string getKeyword() const { return "NonbondedCutoffB200"; }

  virtual std::string getIdNoAlias() const {
    return "LennardJones Coulomb -switchingFunction C2 -switchingFunction C1 -algorithm " +
           getKeyword();
  }

  virtual void getParameters(std::vector<Parameter> &parameters) const {
    parameters.push_back(Parameter("-switchon",
                                   Value(myParams.switchon, ConstraintValueType::NotNegative()),
                                   Text("C2 swf switch on")));
    parameters.push_back(Parameter("-cutoff",
                                   Value(myParams.cutoff_lj, ConstraintValueType::Positive()),
                                   Text("C2 swf cutoff")));
    parameters.push_back(Parameter("-cutoff",
                                   Value(myParams.cutoff_coul, ConstraintValueType::Positive()),
                                   Text("C1 swf cutoff")));
    parameters.push_back(Parameter("-cutoff",
                                   Value(myParams.cutoff_alg, ConstraintValueType::Positive()),
                                   Text("algorithm cutoff")));
  }

private:
  // one device context per force object: not copyable
  B200CutoffSystemForce(const B200CutoffSystemForce &);
  B200CutoffSystemForce &operator=(const B200CutoffSystemForce &);

  virtual Force *doMake(const std::vector<Value> &values) const {
    Real ron, rcLJ, rcC, rc;
    values[0].get(ron);
    values[1].get(rcLJ);
    values[2].get(rcC);
    values[3].get(rc);
    return new B200CutoffSystemForce(ron, rcLJ, rcC, rc, myParams.precision, myParams.device);
  }

  void setParams(Real ron, Real rcLJ, Real rcC, Real rc) {
    myParams.precision = PMB200_MIXED;
    myParams.device = 0;
    myParams.switchon = ron;
    myParams.cutoff_lj = rcLJ;
    myParams.cutoff_coul = rcC;
    myParams.cutoff_alg = rc;
    myParams.cellsize = 0.0;
  }

  void check(int rc) const {
    if (rc) THROW(std::string("B200 cutoff force: ") + pmb200_last_error(myCtx));
  }

  // Copies the topology arrays the pair function reads and the box.
  void upload(const RealTopologyType &t) {
    check(b200UploadTopology(myCtx, t));
    myCached = &t;
  }

  pmb200_params myParams;
  pmb200_ctx *myCtx;
  const GenericTopology *myCached;
};

}  // namespace ProtoMol

#endif  // PMB200_B200CUTOFFSYSTEMFORCE_H
