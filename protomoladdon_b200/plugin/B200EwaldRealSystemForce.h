/* -*- c++ -*- */
// ProtoMol SystemForce that evaluates the real-space term of the Ewald sum on
// a B200 through libpmb200 (include/pmb200.h, pmb200_create_ewald_real).
//
// It stands where ProtoMol registers
//   NonbondedFullEwaldSystemForce<PeriodicBoundaryConditions,
//     CubicCellManager, true, false, false, CutoffSwitchingFunction>
// (protomol/src/protomol/module/NonbondedFullElectrostaticForceModule.cpp:34,
// id "Coulomb -algorithm FullEwald -real") under its own algorithm keyword,
// FullEwaldB200, because duplicate ids throw
// (protomol/src/protomol/base/Factory.h:50-58).  Parameters in the
// reference's order and with its defaults
// (NonbondedFullEwaldSystemForce::getParameters, .../force/nonbonded/
// NonbondedFullEwaldSystemForce.h:1226-1235): -alpha (default -1: derived
// from N and the volume) and -accuracy (default 1e-5).  The erfc form is the
// reference's default build's (Abramowitz & Stegun polynomial) unless the
// host compiles this header with USE_EWALD_EXACT_ERF, as the reference's
// own switch does.  C++98, like the reference.
#ifndef PMB200_B200EWALDREALSYSTEMFORCE_H
#define PMB200_B200EWALDREALSYSTEMFORCE_H

#include <protomol/force/system/SystemForce.h>
#include <protomol/force/CoulombForce.h>
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

class B200EwaldRealSystemForce : public SystemForce {
  typedef Topology<PeriodicBoundaryConditions, CubicCellManager> RealTopologyType;

public:
  // Prototype for the factory (no device context).
  B200EwaldRealSystemForce() : myCtx(0), myCached(0) { setParams(-1.0, 0.00001); }

  // A working force; the parameters are checked like the reference's doMake
  // (a valid alpha; accuracy > 0 from its Positive constraint).
  B200EwaldRealSystemForce(Real alpha, Real accuracy, int precision = PMB200_MIXED,
                           int device = 0)
      : myCtx(0), myCached(0) {
    setParams(alpha, accuracy);
    myParams.precision = precision;
    myParams.device = device;
    const int rc = pmb200_create_ewald_real(&myParams, &myCtx);
    if (rc == PMB200_ECUDA)
      THROW("B200 Ewald real-space force: no usable CUDA device " + toString(device) + ".");
    if (rc)
      THROW("B200 Ewald real-space force: parameters rejected (status " + toString(rc) +
            "); need 0 < accuracy < 1.");
  }

  virtual ~B200EwaldRealSystemForce() { pmb200_destroy(myCtx); }

  // SystemForce::evaluate (protomol/src/protomol/force/system/SystemForce.h:
  // 32-35): forces accumulated into; the term's energy is added to COULOMB,
  // the virial and molecular virial when the ScalarStructure asks for them.
  virtual void evaluate(const GenericTopology *topo, const Vector3DBlock *positions,
                        Vector3DBlock *forces, ScalarStructure *energies) {
    run(topo, positions, forces, energies, false);
  }

  // SystemForce::parallelEvaluate: this rank's blocks of cells only (the
  // reference's Ewald force deals its work through Parallel::next() too,
  // NonbondedFullEwaldSystemForce.h:115, 518-540); Parallel::reduce sums
  // the ranks' shares.
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
    if (!myCtx) THROW("B200 Ewald real-space force: evaluate called on the factory prototype.");
    const RealTopologyType *t = dynamic_cast<const RealTopologyType *>(topo);
    if (!t) THROW("B200 Ewald real-space force: needs periodic boundaries and the cubic cell manager.");
    if (myCached != topo) {
      check(b200UploadTopology(myCtx, *t));
      myCached = topo;
    }
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
    for (int k = 0; k < 9; k++) {
      if (flags & PMB200_VIRIAL)
        (*energies)[(ScalarStructure::Index)(ScalarStructure::VIRIALXX + k)] += vir[k];
      if (flags & PMB200_MOLVIRIAL)
        (*energies)[(ScalarStructure::Index)(ScalarStructure::MOLVIRIALXX + k)] += mvir[k];
    }
  }

public:
  virtual void uncache() { myCached = 0; }

  virtual std::string getKeyword() const { return "FullEwaldB200"; }

  // The reference's id form (NonbondedFullEwaldSystemForce.h:1203-1215)
  // with only the real-space term.
  virtual std::string getIdNoAlias() const {
    return CoulombForce::keyword + " -algorithm " + getKeyword() + " -real";
  }

  virtual void getParameters(std::vector<Parameter> &parameters) const {
    parameters.push_back(Parameter("-alpha", Value(myParams.alpha), -1.0, Text("splitting")));
    parameters.push_back(Parameter("-accuracy",
                                   Value(myParams.accuracy, ConstraintValueType::Positive()),
                                   0.00001));
  }
  virtual unsigned int getParameterSize() const { return 2; }

private:
  B200EwaldRealSystemForce(const B200EwaldRealSystemForce &);
  B200EwaldRealSystemForce &operator=(const B200EwaldRealSystemForce &);

  virtual Force *doMake(const std::vector<Value> &values) const {
    std::string err;
    if (!values[0].valid()) err += " alpha '" + values[0].getString() + "' not valid.";
    if (!values[1].valid()) err += " accuracy '" + values[1].getString() + "' not valid.";
    if (!err.empty()) THROW(" force " + getKeyword() + " :" + err);
    Real alpha, accuracy;
    values[0].get(alpha);
    values[1].get(accuracy);
    return new B200EwaldRealSystemForce(alpha, accuracy, myParams.precision, myParams.device);
  }

  void setParams(Real alpha, Real accuracy) {
    myParams.precision = PMB200_MIXED;
    myParams.device = 0;
#ifdef USE_EWALD_EXACT_ERF
    myParams.erfc = PMB200_ERFC_EXACT;
#else
    myParams.erfc = PMB200_ERFC_POLY5;
#endif
    myParams.alpha = alpha;
    myParams.accuracy = accuracy;
    myParams.cellsize = 0.0;
  }

  void check(int rc) const {
    if (rc) THROW(std::string("B200 Ewald real-space force: ") + pmb200_last_error(myCtx));
  }

  pmb200_ewald_params myParams;
  pmb200_ctx *myCtx;
  const GenericTopology *myCached;
};

}  // namespace ProtoMol

#endif  // PMB200_B200EWALDREALSYSTEMFORCE_H
