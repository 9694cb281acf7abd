/* -*- c++ -*- */
// ProtoMol SystemForce for the other cutoff registrations of
// NonbondedCutoffForceModule (protomol/src/protomol/module/
// NonbondedCutoffForceModule.cpp:53-134) on a B200 through libpmb200
// (pmb200_create_pair): OneAtomPair<BC, S, LennardJonesForce>,
// OneAtomPair<BC, S, CoulombForce> and OneAtomPairTwo<BC, S1,
// LennardJonesForce, S2, CoulombForce> with S among C1, C2, Cn and
// ComplimentCnCn (CmpCnCnSwitchingFunction), and OneAtomPair<BC,
// UniversalSwitchingFunction, LennardJonesTableForce<S, 7, Real>> with S
// among C2, Cn, ComplimentCnCn (id LennardJonesTable; NonbondedCutoffForce
// Module.cpp:67-72, 121-126), for periodic
// boundaries (BC = PeriodicBoundaryConditions) or vacuum
// (VacuumBoundaryConditions).  One prototype per (LJ switch, Coulomb switch)
// pair is registered under the algorithm keyword NonbondedCutoffB200; its id
// and parameter list follow the reference's (OneAtomPair::getId,
// OneAtomPairTwo::getId, NonbondedCutoffForce::getIdNoAlias and
// getParameters, .../force/nonbonded/NonbondedCutoffForce.h:81-91), e.g.
//   force LennardJones Coulomb -switchingFunction C2 -switchingFunction Cn
//         -algorithm NonbondedCutoffB200
//         -switchon 6.5 -cutoff 8 -n 4 -switchon 5 -switchoff 0 -cutoff 8 -cutoff 8
// Vacuum: the cell domain is the atoms' bounding box plus a margin of one
// cutoff, reset whenever an atom leaves it.  C++98, like the reference.
#ifndef PMB200_B200PAIRSYSTEMFORCE_H
#define PMB200_B200PAIRSYSTEMFORCE_H

#include <protomol/force/system/SystemForce.h>
#include <protomol/topology/Topology.h>
#include <protomol/topology/PeriodicBoundaryConditions.h>
#include <protomol/topology/VacuumBoundaryConditions.h>
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

template <class TBC>
class B200PairSystemForce : public SystemForce {
  typedef Topology<TBC, CubicCellManager> RealTopologyType;

public:
  // Prototype for (ljSwitch, coulombSwitch), each PMB200_SW_* (NONE: term
  // absent; ljSwitch | PMB200_SW_TABLE: the tabulated LJ).
  B200PairSystemForce(int ljSwitch, int coulombSwitch) : myCtx(0), myCached(0) {
    init(ljSwitch, coulombSwitch);
  }

  // A working force: p* = {switchon, cutoff, order, switchoff}.
  B200PairSystemForce(int ljSwitch, int coulombSwitch, const double *pl, const double *pc,
                      Real cutoff, int precision = PMB200_MIXED, int device = 0)
      : myCtx(0), myCached(0) {
    init(ljSwitch, coulombSwitch);
    for (int k = 0; k < 4; k++) {
      myParams.lj[k] = pl[k];
      myParams.coulomb[k] = pc[k];
    }
    myParams.cutoff_alg = cutoff;
    myParams.precision = precision;
    myParams.device = device;
    const int rc = pmb200_create_pair(&myParams, &myCtx);
    if (rc == PMB200_ECUDA)
      THROW("B200 cutoff force: no usable CUDA device " + toString(device) + ".");
    if (rc)
      THROW("B200 cutoff force " + getIdNoAlias() + ": parameters rejected (status " +
            toString(rc) + ").");
  }

  virtual ~B200PairSystemForce() { pmb200_destroy(myCtx); }

  virtual void evaluate(const GenericTopology *topo, const Vector3DBlock *positions,
                        Vector3DBlock *forces, ScalarStructure *energies) {
    run(topo, positions, forces, energies, false);
  }

  // SystemForce::parallelEvaluate: this rank's blocks of cells only, as
  // NonbondedCutoffSystemForce::parallelEvaluate does; Parallel::reduce sums
  // the ranks' shares.
  virtual void parallelEvaluate(const GenericTopology *topo, const Vector3DBlock *positions,
                                Vector3DBlock *forces, ScalarStructure *energies) {
    run(topo, positions, forces, energies, true);
  }

  // Force::numberOfBlocks: the Parallel::next() calls parallelEvaluate makes.
  // (For vacuum boundaries the grid follows the atoms' bounding box, which
  // ForceGroup fixes before it asks; every rank holds the same positions.)
  virtual unsigned int numberOfBlocks(const GenericTopology *topo, const Vector3DBlock *pos) {
    prepare(topo, pos);
    return b200NumberOfBlocks(myCtx);
  }

private:
  void prepare(const GenericTopology *topo, const Vector3DBlock *positions) {
    if (!myCtx) THROW("B200 cutoff force: evaluate called on the factory prototype.");
    const RealTopologyType *t = dynamic_cast<const RealTopologyType *>(topo);
    if (!t) THROW("B200 cutoff force: topology type does not match the force's boundaries.");
    if (myCached != topo) {
      upload(*t);
      myCached = topo;
    }
    if (TBC::VACUUM) updateDomain(positions);
  }

  void run(const GenericTopology *topo, const Vector3DBlock *positions, Vector3DBlock *forces,
           ScalarStructure *energies, bool parallel) {
    prepare(topo, positions);
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
  virtual void uncache() { myCached = 0; }
  virtual std::string getKeyword() const { return "NonbondedCutoffB200"; }

  virtual std::string getIdNoAlias() const {
    std::string id;
    if (myParams.lj_switch != PMB200_SW_NONE)
      id = (myParams.lj_switch & PMB200_SW_TABLE) ? "LennardJonesTable" : "LennardJones";
    if (myParams.coulomb_switch != PMB200_SW_NONE) id += id.empty() ? "Coulomb" : " Coulomb";
    if (myParams.lj_switch != PMB200_SW_NONE)
      id += " -switchingFunction " + switchName(base(myParams.lj_switch));
    if (myParams.coulomb_switch != PMB200_SW_NONE)
      id += " -switchingFunction " + switchName(myParams.coulomb_switch);
    return id + " -algorithm " + getKeyword();
  }

  virtual void getParameters(std::vector<Parameter> &parameters) const {
    if (myParams.lj_switch != PMB200_SW_NONE)
      switchParameters(base(myParams.lj_switch), myParams.lj, parameters);
    if (myParams.coulomb_switch != PMB200_SW_NONE)
      switchParameters(myParams.coulomb_switch, myParams.coulomb, parameters);
    parameters.push_back(Parameter("-cutoff",
                                   Value(myParams.cutoff_alg, ConstraintValueType::Positive()),
                                   Text("algorithm cutoff")));
  }

private:
  B200PairSystemForce(const B200PairSystemForce &);
  B200PairSystemForce &operator=(const B200PairSystemForce &);

  static int base(int kind) { return kind & ~PMB200_SW_TABLE; }
  static std::string switchName(int kind) {
    return kind == PMB200_SW_C1   ? "C1"
           : kind == PMB200_SW_C2 ? "C2"
           : kind == PMB200_SW_CN ? "Cn"
                                  : "ComplimentCnCn";
  }
  static int switchArity(int kind) {
    return kind == PMB200_SW_C1 ? 1 : kind == PMB200_SW_C2 ? 2 : 4;
  }

  // The switch's parameters as its getParameters lists them
  // (C1SwitchingFunction.cpp:18-22, C2SwitchingFunction.cpp:20-28,
  // CnSwitchingFunction.cpp:64-80, CmpCnCnSwitchingFunction.cpp:35-50).
  static void switchParameters(int kind, const double *p, std::vector<Parameter> &out) {
    const std::string n = switchName(kind);
    if (kind == PMB200_SW_CMPCNCN) {
      out.push_back(Parameter("-switchon", Value(p[0], ConstraintValueType::NotNegative()),
                              Text("CmpCnCn swf switch on")));
      out.push_back(Parameter("-switchoff", Value(p[3], ConstraintValueType::Positive()),
                              Text("CmpCnCn swf switchoff")));
      out.push_back(Parameter("-cutoff", Value(p[1], ConstraintValueType::Positive()),
                              Text("CmpCnCn swf cutoff")));
      out.push_back(Parameter("-n", Value(p[2], ConstraintValueType::Positive()), 2.0,
                              Text("CmpCnCn swf smoothness")));
      return;
    }
    if (kind == PMB200_SW_CN)
      out.push_back(Parameter("-n", Value(p[2], ConstraintValueType::Positive()),
                              Text(n + " swf smoothness")));
    if (kind != PMB200_SW_C1)
      out.push_back(Parameter("-switchon", Value(p[0], ConstraintValueType::NotNegative()),
                              Text(n + " swf switch on")));
    if (kind == PMB200_SW_CN)
      out.push_back(Parameter("-switchoff", Value(p[3], ConstraintValueType::NotNegative()),
                              0.0, Text(n + " swf switchoff")));
    out.push_back(Parameter("-cutoff", Value(p[1], ConstraintValueType::Positive()),
                            Text(n + " swf cutoff")));
  }

  // values: LJ switch parameters, Coulomb switch parameters, algorithm cutoff.
  virtual Force *doMake(const std::vector<Value> &values) const {
    double pl[4] = {0, 0, 0, 0}, pc[4] = {0, 0, 0, 0};
    unsigned int k = 0;
    const int kinds[2] = {myParams.lj_switch, myParams.coulomb_switch};
    double *dst[2] = {pl, pc};
    for (int s = 0; s < 2; s++) {
      if (kinds[s] == PMB200_SW_NONE) continue;
      Real v[4] = {0, 0, 0, 0};
      const int kd = base(kinds[s]);
      for (int a = 0; a < switchArity(kd); a++) values[k++].get(v[a]);
      if (kd == PMB200_SW_C1) { dst[s][1] = v[0]; }
      else if (kd == PMB200_SW_C2) { dst[s][0] = v[0]; dst[s][1] = v[1]; }
      else if (kd == PMB200_SW_CN) {
        dst[s][2] = v[0]; dst[s][0] = v[1]; dst[s][3] = v[2]; dst[s][1] = v[3];
      } else {  // ComplimentCnCn: switchon, switchoff, cutoff, n
        dst[s][0] = v[0]; dst[s][3] = v[1]; dst[s][1] = v[2]; dst[s][2] = v[3];
      }
    }
    Real rc;
    values[k].get(rc);
    return new B200PairSystemForce(kinds[0], kinds[1], pl, pc, rc, myParams.precision,
                                   myParams.device);
  }

  void init(int ljSwitch, int coulombSwitch) {
    myParams.precision = PMB200_MIXED;
    myParams.device = 0;
    myParams.lj_switch = ljSwitch;
    myParams.coulomb_switch = coulombSwitch;
    for (int k = 0; k < 4; k++) myParams.lj[k] = myParams.coulomb[k] = 0.0;
    myParams.cutoff_alg = 0.0;
    myParams.cellsize = 0.0;
    myLo[0] = myLo[1] = myLo[2] = 0.0;
    myHi[0] = myHi[1] = myHi[2] = -1.0;
  }

  void check(int rc) const {
    if (rc) THROW(std::string("B200 cutoff force: ") + pmb200_last_error(myCtx));
  }

  static int setBoundaries(pmb200_ctx *ctx, const PeriodicBoundaryConditions &bc) {
    return pmb200_set_box(ctx, bc.e1().c, bc.e2().c, bc.e3().c, bc.origin().c);
  }
  static int setBoundaries(pmb200_ctx *, const VacuumBoundaryConditions &) {
    return PMB200_OK;  // the domain follows the atoms (updateDomain)
  }

  void upload(const RealTopologyType &t) {
    check(b200UploadAtoms(myCtx, t));
    check(setBoundaries(myCtx, t.boundaryConditions));
    myHi[0] = myHi[1] = myHi[2] = -1.0;  // vacuum: domain set on the next evaluation
  }

  // Vacuum: keep the cell domain around the atoms.
  void updateDomain(const Vector3DBlock *positions) {
    const unsigned int n = positions->size();
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (unsigned int i = 0; i < n; i++)
      for (int a = 0; a < 3; a++) {
        const double x = (*positions)[i].c[a];
        if (i == 0 || x < lo[a]) lo[a] = x;
        if (i == 0 || x > hi[a]) hi[a] = x;
      }
    bool inside = true;
    for (int a = 0; a < 3; a++) inside = inside && lo[a] >= myLo[a] && hi[a] <= myHi[a];
    if (inside) return;
    const double m = myParams.cutoff_alg;
    for (int a = 0; a < 3; a++) {
      myLo[a] = lo[a] - m;
      myHi[a] = hi[a] + m;
    }
    check(pmb200_set_vacuum_domain(myCtx, myLo, myHi));
  }

  pmb200_pair_params myParams;
  pmb200_ctx *myCtx;
  const GenericTopology *myCached;
  double myLo[3], myHi[3];
};

}  // namespace ProtoMol

#endif  // PMB200_B200PAIRSYSTEMFORCE_H
