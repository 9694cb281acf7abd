// Test infrastructure only: a thin C entry into the reference's own
// NonbondedCutoffSystemForce, compiled together with the reference sources
// (see oracle/Makefile) into oracle/_ref/libpmref.so.  Tests, the smoke check
// and the CPU-baseline leg of bench.py call it as the checker; nothing in the
// product links it.
//
// The force instantiated here is exactly the registered prototype
//   NonbondedCutoffSystemForce<CubicCellManager,
//     OneAtomPairTwo<PeriodicBoundaryConditions, C2SwitchingFunction,
//                    LennardJonesForce, C1SwitchingFunction, CoulombForce>>
// (protomol/src/protomol/module/NonbondedCutoffForceModule.cpp:75-76), built
// on a Topology<PeriodicBoundaryConditions, CubicCellManager> filled from flat
// arrays (protomol/src/protomol/topology/Topology.h:26-31).
#include <protomol/force/nonbonded/NonbondedCutoffSystemForce.h>
#include <protomol/force/nonbonded/NonbondedSimpleFullSystemForce.h>
#include <protomol/force/OneAtomPairTwo.h>
#include <protomol/force/LennardJonesForce.h>
#include <protomol/force/CoulombForce.h>
#include <protomol/switch/C1SwitchingFunction.h>
#include <protomol/switch/C2SwitchingFunction.h>
#include <protomol/topology/PeriodicBoundaryConditions.h>
#include <protomol/topology/CubicCellManager.h>
#include <protomol/topology/CellListEnumeratorPeriodicBoundaries.h>
#include <protomol/topology/Topology.h>
#include <protomol/topology/TopologyUtilities.h>
#include <protomol/topology/BuildTopology.h>
#include <protomol/type/ScalarStructure.h>
#include <protomol/type/Vector3DBlock.h>
#include <protomol/type/PSF.h>
#include <protomol/type/PAR.h>
#include <protomol/type/PDB.h>
#include <protomol/io/PSFReader.h>
#include <protomol/io/PARReader.h>
#include <protomol/io/PDBReader.h>
#include <protomol/base/PMConstants.h>
#include <protomol/base/Report.h>

#include <cstring>
#include <string>
#include <vector>

using namespace ProtoMol;

typedef Topology<PeriodicBoundaryConditions, CubicCellManager> PTopo;
typedef OneAtomPairTwo<PeriodicBoundaryConditions, C2SwitchingFunction,
                       LennardJonesForce, C1SwitchingFunction, CoulombForce>
  PPair;
typedef NonbondedCutoffSystemForce<CubicCellManager, PPair> PForce;

struct pmref_sys {
  PTopo *topo;
  PForce *force;
  Vector3DBlock pos, frc, vel;
  ScalarStructure energies;
  int n;
  double ron, rc_lj, rc_coul;  // the switches, for pmref_eval_allpairs
};

extern "C" {

// Builds a periodic topology + the reference force.  lj holds ntypes*ntypes
// records {A, B, A14, B14}; excl holds nexcl triples {a1, a2, kind} with kind
// 1 = modified (1-4), 2 = full.  mass (may be NULL) sets scaledMass and the
// molecule masses used by the molecular virial.
void *pmref_create(int n, const int *type, const double *qscaled,
                   const int *mol, const double *mass, int ntypes,
                   const double *lj, int nexcl, const int *excl,
                   double coulomb_scaling, const double box[3],
                   const double origin[3], double cellsize, double ron,
                   double rc_lj, double rc_coul, double rc_alg) {
  Report::report << Report::reportlevel(-4);
  pmref_sys *s = new pmref_sys();
  s->n = n;
  PeriodicBoundaryConditions bc(Vector3D(box[0], 0, 0), Vector3D(0, box[1], 0),
                                Vector3D(0, 0, box[2]),
                                Vector3D(origin[0], origin[1], origin[2]));
  s->topo = new PTopo(coulomb_scaling, ExclusionType(ExclusionType::ONE2),
                      bc, CubicCellManager(cellsize), 16.0f);
  PTopo &t = *s->topo;
  t.atoms.resize(n);
  int nmol = 0;
  for (int i = 0; i < n; i++) {
    t.atoms[i].type = type[i];
    t.atoms[i].scaledCharge = qscaled[i];
    t.atoms[i].molecule = mol[i];
    t.atoms[i].scaledMass = mass ? mass[i] : 1.0;
    t.atoms[i].cellListNext = -1;
    if (mol[i] + 1 > nmol) nmol = mol[i] + 1;
  }
  t.atomTypes.resize(ntypes);
  t.lennardJonesParameters.resize(ntypes);
  for (int a = 0; a < ntypes; a++)
    for (int b = 0; b < ntypes; b++) {
      const double *p = lj + 4 * (a * ntypes + b);
      t.lennardJonesParameters.set(a, b,
                                   LennardJonesParameters(p[0], p[1], p[2], p[3]));
    }
  t.molecules.resize(nmol);
  for (int m = 0; m < nmol; m++) t.molecules[m].mass = 0.0;
  for (int i = 0; i < n; i++) {
    t.molecules[mol[i]].atoms.push_back(i);
    t.molecules[mol[i]].mass += t.atoms[i].scaledMass;
  }
  t.exclusions.resize(n);
  for (int e = 0; e < nexcl; e++)
    t.exclusions.add(excl[3 * e], excl[3 * e + 1],
                     excl[3 * e + 2] == 1 ? EXCLUSION_MODIFIED : EXCLUSION_FULL);
  t.exclusions.optimize();
  s->pos.resize(n);
  s->frc.resize(n);
  s->vel.resize(n);
  s->ron = ron;
  s->rc_lj = rc_lj;
  s->rc_coul = rc_coul;
  s->force = new PForce(rc_alg, PPair(LennardJonesForce(),
                                      C2SwitchingFunction(ron, rc_lj),
                                      CoulombForce(),
                                      C1SwitchingFunction(rc_coul)));
  return s;
}

// A general periodic cell: PeriodicBoundaryConditions::set with any basis
// (the non-orthogonal minimal image of
// protomol/src/protomol/topology/PeriodicBoundaryConditions.h:62-67, 95-100);
// the cell lists are rebuilt at the next evaluation.
int pmref_set_box(void *h, const double e1[3], const double e2[3], const double e3[3],
                  const double origin[3]) {
  pmref_sys *s = (pmref_sys *)h;
  s->topo->boundaryConditions.set(Vector3D(e1[0], e1[1], e1[2]), Vector3D(e2[0], e2[1], e2[2]),
                                  Vector3D(e3[0], e3[1], e3[2]),
                                  Vector3D(origin[0], origin[1], origin[2]));
  s->topo->uncacheCellList();
  return 0;
}

// The same pair function over every pair i < j
// (NonbondedSimpleFullSystemForce, protomol/src/protomol/force/nonbonded/
// NonbondedSimpleFullSystemForce.h): no cell list, each pair at the minimal
// image of PeriodicBoundaryConditions::minimalDifference.  Arguments as
// pmref_eval.
int pmref_eval_allpairs(void *h, const double *pos, double *forces, double *energies,
                        double *virial, double *molvirial, int virial_mode) {
  pmref_sys *s = (pmref_sys *)h;
  const int n = s->n;
  NonbondedSimpleFullSystemForce<PPair> full(
      PPair(LennardJonesForce(), C2SwitchingFunction(s->ron, s->rc_lj), CoulombForce(),
            C1SwitchingFunction(s->rc_coul)));
  memcpy(s->pos.c, pos, sizeof(double) * 3 * n);
  memcpy(s->frc.c, forces, sizeof(double) * 3 * n);
  s->energies.clear();
  s->energies.virial(virial_mode >= 1);
  s->energies.molecularVirial(virial_mode >= 2);
  if (virial_mode >= 2) buildMolecularCenterOfMass(&s->pos, s->topo);
  full.evaluate(s->topo, &s->pos, &s->frc, &s->energies);
  memcpy(forces, s->frc.c, sizeof(double) * 3 * n);
  energies[0] = s->energies[ScalarStructure::COULOMB];
  energies[1] = s->energies[ScalarStructure::LENNARDJONES];
  if (virial)
    for (int k = 0; k < 9; k++)
      virial[k] = s->energies[(ScalarStructure::Index)(ScalarStructure::VIRIALXX + k)];
  if (molvirial)
    for (int k = 0; k < 9; k++)
      molvirial[k] =
        s->energies[(ScalarStructure::Index)(ScalarStructure::MOLVIRIALXX + k)];
  return 0;
}

// The Topology<PeriodicBoundaryConditions, CubicCellManager> built by
// pmref_create (for test harnesses that evaluate other forces on it).
void *pmref_topology(void *h) { return ((pmref_sys *)h)->topo; }

void pmref_destroy(void *h) {
  pmref_sys *s = (pmref_sys *)h;
  delete s->force;
  delete s->topo;
  delete s;
}

// One SystemForce::evaluate.  forces (3n, AoS) are ACCUMULATED into, like the
// reference; energies[0] = Coulomb, energies[1] = Lennard-Jones; virial (9)
// and molvirial (9) are written when the flags ask for them (virial_mode 0 =
// none, 1 = atomic, 2 = atomic + molecular).
int pmref_eval(void *h, const double *pos, double *forces, double *energies,
               double *virial, double *molvirial, int virial_mode) {
  pmref_sys *s = (pmref_sys *)h;
  const int n = s->n;
  memcpy(s->pos.c, pos, sizeof(double) * 3 * n);
  memcpy(s->frc.c, forces, sizeof(double) * 3 * n);
  s->energies.clear();
  s->energies.virial(virial_mode >= 1);
  s->energies.molecularVirial(virial_mode >= 2);
  if (virial_mode >= 2) buildMolecularCenterOfMass(&s->pos, s->topo);
  s->topo->uncacheCellList();
  s->force->evaluate(s->topo, &s->pos, &s->frc, &s->energies);
  memcpy(forces, s->frc.c, sizeof(double) * 3 * n);
  energies[0] = s->energies[ScalarStructure::COULOMB];
  energies[1] = s->energies[ScalarStructure::LENNARDJONES];
  if (virial)
    for (int k = 0; k < 9; k++)
      virial[k] = s->energies[(ScalarStructure::Index)(ScalarStructure::VIRIALXX + k)];
  if (molvirial)
    for (int k = 0; k < 9; k++)
      molvirial[k] =
        s->energies[(ScalarStructure::Index)(ScalarStructure::MOLVIRIALXX + k)];
  return 0;
}

// Leapfrog steps with this force alone, following
// LeapfrogIntegrator::run / doKickdoDrift
// (protomol/src/protomol/integrator/leapfrog/LeapfrogIntegrator.cpp:58-105)
// with no modifiers: half kick + drift, force, (kick + drift, force)*, half
// kick.  dt in fs; pos/vel (3n) are updated in place; mass per atom.
int pmref_leapfrog(void *h, double *pos, double *vel, const double *mass,
                   double dt_fs, int nsteps, double *energies) {
  pmref_sys *s = (pmref_sys *)h;
  const int n = s->n;
  const double hstep = dt_fs * Constant::INV_TIMEFACTOR;
  std::vector<double> f(3 * n, 0.0);
  double e[2] = {0, 0};
  // initial forces
  pmref_eval(h, pos, &f[0], e, NULL, NULL, 0);
  for (int step = 0; step < nsteps; step++) {
    const double kick = (step == 0) ? 0.5 * hstep : hstep;
    for (int i = 0; i < n; i++)
      for (int k = 0; k < 3; k++) vel[3 * i + k] += f[3 * i + k] * kick / mass[i];
    for (int i = 0; i < 3 * n; i++) pos[i] += vel[i] * hstep;
    for (int i = 0; i < 3 * n; i++) f[i] = 0.0;
    pmref_eval(h, pos, &f[0], e, NULL, NULL, 0);
  }
  for (int i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) vel[3 * i + k] += f[3 * i + k] * 0.5 * hstep / mass[i];
  if (energies) {
    energies[0] = e[0];
    energies[1] = e[1];
  }
  return 0;
}

// Reads a PSF/PAR/PDB triple with the reference's own readers and topology
// builder (protomol/src/protomol/module/IOModule.cpp:160-190,
// protomol/src/protomol/topology/BuildTopology.cpp) and exports the arrays the
// nonbonded force consumes.  Call once with out pointers NULL to get the
// counts (n, ntypes, nexcl), then again with buffers of those sizes.
int pmref_load_psf(const char *psf_file, const char *par_file,
                   const char *pdb_file, const char *exclude,
                   int *n_out, int *ntypes_out, int *nexcl_out, double *pos,
                   int *type, double *qscaled, int *mol, double *mass,
                   double *lj, int *excl) {
  Report::report << Report::reportlevel(-4);
  PSF psf;
  PAR par;
  PSFReader psfReader;
  if (!psfReader.open(psf_file) || !(psfReader >> psf)) return 1;
  PARReader parReader;
  if (!parReader.open(par_file) || !(parReader >> par)) return 2;
  PDBReader pdbReader(pdb_file);
  PDB pdb;
  if (!(pdbReader >> pdb)) return 3;
  PTopo topo(1.0, ExclusionType(exclude), PeriodicBoundaryConditions(),
             CubicCellManager(1.0), 16.0f);
  buildTopology(&topo, psf, par,
                parReader.getCharmmTypeDetected() != PAR::CHARMM28, NULL);
  const int n = topo.atoms.size();
  const int nt = topo.atomTypes.size();
  const std::vector<ExclusionPair> &tab = topo.exclusions.getTable();
  *n_out = n;
  *ntypes_out = nt;
  *nexcl_out = tab.size();
  if (!pos) return 0;
  for (int i = 0; i < n; i++) {
    for (int k = 0; k < 3; k++) pos[3 * i + k] = pdb.coords[i].c[k];
    type[i] = topo.atoms[i].type;
    qscaled[i] = topo.atoms[i].scaledCharge;
    mol[i] = topo.atoms[i].molecule;
    mass[i] = topo.atoms[i].scaledMass;
  }
  for (int a = 0; a < nt; a++)
    for (int b = 0; b < nt; b++) {
      const LennardJonesParameters &p = topo.lennardJonesParameters(a, b);
      double *o = lj + 4 * (a * nt + b);
      o[0] = p.A; o[1] = p.B; o[2] = p.A14; o[3] = p.B14;
    }
  for (size_t e = 0; e < tab.size(); e++) {
    excl[3 * e] = tab[e].a1;
    excl[3 * e + 1] = tab[e].a2;
    excl[3 * e + 2] = (int)tab[e].excl;
  }
  return 0;
}

}  // extern "C"
