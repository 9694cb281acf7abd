/* CPU oracle for the periodic cutoff nonbonded system force.
 *
 * TEST INFRASTRUCTURE ONLY.  Tests, the smoke check and the CPU-baseline leg
 * of bench.py use this as the checker; the product never calls it.
 *
 * A plain C restatement of
 *   NonbondedCutoffSystemForce<CubicCellManager,
 *     OneAtomPairTwo<PeriodicBoundaryConditions, C2SwitchingFunction,
 *                    LennardJonesForce, C1SwitchingFunction, CoulombForce>>
 * from ProtoMol (protomol/src/protomol/...), following the reference's cell
 * build, cell-pair enumeration order and per-pair arithmetic operation by
 * operation, so that its FP64 results agree with the reference bit for bit on
 * the inputs the tests use.  Parity pins: the reference's own code compiled
 * from its sources (oracle/_ref/libpmref.so, recipe in oracle/Makefile) and
 * the reference's periodic water golden (test/tests/expected/
 * water_CHARMM_PERIODIC_L.energy, t = 0 energies), both checked in tests/.
 */
#ifndef PM_ORACLE_H
#define PM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int n;                 /* atoms */
  int ntypes;            /* LJ atom types */
  const int *type;       /* [n] LJ type index */
  const double *qscaled; /* [n] charge * SQRTCOULOMBCONSTANT */
  const int *mol;        /* [n] molecule id (0..nmol-1) */
  const double *mass;    /* [n] scaled mass; only for the molecular virial */
  const double *lj;      /* [ntypes*ntypes*4] {A, B, A14, B14} */
  int nexcl;             /* exclusion pairs */
  const int *excl;       /* [nexcl*3] {a1, a2, kind}; kind 1 modified, 2 full */
  double coulomb_scaling;/* topology coulombScalingFactor (1-4 Coulomb) */
  double box[3];         /* orthogonal cell basis lengths e1.x, e2.y, e3.z */
  double origin[3];      /* cellorigin */
  double cellsize;       /* CubicCellManager cellsize */
  double ron, rc_lj;     /* C2 switch (Lennard-Jones) */
  double rc_coul;        /* C1 switch (Coulomb) */
  double rc_alg;         /* NonbondedCutoff algorithm cutoff */
} pmo_system;

/* Error codes */
#define PMO_OK 0
#define PMO_EBADARG 1
#define PMO_ENOMEM 2

/* One SystemForce::evaluate.  pos: AoS double[3n] (not wrapped).  forces:
 * AoS double[3n], accumulated into.  energies[0] = Coulomb, [1] = LJ
 * (accumulated into).  virial_mode: 0 none, 1 atomic virial, 2 atomic +
 * molecular virial (virial/molvirial: 9 doubles, accumulated, may be NULL
 * when not requested).  brute: 0 = cell-list walk exactly as the reference,
 * 1 = all pairs i<j with the same per-pair code (the reference's
 * NonbondedSimpleFull cross-check). */
int pmo_eval(const pmo_system *s, const double *pos, double *forces,
             double *energies, double *virial, double *molvirial,
             int virial_mode, int brute);

/* Unique pairs (i<j, not fully excluded) inside max(rc_lj, rc_coul) under
 * the minimum image; the Gpairs/s unit. */
long long pmo_count_pairs(const pmo_system *s, const double *pos);

/* The real-space term of ProtoMol's Ewald sum,
 *   NonbondedFullEwaldSystemForce<PeriodicBoundaryConditions,
 *     CubicCellManager, real = true, reciprocal = false, correction = false,
 *     CutoffSwitchingFunction>
 * (registered in module/NonbondedFullElectrostaticForceModule.cpp:34 as
 * "Coulomb -algorithm FullEwald -real"): qq erfc(alpha r) / r for every pair
 * within rc = sqrt(-log(accuracy)) / alpha, MODIFIED pairs scaled by
 * coulomb_scaling, FULL pairs skipped.  alpha <= 0 selects the reference's
 * default.  exact_erfc 0 evaluates erfc with the Abramowitz & Stegun
 * polynomial of the reference's default build, 1 with libm erfc (the
 * reference built with -DUSE_EWALD_EXACT_ERF).  The cell walk uses the
 * system's cellsize and the cutoff rc; rc_lj/rc_coul/ron/rc_alg are ignored.
 * Every box edge must be >= 2 rc (no lattice images).  energies[0] (Coulomb)
 * is accumulated into; energies[1] is untouched. */
int pmo_eval_ewald_real(const pmo_system *s, double alpha, double accuracy,
                        int exact_erfc, const double *pos, double *forces,
                        double *energies, double *virial, double *molvirial,
                        int virial_mode, int brute);

/* out = {alpha, rc, 2 alpha / sqrt(pi), alpha^2} as the Ewald force derives
 * them (alpha <= 0: the reference's default from N and the volume). */
int pmo_ewald_constants(const pmo_system *s, double alpha, double accuracy,
                        double out[4]);

/* Unique pairs within the Ewald real-space cutoff (not fully excluded). */
long long pmo_count_pairs_ewald(const pmo_system *s, double alpha, double accuracy,
                                const double *pos);

/* Leapfrog with this force alone (LeapfrogIntegrator::run with no
 * modifiers): initial force, then per step kick (half on the first step) +
 * drift + force, and a closing half kick.  dt in fs. */
int pmo_leapfrog(const pmo_system *s, double *pos, double *vel,
                 const double *mass, double dt_fs, int nsteps,
                 double *energies);

/* SETTLE (Miyamoto & Kollman, J. Comput. Chem. 13, 952 (1992)): analytic
 * constraint of rigid 3-site waters.  widx[3*w] = {O, H1, H2}; every water
 * uses the masses of the first one.  new_pos (3n) holds unconstrained
 * positions on entry and constrained ones on return; old_pos satisfies the
 * constraints.  Not part of the reference (which constrains water with
 * iterative SHAKE, protomol/src/protomol/modifier/ModifierShake.cpp); the
 * tests check it against a converged SHAKE. */
void pmo_settle(int nwater, const int *widx, const double *mass, double doh,
                double dhh, const double *old_pos, double *new_pos);

/* pmo_leapfrog with rigid waters: after each kick + drift the listed waters
 * are put back on their constraints by SETTLE and their velocities become
 * (x_new - x_old) / h, as a position-constraint modifier does in ProtoMol's
 * leapfrog (postDriftOrNextModify).  The closing half kick is unconstrained. */
int pmo_leapfrog_rigid(const pmo_system *s, double *pos, double *vel,
                       const double *mass, double dt_fs, int nsteps, int nwater,
                       const int *widx, double doh, double dhh,
                       double *energies);

#ifdef __cplusplus
}
#endif
#endif
