/* pmb200 -- B200 (sm_100a) periodic cutoff nonbonded system force.
 *
 * C ABI of libpmb200.so: plain pointers, sizes and int status codes; no C++
 * or CUDA types cross it.  It replaces ProtoMol's
 *
 *   NonbondedCutoffSystemForce<CubicCellManager,
 *     OneAtomPairTwo<PeriodicBoundaryConditions, C2SwitchingFunction,
 *                    LennardJonesForce, C1SwitchingFunction, CoulombForce>>
 *
 * registered at protomol/src/protomol/module/NonbondedCutoffForceModule.cpp:
 * 75-76 and selected in a config by
 *   force LennardJones Coulomb -algorithm NonbondedCutoff
 *         -switchingFunction C2 -switchingFunction C1
 *         -switchon <ron> -cutoff <rc_lj> -cutoff <rc_coul> -cutoff <rc_alg>
 * (parameter order: OneAtomPairTwo::getParameters,
 * protomol/src/protomol/force/OneAtomPairTwo.h:127-132, then
 * NonbondedCutoffForce::getParameters, .../nonbonded/NonbondedCutoffForce.h:
 * 85-91).  Every function returns 0 on success or a PMB200_E* code; the text
 * of the last error is available from pmb200_last_error().  Nothing throws
 * across this boundary.
 *
 * Units are ProtoMol's: Angstrom, kcal/mol, amu, charges pre-scaled by
 * SQRTCOULOMBCONSTANT (Atom::scaledCharge).  Arrays are caller-owned host
 * memory unless a name says "device".
 */
#ifndef PMB200_H
#define PMB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define PMB200_OK 0
#define PMB200_EINVAL 1      /* bad argument (message says which) */
#define PMB200_ECUDA 2       /* CUDA runtime error */
#define PMB200_ESTATE 3      /* call order: topology/box not set */
#define PMB200_EUNSUPPORTED 4/* valid in ProtoMol but outside this force */
#define PMB200_EDEVICE 5     /* device-side check failed (non-finite input) */
#define PMB200_ENOMEM 6

/* ---- precision of the pair arithmetic ---- */
#define PMB200_MIXED 0 /* FP32 pair math, int64 fixed-point forces, FP64 totals */
#define PMB200_FP64 1  /* plain FP64 pair math */

/* ---- what an evaluation produces (bit flags) ---- */
#define PMB200_ENERGY 1u     /* LENNARDJONES and COULOMB energies */
#define PMB200_VIRIAL 2u     /* atomic virial (9) */
#define PMB200_MOLVIRIAL 4u  /* molecular virial (9); needs masses */

typedef struct pmb200_ctx pmb200_ctx;

/* Construction parameters.  Replaces the force-id parse
 * ForceFactory::make -> NonbondedCutoffForce::doMake -> OneAtomPairTwo::make
 * -> C2SwitchingFunction::make / C1SwitchingFunction::make
 * (protomol/src/protomol/factory/ForceFactory.cpp:21-242,
 *  .../force/nonbonded/NonbondedCutoffForce.h:71-75,
 *  .../force/OneAtomPairTwo.h:142-155,
 *  .../switch/C2SwitchingFunction.cpp:30-41, C1SwitchingFunction.cpp:25-27).
 * C2 validation is the reference's: 0 <= switchon < cutoff_lj. */
typedef struct {
  int precision;      /* PMB200_MIXED or PMB200_FP64 */
  int device;         /* CUDA device ordinal */
  double switchon;    /* C2 -switchon (Lennard-Jones) */
  double cutoff_lj;   /* C2 -cutoff */
  double cutoff_coul; /* C1 -cutoff */
  double cutoff_alg;  /* algorithm -cutoff; must be >= both switch cutoffs */
  double cellsize;    /* grid cell edge hint; 0 = max(cutoff_lj, cutoff_coul)/2 */
} pmb200_params;

/* Replaces constructing the force prototype + ForceGroup ownership
 * (protomol/src/protomol/force/ForceGroup.cpp:31-52). */
int pmb200_create(const pmb200_params *params, pmb200_ctx **out);
int pmb200_destroy(pmb200_ctx *ctx);
const char *pmb200_last_error(const pmb200_ctx *ctx);

/* Topology the force reads (replaces the per-evaluation reads of
 * GenericTopology in OneAtomPairTwo::doOneAtomPair,
 * protomol/src/protomol/force/OneAtomPairTwo.h:57-125):
 *   type[n]      Atom::type (index into the LJ table)
 *   q_scaled[n]  Atom::scaledCharge
 *   molecule[n]  Atom::molecule
 *   mass[n]      Atom::scaledMass (may be NULL; needed for PMB200_MOLVIRIAL
 *                and the integrator)
 *   lj[ntypes*ntypes*4]  LennardJonesParameterTable {A, B, A14, B14}
 *                (protomol/src/protomol/topology/LennardJonesParameterTable.h:34-36);
 *                ntypes <= 1024 (the derivative kernels: <= 39; batches: <= 16)
 *   excl[nexcl*3]  ExclusionTable entries {a1, a2, kind}, kind 1 =
 *                EXCLUSION_MODIFIED, 2 = EXCLUSION_FULL; later duplicates
 *                override earlier ones like ExclusionTable::add
 *                (protomol/src/protomol/topology/ExclusionTable.cpp:103-120)
 *   coulomb_scaling  GenericTopology::coulombScalingFactor
 * Copies everything to the device. */
int pmb200_set_topology(pmb200_ctx *ctx, int n, const int *type,
                        const double *q_scaled, const int *molecule,
                        const double *mass, int ntypes, const double *lj,
                        int nexcl, const int *excl, double coulomb_scaling);

/* Periodic cell (replaces PeriodicBoundaryConditions::set,
 * protomol/src/protomol/topology/PeriodicBoundaryConditions.cpp:32-77).
 * Any basis e1, e2, e3 (origin = the cell's centre).  Orthogonal boxes: every
 * edge >= 2 * max switch cutoff.  General cells: pairs are taken at the
 * reference's minimal image (PeriodicBoundaryConditions.h:62-67: fractional
 * differences rounded to the nearest lattice vector); the distance between
 * opposite faces must be about 3 cutoffs or more (each axis must hold
 * 2 ceil(rc / cell width) + 1 cells of at least rc / 4; PMB200_EUNSUPPORTED
 * otherwise).  Batches take orthogonal boxes only. */
int pmb200_set_box(pmb200_ctx *ctx, const double e1[3], const double e2[3],
                   const double e3[3], const double origin[3]);

/* One SystemForce::evaluate
 * (protomol/src/protomol/force/nonbonded/NonbondedCutoffSystemForce.h:42-53)
 * on host buffers.  pos[3n] AoS positions (not wrapped).  forces[3n] AoS:
 * ACCUMULATED into, like the reference.  energies[2] = {COULOMB,
 * LENNARDJONES}: accumulated into (may be NULL when !(flags&ENERGY)).
 * virial[9], molvirial[9] row-major xx..zz: accumulated into when the flag is
 * set (else may be NULL).  A PMB200_MIXED context's forces reach the host in
 * FP32 (its kernels' forces are good to ~1e-6; the device entry points return
 * them in FP64). */
int pmb200_eval(pmb200_ctx *ctx, const double *pos, double *forces,
                double *energies, double *virial, double *molvirial,
                unsigned flags);

/* The share of one rank in the reference's parallel evaluation
 * (NonbondedCutoffSystemForce::parallelEvaluate,
 * protomol/src/protomol/force/nonbonded/NonbondedCutoffSystemForce.h:57-77,
 * which splits its cells into numberOfBlocks() ranges and evaluates the
 * ranges Parallel::next() grants; Parallel::reduce then sums forces and
 * energies over the ranks, force/ForceGroup.cpp:79-116).  Evaluates on host
 * buffers only the pairs whose i-cell (this library's grid, pmb200_grid) lies
 * in [cell_lo, cell_hi): with the mixed kernel the half-shell pairs of those
 * cells, with the FP64 kernel the forces on their atoms and half their pair
 * energies.  Arguments and accumulation as pmb200_eval; over a partition of
 * [0, number of cells) the shares sum to pmb200_eval's result. */
int pmb200_eval_cells(pmb200_ctx *ctx, const double *pos, double *forces,
                      double *energies, double *virial, double *molvirial,
                      unsigned flags, int cell_lo, int cell_hi);

/* Same evaluation on device buffers, asynchronous on `stream` (a
 * cudaStream_t, NULL = the context's stream).  d_pos[3n], d_forces[3n]
 * (accumulated into), d_out[20] receives {COULOMB, LENNARDJONES, virial[9],
 * molvirial[9]} (overwritten, FP64) when flags ask for them; may be NULL
 * when flags == 0.  Errors detected on the device are reported by the next
 * pmb200_sync(). */
int pmb200_eval_device(pmb200_ctx *ctx, const double *d_pos, double *d_forces,
                       double *d_out, unsigned flags, void *stream);

/* Autotuner of one context's evaluation.  Times the whole evaluation (cell
 * build, pair kernel, force finalisation, reductions) on the device
 * positions d_pos[3n], reps timed launches per configuration (median), with
 * and without energies, over the grid's cell size (hints cutoff / 1.5, / 2,
 * / 2.5, / 3, / 3.5, / 4, each as pmb200_params::cellsize; hints that give
 * the same grid are timed once, grids the stencil limits refuse are skipped)
 * and, for PMB200_MIXED contexts, the pair kernel (search or cluster-pair,
 * see pmb200_set_pair_kernel) and its warps per i-cell (2, 4, 8), chosen
 * separately for energy launches and forces-only launches, then the
 * supercluster kernel on the chosen grid where it applies; keeps the grid
 * with the fastest evaluation with energies (the reference's integrators
 * ask for energies every step) and applies it.  The library's defaults are
 * timed first and another configuration replaces them only when it is 2%
 * faster (timing noise between near-equal ones does not move the choice).  The choice is cached for the
 * process under a key of the device, the force (kind, precision, cutoffs,
 * switches), the atom and type counts and the box: a later context with the
 * same key takes it without timing.  result[8] (may be NULL) = {cell-size
 * hint, warps per i-cell with energies, warps per i-cell forces-only (0 for
 * FP64), ms with energies, ms forces-only, configurations timed (0: taken
 * from the cache), pair kernel with energies, pair kernel forces-only
 * (PMB200_KERNEL_*)}.  Forces and energies after tuning agree with the
 * untuned ones to the kernel's precision (the cell grid sets the FP32
 * cell-unit coordinates).  The device work runs on `stream` (NULL: the
 * context's) and is synchronised. */
int pmb200_autotune(pmb200_ctx *ctx, const double *d_pos, void *stream, int reps,
                    double result[8]);

/* The mixed pair kernel of a context.  PMB200_KERNEL_SEARCH (the default):
 * per-atom candidate search in every evaluation (culled staging, per-lane
 * lists).  PMB200_KERNEL_TILES: cluster pairs -- runs of 4 atoms of a cell
 * (sorted by height) as clusters, one bounding-box test per cluster pair,
 * and 4 x 4 tiles of atom pairs evaluated with masks; the same pair set and
 * pair arithmetic.  The tile kernel serves the cutoff and real-space Ewald
 * forms of mixed contexts without virial on orthogonal grids with at most
 * 16 LJ types; other evaluations of the context use the search kernel.
 * PMB200_KERNEL_CLUSTERS: superclusters -- each super-column's atoms cut by
 * height into groups of 32, each split into eight 4-atom clusters (2 x 2 x 2);
 * per group a list of the clusters within the cutoff with atom-pair masks
 * (exclusions, each pair once), built on the device at every evaluation;
 * 4 x 4 tiles evaluated with the exact cutoff test and the same pair
 * arithmetic.  It serves energy and forces-only evaluations of the mixed
 * cutoff form (LJ(C2) + Coulomb(C1)) without virial, in orthogonal periodic
 * boxes whose x and y edges hold at least five 32-atom columns across the
 * cutoff (about 2 rc + 14 A at water density), with at most 16 LJ types and
 * no modified (1-4) pairs; other evaluations use the search kernel.  A
 * system packed too densely or sparsely for its lists makes the evaluation
 * report PMB200_EDEVICE (PMB200_KERNEL_SEARCH then serves it). */
#define PMB200_KERNEL_SEARCH 0
#define PMB200_KERNEL_TILES 1
#define PMB200_KERNEL_CLUSTERS 2
int pmb200_set_pair_kernel(pmb200_ctx *ctx, int kernel);

/* Force decomposition over several GPUs, one process and one context per GPU,
 * every context holding the same topology, box and positions: the
 * replicated-data decomposition of the reference's parallel evaluation
 * (NonbondedCutoffSystemForce::parallelEvaluate, protomol/src/protomol/force/
 * nonbonded/NonbondedCutoffSystemForce.h:57-77, which deals contiguous runs
 * of cell pairs to the ranks and sums the forces with MPI; here contiguous
 * runs of i-cells).  Shard `shard` of `nshards` evaluates the half-shell pairs
 * of the i-cells [ncell * shard / nshards, ncell * (shard + 1) / nshards)
 * into d_facc[3n] (int64, overwritten): the forces in the library's fixed
 * point, an opaque layout whose only use is an element-wise integer sum over
 * the shards (an all-reduce with ncclInt64 / ncclSum, say), exact whatever
 * the reduction order.  d_out[20] (overwritten when flags ask for it)
 * receives the shard's share of the energies and virials, as for
 * pmb200_eval_device; the caller sums these too.  pmb200_shard_finalize then
 * adds the forces of the summed accumulator to d_forces[3n] (caller order,
 * accumulated into, as pmb200_eval_device) using the cell order of this
 * context's latest shard evaluation (the same on every shard: the cell build
 * is deterministic).  The summed forces equal a single pmb200_eval_device
 * bit for bit.  Mixed-precision contexts only. */
int pmb200_shard_eval_device(pmb200_ctx *ctx, const double *d_pos, int shard, int nshards,
                             long long *d_facc, double *d_out, unsigned flags, void *stream);
int pmb200_shard_finalize(pmb200_ctx *ctx, const long long *d_facc, double *d_forces,
                          void *stream);

/* Waits for the context's work and reports device-side check failures. */
int pmb200_sync(pmb200_ctx *ctx);

/* Leapfrog steps on device memory with this force alone, following
 * LeapfrogIntegrator::run / doKickdoDrift without modifiers
 * (protomol/src/protomol/integrator/leapfrog/LeapfrogIntegrator.cpp:58-105):
 * forces at the start, then per step a kick (a half kick on the first step)
 * and a drift, new forces; a closing half kick.  dt_fs in fs.  d_pos[3n],
 * d_vel[3n] updated in place; d_forces[3n] holds the final forces.  Steps
 * after the first run as one captured CUDA graph.  d_out as for
 * pmb200_eval_device, for the final step's forces. */
int pmb200_leapfrog_device(pmb200_ctx *ctx, double *d_pos, double *d_vel,
                           double *d_forces, double *d_out, double dt_fs,
                           int nsteps, unsigned flags, void *stream);

/* One steady-state leapfrog iteration on device memory: doKickdoDrift()
 * then calculateForces() (LeapfrogIntegrator::run's loop body,
 * protomol/src/protomol/integrator/leapfrog/LeapfrogIntegrator.cpp:98-101):
 * v += F h / m, x += v h, then d_forces is OVERWRITTEN with the forces at the
 * new positions (StandardIntegrator::calculateForces zeroes forces first,
 * .../integrator/StandardIntegrator.cpp:48).  Replays a CUDA graph captured on
 * the first call for the same buffers and stream (the stream must not be the
 * legacy default stream). */
int pmb200_step_device(pmb200_ctx *ctx, double *d_pos, double *d_vel,
                       double *d_forces, double *d_out, double dt_fs,
                       unsigned flags, void *stream);

/* Rigid 3-site waters for the device integrator (pmb200_leapfrog_device,
 * pmb200_step_device): after each kick + drift the listed waters are put
 * back on their O-H (d_oh) and H-H (d_hh) lengths by SETTLE and their
 * velocities become (x_new - x_old) / h, the effect of ProtoMol's SHAKE
 * position modifier on a water (protomol/src/protomol/modifier/
 * ModifierShake.cpp, run by LeapfrogIntegrator's postDriftOrNextModify).
 * widx[3*nwater] = {O, H1, H2} per water; all waters must share the first
 * one's masses.  nwater = 0 turns the constraints off. */
int pmb200_set_rigid_waters(pmb200_ctx *ctx, int nwater, const int *widx,
                            double d_oh, double d_hh);

/* When on, CUDA events bracket every directly launched pair kernel
 * (pmb200_eval, pmb200_eval_device; not graph replays);
 * pmb200_last_kernel_ms returns the duration of the last one (valid after
 * the work has completed). */
int pmb200_set_kernel_timing(pmb200_ctx *ctx, int on);
int pmb200_last_kernel_ms(pmb200_ctx *ctx, float *ms);

/* Unique in-cutoff pairs found by the last evaluation (the pair count the
 * Gpairs/s unit counts; fully excluded pairs are not counted).  Requires a
 * pmb200_sync() after the evaluation. */
int pmb200_last_pair_count(pmb200_ctx *ctx, long long *pairs);

/* Host-side integrator helper for callers that keep the state on the host
 * and call pmb200_eval per step (a ProtoMol integrator driving this force):
 * one LeapfrogIntegrator::doKickdoDrift (v += F kick h / m, x += v h,
 * protomol/src/protomol/integrator/leapfrog/LeapfrogIntegrator.cpp:72-85)
 * followed, for the listed rigid waters, by SETTLE and v = (x_new - x_old)/h
 * (the role of ProtoMol's SHAKE modifier).  kick is 1 for a full kick, 0.5
 * for the first half kick.  An atom belongs to at most one water
 * (PMB200_EINVAL otherwise); each water's atoms are kicked, drifted and
 * constrained in one pass.  clear_forces != 0: each force entry is set to
 * zero once it has been used, ready for the next evaluation to add into (the
 * myForces->zero() of StandardIntegrator::calculateForces,
 * .../integrator/StandardIntegrator.cpp:44-48), in the same pass.  Runs on the host (OpenMP threads for
 * large systems); no GPU. */
int pmb200_host_kick_drift(int n, double *pos, double *vel,
                           double *forces, const double *mass,
                           double dt_fs, double kick, int nwater,
                           const int *widx, double d_oh, double d_hh,
                           int clear_forces);

/* Measurement helper (no counterpart in the reference): FP32 FMA throughput
 * of `device` in TFLOP/s (2 flops per FMA), from a 148-SM-filling chain of
 * independent fused multiply-adds timed with CUDA events.  The pair kernels
 * are bounded by this pipe, not by HBM or tensor cores. */
int pmb200_measure_fp32_peak(int device, double *tflops);

/* Mixed-precision evaluation that allocates no memory (no counterpart in the
 * reference: ProtoMol's force owns heap-allocated cell lists).  For callers
 * that must not allocate device memory -- hosts that give all device memory
 * to their own pool allocator and forbid libraries to take more, or that
 * cannot afford cudaFree's implicit device synchronisation inside a time
 * step.  It needs no pmb200_ctx: every input and output is the caller's,
 * and the scratch (cell lists, sorted copies, fixed-point accumulators,
 * partial sums) lives in one statically sized device array inside the
 * library, held on every device that loads it until the process exits.
 *
 * Limits: n <= 32768 atoms and at most 8192 grid cells (PMB200_ENOMEM
 * beyond either), at most 16 LJ types, precision PMB200_MIXED only.
 * Inputs: device arrays d_pos[3n], d_type[n], d_q[n] (scaledCharge),
 * d_mol[n], and the exclusions as per-atom lists sorted by partner:
 * d_ex_start[n+1] offsets into d_ex, which holds int pairs {partner atom,
 * kind} (kind 1 = modified, 2 = full; each pair listed under both of its
 * atoms; 8-byte aligned); host arrays lj[ntypes^2*4]
 * {A, B, A14, B14} (finite), box[3] (orthogonal edges), origin[3].
 * Outputs: d_forces[3n] is OVERWRITTEN with this evaluation's forces;
 * d_energy (may be NULL: a forces-only evaluation) receives exactly two
 * doubles {COULOMB, LENNARDJONES} and nothing beyond them; d_status (may be
 * NULL) receives one int when the work completes: PMB200_OK, or
 * PMB200_EDEVICE when a device-side check failed (a non-finite coordinate,
 * or a pair force beyond the fixed-point range, as for coincident atoms) --
 * the forces and energies of such a call are not meaningful.  With
 * d_status NULL those failures go unreported.  The return value covers the
 * host-side checks and the launches only (the work is asynchronous).  Work
 * is queued on `stream`; the first call on a device looks up the array's
 * device address (cudaGetSymbolAddress) and should come before any stream
 * capture.  Every call shares the one array and it keeps the previous
 * call's contents, so calls whose GPU work overlaps (different streams,
 * threads or processes sharing a context) race; serialise them. */
int pmb200_eval_noalloc(const pmb200_params *params, int n, const double *d_pos,
                        const int *d_type, const double *d_q, const int *d_mol,
                        const int *d_ex_start, const int *d_ex, int ntypes,
                        const double *lj, double coulomb_scaling,
                        const double box[3], const double origin[3],
                        double *d_forces, double *d_energy, int *d_status,
                        void *stream);

/* Geometry of the device cell grid chosen for the current box. */
int pmb200_grid(const pmb200_ctx *ctx, int dims[3], double edge[3]);

/* ---- other switching functions ----
 * A context of the third kind covers the other registrations of
 * NonbondedCutoffForceModule for periodic boundaries
 * (protomol/src/protomol/module/NonbondedCutoffForceModule.cpp:53-82):
 * OneAtomPair<PBC, S, LennardJonesForce>, OneAtomPair<PBC, S, CoulombForce>
 * (a single potential: the other switch PMB200_SW_NONE) and
 * OneAtomPairTwo<PBC, S1, LennardJonesForce, S2, CoulombForce>, with S from
 * C1 (.../switch/C1SwitchingFunction.h), C2 (C2SwitchingFunction.h), Cn
 * (CnSwitchingFunction.cpp, orders 2, 3, 4 and 6; the reference's order 5
 * has an all-zero coefficient table and is refused with
 * PMB200_EUNSUPPORTED) and ComplimentCnCn (CmpCnCnSwitchingFunction.h/.cpp:
 * 0 below switchon, rising to 1 at switchoff, falling to 0 at the cutoff;
 * orders 2, 3, 4, 6, and 5 read as 2 as the reference does; non-integer
 * orders, which the reference truncates, are refused with
 * PMB200_EUNSUPPORTED).  Each potential is multiplied by its own switch,
 * F' = F S - E dS, E' = E S (OneAtomPair.h:80-88).  Per switch the array
 * holds {switchon, cutoff, order, switchoff}: C1 reads the cutoff only, C2
 * switchon and cutoff, Cn and ComplimentCnCn all four (Cn: switchoff 0 or
 * equal to the cutoff, as CnSwitchingFunction::make requires;
 * ComplimentCnCn: 0 <= switchon < switchoff <= cutoff, as
 * CmpCnCnSwitchingFunction::make requires).
 * Energies: LENNARDJONES and COULOMB as for the first kind.
 *
 * Tabulated LJ: lj_switch = PMB200_SW_TABLE | S (S = C2, Cn or
 * ComplimentCnCn) with coulomb_switch = PMB200_SW_NONE stands for
 * OneAtomPair<BC, UniversalSwitchingFunction, LennardJonesTableForce<S, 7,
 * Real>> (NonbondedCutoffForceModule.cpp:67-72 periodic, 121-126 vacuum;
 * .../force/table/LennardJonesTableForce.h, LookupTable.h): the switched LJ
 * potential tabulated over r^2 from 1/16 A^2 with 128 cubic Hermite
 * intervals per octave, pairs beyond the switch's cutoff skipped and no
 * further switch applied.  The FP64 kernel reads that table (built from the
 * same recipe at creation); the mixed kernel evaluates the switched LJ the
 * table approximates (the table's own interpolation error is below 2e-6 of
 * the force and 3e-8 of the energy, measured over r^2 in [2, 64] A^2).
 * Other combinations with PMB200_SW_TABLE: PMB200_EUNSUPPORTED. */
#define PMB200_SW_NONE 0
#define PMB200_SW_C1 1
#define PMB200_SW_C2 2
#define PMB200_SW_CN 3
#define PMB200_SW_CMPCNCN 4  /* ComplimentCnCn (CmpCnCnSwitchingFunction) */
#define PMB200_SW_TABLE 16   /* flag on lj_switch: LennardJonesTableForce */

typedef struct {
  int precision;       /* PMB200_MIXED or PMB200_FP64 */
  int device;
  int lj_switch;       /* PMB200_SW_*; NONE: no Lennard-Jones term */
  double lj[4];        /* {switchon, cutoff, order, switchoff} */
  int coulomb_switch;  /* PMB200_SW_*; NONE: no Coulomb term */
  double coulomb[4];
  double cutoff_alg;   /* algorithm -cutoff; >= both switch cutoffs */
  double cellsize;     /* grid cell edge hint; 0 = largest cutoff / 2 */
} pmb200_pair_params;

/* Replaces constructing those NonbondedCutoffSystemForce prototypes through
 * the factory (NonbondedCutoffForce::doMake, .../force/nonbonded/
 * NonbondedCutoffForce.h:71-75, with the switch's make). */
int pmb200_create_pair(const pmb200_pair_params *params, pmb200_ctx **out);

/* Vacuum boundaries, in place of pmb200_set_box: the force with
 * VacuumBoundaryConditions (plain differences, no images,
 * protomol/src/protomol/topology/VacuumBoundaryConditions.h) as the
 * vacuum registrations of NonbondedCutoffForceModule build it
 * (NonbondedCutoffForceModule.cpp:84-134, cells walked by
 * CellListEnumeratorStandard.h).  [lo, hi] is the cell-grid domain (any size;
 * edges need not exceed the cutoff).  Atoms outside it are binned into its
 * boundary cells with their true coordinates, so every pair is still found,
 * but FP32 cell-relative coordinates lose precision far outside: keep the
 * domain around the atoms (e.g. their bounding box plus a margin).  Any
 * context kind except the Ewald term; pmb200_set_box makes it periodic
 * again. */
int pmb200_set_vacuum_domain(pmb200_ctx *ctx, const double lo[3], const double hi[3]);

/* ---- derivatives (the differentiable form) ----
 * FP64 pair arithmetic whatever the context's precision; contexts of the
 * cutoff kind only (PMB200_EUNSUPPORTED otherwise).  Units and tables are the
 * ones set_topology takes: q_scaled, and the LJ table entries
 * {A, B, A14, B14} per ordered type pair (a, b) as the pair loop reads them
 * (an unordered pair's derivative is split half to (a, b), half to (b, a)).
 * Work is queued on `stream` (NULL: the context's stream).  H w and dE/dq
 * are summed in exact fixed point (bitwise reproducible) except for the
 * parameter derivatives of tables of more than four types, which take a
 * full-shell kernel summing in FP64 per atom; table derivatives are FP64
 * sums.  A term beyond the fixed-point range (atoms overlapping) sets the
 * device error flag (pmb200_sync reports PMB200_EDEVICE).
 *
 * Parameter gradients: d_dq[n] = dE/dq_scaled per atom, d_dlj[ntypes^2 * 4]
 * = dE/d{A, B, A14, B14}, both overwritten (E = LJ + Coulomb energy).  The
 * reference has no such entry: it replaces finite differences of
 * SystemForce::evaluate over its parameters.  */
int pmb200_param_grad_device(pmb200_ctx *ctx, const double *d_pos, double *d_dq,
                             double *d_dlj, void *stream);

/* Hessian-vector product and the mixed second derivatives for a direction
 * w[3n]: d_hv[3n] = H w (H = d^2 E / dx dx), and, for w . grad_x E, its
 * derivatives d_dq[n] (per q_scaled) and d_dlj[ntypes^2 * 4] (per table
 * entry); all overwritten; d_dq / d_dlj may be NULL.  Replaces forming the
 * dense pair Hessian of Hessian::evaluate
 * (protomol/src/protomol/integrator/hessian/Hessian.cpp:353-568, pair blocks
 * 581-691 with ReducedHessLennardJones / ReducedHessCoulomb and the switch
 * Hessians) and multiplying by w. */
int pmb200_hvp_device(pmb200_ctx *ctx, const double *d_pos, const double *d_w, double *d_hv,
                      double *d_dq, double *d_dlj, void *stream);

/* New charges (q_scaled[n]) and/or LJ table (lj[ntypes^2 * 4]) for the same
 * topology; either may be NULL.  Host arrays; the copy is synchronous, so
 * call it when no evaluation of this context is in flight (pmb200_sync).
 * Replaces rebuilding the topology to change force-field parameters. */
int pmb200_update_params(pmb200_ctx *ctx, const double *q_scaled, const double *lj);

/* The same from DEVICE buffers, queued on `stream` (NULL: the context's
 * stream) with no host round trip: d_q_scaled[n] and/or d_lj[ntypes^2 * 4]
 * (either may be NULL) are copied into the context in stream order, so work
 * queued after it on the same stream sees them.  A non-finite value sets the
 * device error flag (the next pmb200_sync reports PMB200_EDEVICE).  A table
 * needs the box (PMB200_ESTATE otherwise).  For callers whose parameters live
 * on the device, such as the differentiable form's autograd functions, which
 * pass theirs before every kernel call. */
int pmb200_update_params_device(pmb200_ctx *ctx, const double *d_q_scaled, const double *d_lj,
                                void *stream);

/* ---- batches of independent systems ----
 * Many periodic systems of uneven size evaluated together: one counting sort
 * over all their atoms, one persistent pair kernel that takes (system,
 * cell, part of the cell's stencil) tasks from a global counter, one
 * fixed-point finalize, one per-system reduction; with a stream the
 * sequence is captured once as a CUDA graph and replayed.  The reference
 * evaluates one system per force object; a batch replaces a loop of
 * SystemForce::evaluate over such objects
 * (protomol/src/protomol/force/system/SystemForce.h:32-35).
 *
 * pmb200_batch_create builds a batch from nsys contexts of precision
 * PMB200_MIXED and the same kind (cutoff or Ewald real-space), each holding
 * its topology and box; it copies what it needs (the contexts stay usable
 * and independent).  Positions and forces are the systems' arrays back to
 * back in system order, [3 * sum n_s]; forces are accumulated into;
 * d_out[nsys][20] receives each system's {COULOMB, LENNARDJONES, virial 9,
 * molecular virial 9 (zero: not offered)}.  The schedule (stencil parts per
 * cell 1..8, task order 0 = by system / 1 = largest estimated cost first,
 * persistent one-warp blocks per SM, 0 = as many as fit) is set directly or chosen
 * by pmb200_batch_autotune, which times every candidate on the given
 * positions (reps timed launches each) and keeps the fastest; sched[4] =
 * {parts, order, blocks per SM, tasks}. */
typedef struct pmb200_batch pmb200_batch;
int pmb200_batch_create(pmb200_ctx *const *systems, int nsys, pmb200_batch **out);
int pmb200_batch_destroy(pmb200_batch *batch);
const char *pmb200_batch_last_error(const pmb200_batch *batch);
int pmb200_batch_eval_device(pmb200_batch *batch, const double *d_pos, double *d_forces,
                             double *d_out, unsigned flags, void *stream);
int pmb200_batch_set_schedule(pmb200_batch *batch, int parts, int order, int blocks_per_sm);
int pmb200_batch_get_schedule(const pmb200_batch *batch, int sched[4]);
int pmb200_batch_autotune(pmb200_batch *batch, const double *d_pos, void *stream, int reps,
                          int sched[4], float *best_ms);
/* CUDA-event time of the last directly launched pair kernel (timing on:
 * launches are direct, not graph replays). */
int pmb200_batch_set_kernel_timing(pmb200_batch *batch, int on);
int pmb200_batch_last_kernel_ms(pmb200_batch *batch, float *ms);
/* In-cutoff pair count per system of the last evaluation with energies. */
int pmb200_batch_pair_counts(pmb200_batch *batch, long long *counts);
/* Waits for `stream` (NULL: the whole device) and reports a device-side
 * error of the batch's evaluations since the last call (PMB200_EDEVICE:
 * a non-finite position, or a pair force beyond the fixed-point range). */
int pmb200_batch_sync(pmb200_batch *batch, void *stream);

/* ---- Ewald real-space term ----
 * A context of the second kind replaces the real-space part of ProtoMol's
 * Ewald sum,
 *   NonbondedFullEwaldSystemForce<PeriodicBoundaryConditions,
 *     CubicCellManager, real = true, reciprocal = false, correction = false,
 *     CutoffSwitchingFunction>
 * (protomol/src/protomol/module/NonbondedFullElectrostaticForceModule.cpp:34;
 * config "force Coulomb -algorithm FullEwald -real -alpha <a> -accuracy
 * <acc>"; pair term .../force/nonbonded/NonbondedFullEwaldSystemForce.h:
 * 776-851): E = sum over pairs within rc of q_i q_j erfc(alpha r) / r,
 * modified (1-4) pairs scaled by coulombScalingFactor, full exclusions
 * skipped.  rc = sqrt(-log(accuracy)) / alpha and, for alpha <= 0, the
 * reference's default alpha = sqrt(pi) (5.5 N / V^2)^(1/6) are derived as
 * in NonbondedFullEwaldSystemForce::initialize (same header, 586-598), once
 * the topology and the box are both set.  Every box edge must be >= 2 rc
 * (the reference then adds no lattice image, PeriodicBoundaryConditions::
 * buildLatticeVectors, .../topology/PeriodicBoundaryConditions.cpp:80-104).
 * All other calls (set_topology, set_box, eval, eval_device, leapfrog_device,
 * step_device, ...) work on it unchanged; the energy goes to COULOMB and
 * LENNARDJONES receives 0.  The LJ table passed to set_topology is not used. */
#define PMB200_ERFC_POLY5 0 /* Abramowitz & Stegun 7.1.26, the reference's default build */
#define PMB200_ERFC_EXACT 1 /* erfc() itself: the reference built with -DUSE_EWALD_EXACT_ERF */

typedef struct {
  int precision;   /* PMB200_MIXED or PMB200_FP64 */
  int device;      /* CUDA device ordinal */
  int erfc;        /* PMB200_ERFC_POLY5 or PMB200_ERFC_EXACT */
  double alpha;    /* -alpha (1/Angstrom); <= 0 selects the reference's default */
  double accuracy; /* -accuracy, in (0, 1) */
  double cellsize; /* grid cell edge hint; 0 = rc / 2 */
} pmb200_ewald_params;

/* Replaces constructing NonbondedFullEwaldSystemForce(alpha, accuracy, 3.0)
 * through its doMake (NonbondedFullEwaldSystemForce.h:118-142). */
int pmb200_create_ewald_real(const pmb200_ewald_params *params, pmb200_ctx **out);

/* The alpha and real-space cutoff in use (PMB200_ESTATE until the topology
 * and the box are set, or for a context of the first kind). */
int pmb200_ewald_info(const pmb200_ctx *ctx, double *alpha, double *rc);

#ifdef __cplusplus
}
#endif
#endif /* PMB200_H */
