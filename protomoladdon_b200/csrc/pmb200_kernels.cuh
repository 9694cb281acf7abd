// Device kernels of libpmb200: cell build (counting sort), the mixed-precision
// and FP64 cell-pair force kernels, reductions and the leapfrog update.
//
// Data layout in HBM (per context, n atoms, C cells, x fastest):
//   cell_of[n]        int    cell id of each atom (original order)
//   cell_count[C]     int    atoms per cell (histogram)
//   cell_start[C+1]   int    exclusive scan of cell_count
//   slot_tmp[n]       int    original index at an unsorted position in its cell
//   sidx[n]           int    original index at each cell-sorted position
//   spos32[n]         float4 (x, y, z, q') in cell units, relative to the cell's
//                            lower corner; q' = scaledCharge / sqrt(edge)
//   spos64[n]         double4 (x, y, z, q) in Angstrom relative to the cell's
//                            lower corner (FP64 kernel)
//   smeta[n]          int2   (LJ type, molecule id) at sorted positions
//   rel32[n]/rel64[n] per-atom wrapped coordinates before the gather
//   partial[C][NACC]  double per-cell-warp energy/virial/pair-count partials
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace pmb200 {

constexpr int kMaxRows = 128;         // stencil rows (dy, dz), passed by value
constexpr int kMaxTypes = 16;         // LJ types held in shared memory
constexpr int kMaxTypesTable = 1024;  // LJ types of a context (more than kMaxTypes:
                                      // the mixed kernel reads the table through L1)
constexpr int kNacc = 16;             // slots per partial-sum row (>= ACC_MV)
constexpr double kFixScale = 4294967296.0;          // 2^32 per force unit
constexpr double kFixInv = 1.0 / 4294967296.0;

// accumulator slot indices (partial[w][k])
enum {
  ACC_ECOUL = 0,// Coulomb energy
  ACC_ELJ = 1,  // Lennard-Jones energy
  ACC_PAIRS = 2,// in-cutoff pairs
  ACC_W = 3,    // 6 virial components xx xy xz yy yz zz (3..8)
  ACC_MW = 9,   // 6 molecular-virial components f_a comDiff_b, a <= b (9..14)
  ACC_MV = 15,  // number of slots in use
  ACC_E = 3,    // the slots an energy launch without virial fills
};

static_assert(kNacc >= ACC_MV, "partial-sum rows hold every slot");

struct Row {        // one (dy, dz) row of the neighbour-cell stencil
  int dy, dz, dxlo, dxhi;
};

struct GridParams {
  int nx, ny, nz, ncell;
  double edge[3];    // cell edges (A); general cells: the cells' widths
  double boxmin[3];  // lower box corner
  double boxlen[3];  // box edges
  double unit;       // cell-unit length scale (= edge[0]; general cells: the smallest width)
  int nrows;
  int periodic;      // 1: periodic box (wrap, minimum image); 0: vacuum domain
  // General (non-orthogonal) periodic cell: the grid is n_k cells along each
  // basis vector e_k; an atom is binned by its fractional coordinates and
  // stored as its Cartesian offset from its cell's lattice corner, so the
  // pair kernels see Cartesian differences as for an orthogonal box and only
  // the shift of a neighbour cell (a lattice vector) changes.
  int tric;          // 1: general basis (the fields below)
  double org[3];     // box centre (PeriodicBoundaryConditions origin)
  double lat[9];     // rows: n_k times the reciprocal vector e_k^r (lattice coordinates)
  double ec[9];      // ec[3 r + k] = component r of e_k / n_k (a cell's edge vectors, A)
  double m[9];       // ec / unit: the shift of a cell offset in cell units
};

// Cartesian shift (A when `mat` is ec, cell units when it is m) of the cell
// offset (dx, dy, dz): for an orthogonal grid (dx edge0, dy edge1, dz edge2).
__host__ __device__ __forceinline__ void cell_shift(const GridParams &g, const double *mat,
                                                   double scale, int dx, int dy, int dz,
                                                   double &sx, double &sy, double &sz) {
  if (g.tric) {
    sx = mat[0] * dx + mat[1] * dy + mat[2] * dz;
    sy = mat[3] * dx + mat[4] * dy + mat[5] * dz;
    sz = mat[6] * dx + mat[7] * dy + mat[8] * dz;
  } else {
    sx = dx * g.edge[0] * scale;
    sy = dy * g.edge[1] * scale;
    sz = dz * g.edge[2] * scale;
  }
}

// PeriodicBoundaryConditions constants for minimalDifference
// (protomol/src/protomol/topology/PeriodicBoundaryConditions.cpp:32-77,
// orthogonal box), used for the molecule-centre differences of the
// molecular virial.
struct PbcRef {
  double e[3], er[3], h[3], h2[3], d;
  int tric;                 // general basis: the vectors below
  double ev[9], erv[9];     // rows: e1, e2, e3 and e1r, e2r, e3r
};

// PeriodicBoundaryConditions::minimalDifference
// (protomol/src/protomol/topology/PeriodicBoundaryConditions.h:53-70, and the
// general branch 62-67: diff -= e1 rint(e1r.diff) + e2 rint(e2r.diff) +
// e3 rint(e3r.diff)).
__device__ __forceinline__ void ref_min_image(const PbcRef &b, double v[3]) {
  if (b.tric) {
    double k[3];
    for (int a = 0; a < 3; a++)
      k[a] = rint(b.erv[3 * a] * v[0] + b.erv[3 * a + 1] * v[1] + b.erv[3 * a + 2] * v[2]);
    double w[3];
    for (int c = 0; c < 3; c++)
      w[c] = b.ev[c] * k[0] + b.ev[3 + c] * k[1] + b.ev[6 + c] * k[2];
    for (int c = 0; c < 3; c++) v[c] -= w[c];
    return;
  }
  if (v[0] * v[0] + v[1] * v[1] + v[2] * v[2] > b.d) {
    for (int k = 0; k < 3; k++) {
      if (v[k] < -b.h2[k]) v[k] += b.h[k];
      else if (v[k] > b.h2[k]) v[k] -= b.h[k];
    }
    if (v[0] * v[0] + v[1] * v[1] + v[2] * v[2] > b.d)
      for (int k = 0; k < 3; k++) v[k] -= b.e[k] * rint(b.er[k] * v[k]);
  }
}

// Pair potential of a context: ProtoMol's cutoff LJ (C2) + Coulomb (C1)
// force, or the real-space Ewald term with erfc from the Abramowitz & Stegun
// polynomial (the reference's default build) or from erfc itself.
enum PairForm { FORM_CUTOFF = 0, FORM_EWALD_POLY5 = 1, FORM_EWALD_EXACT = 2, FORM_GENERIC = 3 };

// Switching functions of the generic form (each potential its own; SW_OFF:
// the potential is absent).  dS is ProtoMol's "deriv": dS/dr / r.
enum SwitchKind { SW_OFF = 0, SW_C1 = 1, SW_C2 = 2, SW_CN = 3, SW_CMPCNCN = 4 };

template <class T>
struct SwitchSpec {
  int kind, nord;    // SwitchKind; Cn: integer order
  T rc2, ron2, rc;   // cutoff^2, switchon^2, cutoff
  T a, b, c;         // C1: 1.5/rc, 0.5/rc^3, 1.5/rc^3; C2: s1, s2, s3 (C2SwitchingFunction.cpp)
  T ron, inv_range;  // Cn: switchon, 1 / (switchon - cutoff);
                     // ComplimentCnCn: switchon, 1 / (switchoff - cutoff)
  T roff2, roff, inv_in;  // ComplimentCnCn: switchoff^2, switchoff, 1 / (switchoff - switchon)
  T vcoef[7];        // Cn, ComplimentCnCn: binom(2n+1, n+1+j), j = 0..n
  T dpeak;           // Cn, ComplimentCnCn: (2n+1)! / (n!)^2
};

// Value S and deriv dS (= dS/dr / r) at r^2 (rinv = 1/r), following
// C1SwitchingFunction.h:41-50, C2SwitchingFunction.h:42-53 and
// CnSwitchingFunction.cpp:149-172.  Cn: the reference sums
// swcoef_i t^(n+1+i) with t = (r - rc)/(switchon - rc); its tables are the
// smoothstep polynomials, evaluated here in their Bernstein form
//   S = sum_{k=n+1}^{2n+1} binom(2n+1, k) t^k u^(2n+1-k),  u = 1 - t,
//   dS/dt = (2n+1)!/(n!)^2 t^n u^n,
// whose terms are all positive (the power form cancels to ~1e-4 of its
// terms at order 6, too much for FP32); t and u are both taken from r.
// ComplimentCnCn (CmpCnCnSwitchingFunction.h:39-84): 0 below switchon, the
// same polynomial rising on [switchon, switchoff] (the reference's 1 - its
// falling form, which is the rising one by the polynomial's symmetry) and
// falling on (switchoff, cutoff].
template <class T>
__host__ __device__ __forceinline__ void switch_eval(const SwitchSpec<T> &w, T r2, T rinv, T &S,
                                                    T &dS) {
  S = T(0);
  dS = T(0);
  if (r2 > w.rc2) return;
  if (w.kind == SW_C1) {
    const T dist = r2 * rinv;
    S = T(1) - dist * (w.a - r2 * w.b);
    dS = -w.a * rinv + dist * w.c;
  } else if (w.kind == SW_C2) {
    if (r2 < w.ron2) { S = T(1); return; }
    const T c2 = w.rc2 - r2;
    const T c4 = c2 * (w.b + T(2) * r2);
    S = w.a * (c2 * c4);
    dS = w.c * (c2 * c2 - c4);
  } else if (w.kind == SW_CN) {
    if (r2 < w.ron2) { S = T(1); return; }
    const T r = r2 * rinv;
    const T t = (r - w.rc) * w.inv_range;
    const T u = (w.ron - r) * w.inv_range;
    T tn = T(1), un = T(1);
    for (int k = 0; k < w.nord; k++) { tn *= t; un *= u; }
    // sum_j vcoef_j t^j u^(n-j), by Horner in t/u homogeneous form
    T acc = w.vcoef[w.nord], up = T(1);
    for (int j = w.nord - 1; j >= 0; j--) {
      up *= u;
      acc = acc * t + w.vcoef[j] * up;
    }
    S = tn * t * acc;
    dS = w.dpeak * tn * un * w.inv_range * rinv;
  } else if (w.kind == SW_CMPCNCN) {
    if (r2 < w.ron2) return;
    const T r = r2 * rinv;
    const bool fall = r2 > w.roff2;
    // rising: t = (r - switchon) / (switchoff - switchon); falling:
    // t = (r - cutoff) / (switchoff - cutoff); u = 1 - t from r in both
    const T scale = fall ? w.inv_range : w.inv_in;
    const T t = (r - (fall ? w.rc : w.ron)) * scale;
    const T u = (w.roff - r) * scale;
    T tn = T(1), un = T(1);
    for (int k = 0; k < w.nord; k++) { tn *= t; un *= u; }
    T acc = w.vcoef[w.nord], up = T(1);
    for (int j = w.nord - 1; j >= 0; j--) {
      up *= u;
      acc = acc * t + w.vcoef[j] * up;
    }
    S = tn * t * acc;
    dS = w.dpeak * tn * un * scale * rinv;
  }
}

// Abramowitz & Stegun, Handbook of Mathematical Functions, 7.1.26:
// erfc(x) ~ t (a1 + t (a2 + t (a3 + t (a4 + t a5)))) exp(-x^2),
// t = 1 / (1 + p x), |error| <= 1.5e-7 (the reference's poly5,
// protomol/src/protomol/base/MathUtilities.cpp:39-49).
constexpr double kAsP = 0.3275911;
constexpr double kAsA1 = 0.254829592, kAsA2 = -0.284496736, kAsA3 = 1.421413741,
                 kAsA4 = -1.453152027, kAsA5 = 1.061405429;

struct MixedConsts {   // FP32 constants in cell units
  float cut2, rclj2, ron2, rcc2;
  float s1, s2, s3;          // C2
  float c15_1, c05_3, c15_3; // C1 (force path)
  float csf;                 // coulombScalingFactor
  float ey, ez;              // edge[1] / unit, edge[2] / unit (1 for cubic cells)
  double e15, e05;           // C1 energy (FP64): 1.5 / rc_coul and 0.5 / rc_coul^3 (cell units)
  float ea, ea2pi;           // Ewald alpha and 2 alpha / sqrt(pi), per cell unit
  SwitchSpec<float> swl, swc;  // generic form: LJ and Coulomb switches
};

struct Fp64Consts {
  double cut2, rclj2, ron2, rcc2;
  double s1, s2, s3;
  double c15_1, c05_3, c15_3;
  double csf;
  double ea, ea2, ea2pi;     // Ewald alpha, alpha^2, 2 alpha / sqrt(pi) (1/A)
  SwitchSpec<double> swl, swc;  // generic form: LJ and Coulomb switches
  // generic form, tabulated LJ (LennardJonesTableForce): two double4 per grid
  // point, the hash of the first point and the last point (null: analytic)
  const double4 *ljtab;
  int tfirst, tlast;
};

// LookupTable<..., PRE = 7, double>: 2^7 intervals per octave of r^2, so the
// hash of r^2 is its top 64 - 45 bits (sign, exponent, 7 mantissa bits)
constexpr int kTabPre = 7;
constexpr int kTabShift = 52 - kTabPre;

// LennardJonesTableForce::operator() with LookupTable::index / interpolate
// (LennardJonesTableForce.h:68-89, LookupTable.h:196-214): the grid point of
// r^2 from its bit pattern, dt = r^2 minus r^2 with its low 45 bits cleared
// (0 outside the grid, clamped to its ends), then the cubic in dt.  e: the
// energy; f: force / r.
__device__ __forceinline__ void lj_table_eval(const double4 *__restrict__ tab, int first, int last,
                                              double r2, double A, double B, double &e,
                                              double &f) {
  const long long b = __double_as_longlong(r2);
  int i = (int)(b >> kTabShift) - first;
  double dt = 0.0;
  if (i < 0) i = 0;
  else if (i > last) i = last;
  else dt = r2 - __longlong_as_double(b & ~((1LL << kTabShift) - 1));
  const double4 ta = tab[2 * i], tb = tab[2 * i + 1];
  const double a = ta.x * A + tb.x * B;
  const double bb = ta.y * A + tb.y * B;
  const double c = ta.z * A + tb.z * B;
  const double d = ta.w * A + tb.w * B;
  e = ((dt * d + c) * dt + bb) * dt + a;
  f = -2.0 * ((3.0 * dt * d + 2.0 * c) * dt + bb);
}

// The stencil travels by value in the kernel parameters (per launch, so
// contexts with different grids never share it).
struct Stencil {
  Row rows[kMaxRows];
};

// Half-shell neighbour cells, one entry per cell offset, packed as
// (dx + 8) | (dy + 8) << 5 | (dz + 8) << 10 (offsets lie in [-8, 8]).
constexpr int kMaxHalfCells = 512;
struct HalfStencil {
  unsigned short off[kMaxHalfCells];
  int ncells;
};

// ---------------------------------------------------------------------------
// Cell build.
// ---------------------------------------------------------------------------

// Wrap each position into the box in FP64, find its cell (x fastest), count
// cell occupancy, and keep the coordinates relative to the cell's lower
// corner.  Non-finite coordinates raise err bit 1 and are binned at cell 0.
// The cell of one position: wrapped into the box in FP64, the cell
// coordinates c and the offset r from the cell's lower corner (Angstrom).
// Returns false for a non-finite coordinate (binned at the box corner).
// Programmatic dependent launch (the kernels of one evaluation launched as
// dependents of the one before them, so that each launch overlaps its
// predecessor's tail).  pdl_wait: block until the predecessor grid has
// completed and its writes are visible (a no-op for a kernel launched
// normally); every kernel that may be launched so calls it before touching
// data its predecessor reads or writes.  pdl_trigger: this grid's dependent
// may launch now (it still waits for this grid's completion before use).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;"); }

__device__ __forceinline__ bool locate_cell(const double *xin, const GridParams &g, int c[3],
                                            double r[3]) {
  const int nd[3] = {g.nx, g.ny, g.nz};
  bool ok = true;
  if (g.tric) {
    // lattice coordinates t_k = n_k (e_k^r . (x - origin) + 1/2), wrapped
    // into [0, n_k); the offset from the cell's lattice corner, in A
    double x[3];
    for (int a = 0; a < 3; a++) {
      x[a] = xin[a] - g.org[a];
      if (!isfinite(xin[a])) { ok = false; x[a] = 0.0; }
    }
    double u[3];
    for (int k = 0; k < 3; k++) {
      double t = g.lat[3 * k] * x[0] + g.lat[3 * k + 1] * x[1] + g.lat[3 * k + 2] * x[2] +
                 0.5 * nd[k];
      t -= nd[k] * floor(t / nd[k]);
      int ck = (int)floor(t);
      ck = ck < 0 ? 0 : (ck >= nd[k] ? nd[k] - 1 : ck);
      c[k] = ck;
      u[k] = t - ck;
    }
    for (int a = 0; a < 3; a++)
      r[a] = g.ec[3 * a] * u[0] + g.ec[3 * a + 1] * u[1] + g.ec[3 * a + 2] * u[2];
    return ok;
  }
  for (int a = 0; a < 3; a++) {
    double x = xin[a];
    if (!isfinite(x)) { ok = false; x = g.boxmin[a]; }
    double w = x - g.boxmin[a];
    if (g.periodic) w -= g.boxlen[a] * floor(w / g.boxlen[a]);
    // vacuum: atoms outside the domain are clamped into its boundary cells;
    // r keeps their true offset, so no pair is lost (the cell-index map
    // stays 1-Lipschitz)
    int ca = (int)floor(w / g.edge[a]);
    ca = ca < 0 ? 0 : (ca >= nd[a] ? nd[a] - 1 : ca);
    c[a] = ca;
    r[a] = w - ca * g.edge[a];
  }
  return ok;
}

// clear: an accumulator of nclear x n entries zeroed on the way (or null).
__global__ void k_cell_index(int n, const double *__restrict__ pos, GridParams g,
                             int *__restrict__ cell_of, int *__restrict__ cell_count,
                             int *__restrict__ slot, float4 *__restrict__ rel32,
                             double4 *__restrict__ rel64, const double *__restrict__ q,
                             float qscale32, int *__restrict__ err,
                             float4 *__restrict__ rel_lo,
                             unsigned long long *__restrict__ clear = nullptr, int nclear = 3) {
  pdl_trigger();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (clear)
    for (int k = 0; k < nclear; k++) clear[(size_t)k * n + i] = 0;
  int c[3];
  double r[3];
  if (!locate_cell(pos + 3 * (size_t)i, g, c, r)) atomicOr(err, 1);
  int cid = (c[2] * g.ny + c[1]) * g.nx + c[0];
  cell_of[i] = cid;
  slot[i] = atomicAdd(&cell_count[cid], 1);
  double qi = q[i];
  if (rel32) {
    const double inv = 1.0 / g.unit;
    const double v[3] = {r[0] * inv, r[1] * inv, r[2] * inv};
    const float h[3] = {(float)v[0], (float)v[1], (float)v[2]};
    rel32[i] = make_float4(h[0], h[1], h[2], (float)qi * qscale32);
    // the FP32 coordinates' rounding residuals (energy evaluations)
    if (rel_lo)
      rel_lo[i] = make_float4((float)(v[0] - (double)h[0]), (float)(v[1] - (double)h[1]),
                              (float)(v[2] - (double)h[2]), 0.f);
  }
  if (rel64) rel64[i] = make_double4(r[0], r[1], r[2], qi);
}

// Exclusive scan of cell counts in one block (C is a few thousand to a few
// hundred thousand cells; each thread scans a contiguous span).
// (the counts are cleared once read, ready for the next build's atomics)
__global__ void k_scan(int ncell, int *__restrict__ count, int *__restrict__ start) {
  pdl_trigger();
  pdl_wait();
  extern __shared__ int sh[];
  const int T = blockDim.x;
  const int t = threadIdx.x;
  const int span = (ncell + T - 1) / T;
  const int lo = t * span;
  const int hi = min(ncell, lo + span);
  int s = 0;
  for (int c = lo; c < hi; c++) s += count[c];
  // inclusive scan of the per-thread sums: within each warp by shuffles,
  // then over the warps' totals (at most 32 warps; blockDim is a multiple of
  // 32) by the first warp
  const int lane = t & 31, w = t >> 5, nw = T >> 5;
  int x = s;
  for (int off = 1; off < 32; off <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, x, off);
    if (lane >= off) x += v;
  }
  if (lane == 31) sh[w] = x;
  __syncthreads();
  if (w == 0) {
    int y = lane < nw ? sh[lane] : 0;
    for (int off = 1; off < 32; off <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, y, off);
      if (lane >= off) y += v;
    }
    if (lane < nw) sh[lane] = y;
  }
  __syncthreads();
  const int incl = x + (w > 0 ? sh[w - 1] : 0);
  int base = incl - s;
  for (int c = lo; c < hi; c++) {
    const int v = count[c];
    start[c] = base;
    base += v;
    count[c] = 0;
  }
  if (t == T - 1) start[ncell] = incl;
}

__global__ void k_scatter(int n, const int *__restrict__ cell_of, const int *__restrict__ slot,
                          const int *__restrict__ start, int *__restrict__ tmp) {
  pdl_trigger();
  pdl_wait();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  tmp[start[cell_of[i]] + slot[i]] = i;
}

// One warp per cell: order the cell's atoms by original index (rank = number
// of members with a smaller index) and gather their data to sorted positions,
// so the layout, and every sum over it, is the same on every run.
__global__ void k_rank_gather(int ncell, const int *__restrict__ start,
                              const int *__restrict__ tmp, const float4 *__restrict__ rel32,
                              const double4 *__restrict__ rel64, const int *__restrict__ type,
                              const int *__restrict__ mol, int *__restrict__ sidx,
                              float4 *__restrict__ spos32, double4 *__restrict__ spos64,
                              int2 *__restrict__ smeta, const float4 *__restrict__ rel_lo,
                              float4 *__restrict__ spos_lo, int zorder = 0) {
  pdl_trigger();
  pdl_wait();
  const int lane = threadIdx.x & 31;
  const int cell = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (cell >= ncell) return;
  const int s = start[cell], e = start[cell + 1];
  for (int k = s + lane; k < e; k += 32) {
    const int me = tmp[k];
    int rank = 0;
    if (zorder) {  // by height in the cell (FP32 coordinate), then by index
      const float zme = rel32[me].z;
      for (int m = s; m < e; m++) {
        const int o = tmp[m];
        const float zo = rel32[o].z;
        rank += (zo < zme || (zo == zme && o < me));
      }
    } else {
      for (int m = s; m < e; m++) rank += (tmp[m] < me);
    }
    const int d = s + rank;
    sidx[d] = me;
    if (spos32) spos32[d] = rel32[me];
    if (spos64) spos64[d] = rel64[me];
    if (spos_lo) spos_lo[d] = rel_lo[me];
    smeta[d] = make_int2(type[me], mol[me]);
  }
}

// ---------------------------------------------------------------------------
// Exclusion lookup: per original atom, its partners sorted ascending with the
// exclusion kind (1 modified, 2 full), CSR.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int excl_kind(const int2 *__restrict__ ex, int lo, int hi, int j) {
  for (int k = lo; k < hi; k++) {
    int2 e = __ldg(&ex[k]);
    if (e.x == j) return e.y;
    if (e.x > j) break;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Warp helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum_mask(double v, int width) {
  for (int off = 1; off < width; off <<= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// The per-warp partial row of a pair kernel: warp sums of the first ns slots
// of v (ns = ACC_E or ACC_MV), written by lane 0; the rest of the row is left
// as it is (the reductions read only the first ns slots).
template <int ns>
__device__ __forceinline__ void write_partial_row(const double (&v)[ACC_MV], int lane,
                                                  double *__restrict__ row) {
#pragma unroll
  for (int k = 0; k < ns; k++) {
    const double sum = warp_sum_mask(v[k], 32);
    if (lane == 0) row[k] = sum;
  }
}

__device__ __forceinline__ long long warp_sum_ll(long long v, int width) {
  for (int off = 1; off < width; off <<= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// Lanes per i-atom for a chunk of m atoms: the largest power of two L <= 8
// with m * L <= 32.
// floor(a / d) for 0 <= a <= 32 and 1 <= d <= 32: (a + 1/2) / d lies at
// least 1 / 64 from an integer, far more than the error of the fast FP32
// division (a few ulp), so truncation gives the quotient
__device__ __forceinline__ int small_quot(int a, int d) {
  return (int)__fdividef((float)a + 0.5f, (float)d);
}

__device__ __forceinline__ int lanes_per_atom(int m) {
  int L = 1;
  while (L < 8 && m * (L * 2) <= 32) L <<= 1;
  return L;
}

// ---------------------------------------------------------------------------
// Mixed-precision pair kernel (Newton's third law, half-shell stencil).
//
// Work unit: one warp, one i-cell and every nslots-th entry of the cell's
// half-shell stencil (every cell pair once; the home cell pairs i < j).
// Warps never wait for one another.
//
// Per warp: the cell's atoms are taken in chunks of at most 32, every lane
// serving one atom (32 / m or 32 / m + 1 lanes per atom of an m-atom chunk,
// splitting its candidates by index).  Candidate j atoms
// are staged in shared memory in batches of at most kBatch, already shifted
// into the i-cell's frame (integer cell offsets in cell units, so no
// per-offset rounding bias); atoms beyond the cutoff of the box around the
// chunk's i atoms are not staged.  Each lane first scans the batch and
// compacts the indices of its in-range partners into a private list; the
// lists are then walked densely (the pair arithmetic never runs under a
// divergent branch), the longer lists' tails dealt over the whole warp.
//
// Forces: the pair force on j is added to a per-batch int32 fixed-point
// accumulator in shared memory (2^-18 cell-unit force quanta; integer
// atomics, so the sum is independent of order) and flushed per batch into
// the global int64 fixed-point accumulator facc (2^-32 quanta, sorted order,
// [3][n]).  The force on i is summed in FP32 per batch (dealt pairs: int32
// shared quanta), folded into an int64 register, combined over the atom's
// lanes and added to facc once per warp.  Every integer sum is exact, so
// the result does not depend on scheduling.
//
// Pair arithmetic is FP32 in cell units.  The Coulomb energy of the cutoff
// form is summed in FP64 from FP64 distances (q_j g(r) per pair, g the
// C1-switched 1/r); the other forms' as Kahan-compensated FP32 sums.
// ---------------------------------------------------------------------------
#ifndef PMB200_STAGE_BATCH
#define PMB200_STAGE_BATCH 128
#endif
// staged j atoms per warp batch: at most 128, for the byte-wide list indices
// and the int32 shared force sums (checked where the batch is used)
constexpr int kBatch = PMB200_STAGE_BATCH;
#ifndef PMB200_STAGE_BATCH_E
#define PMB200_STAGE_BATCH_E PMB200_STAGE_BATCH
#endif
// the same for the single-system kernel's energy launches (shared memory,
// with the FP64 energy staging, sets their residency)
constexpr int kBatchE = PMB200_STAGE_BATCH_E;

constexpr float kJScale = 262144.0f; // shared j-force quanta (2^-18) per cell-unit force
constexpr int kJShift = 14;          // to the global 2^-32 quanta
constexpr float kJLimit = 6.7e7f;    // per-contribution bound: 32 contributions fit int32
constexpr float kJToGlobal = 16384.0f;  // 2^-18 quanta -> the accumulator's 2^-32 quanta
#ifndef PMB200_DEAL_UNIT
#define PMB200_DEAL_UNIT 3      // leftover entries dealt to a lane at a time
#endif
#ifndef PMB200_SPREAD_COST
#define PMB200_SPREAD_COST 40   // cost of a round of dealt units, in tenths of an own round
#endif
constexpr int kDealUnit = PMB200_DEAL_UNIT;
#ifndef PMB200_PDL
#define PMB200_PDL 1            // pair kernels launched as programmatic dependents
#endif

template <int kB>
struct __align__(16) MixedWarpSmemT {
  static constexpr int kCap = kB;        // staged atoms per batch
  float4 pos[kB];                        // staged j atoms, shifted into the i-cell frame
  int jf[3][kB];                         // per-batch j forces, int32 fixed point (2^-18)
  int fi[3][32];                         // per-lane i forces of leftover pairs (2^-18)
  int2 meta[kB];                         // their (LJ type, molecule)
  int gidx[kB];                          // their sorted indices
  unsigned char list[kB / 2][32];        // per-lane in-range candidate indices
};
using MixedWarpSmem = MixedWarpSmemT<kBatch>;

struct KahanF {
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float x) {
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
  }
};

// j forces: each contribution, in 2^-18 quanta of cell-unit force, goes to
// j's per-batch int32 shared accumulator.  A batch adds at most 32
// contributions to one j, so each must stay within kJLimit quanta (256 cell
// units); a pair with a larger component (close contacts) adds all three
// straight to the global int64 accumulator at 2^-32 resolution instead.
// Both sums are exact integer sums.

// One task of the mixed pair kernel for one warp: i-cell `cell` and the
// stencil entries slot + k * nslots (nslots = 1: the cell's whole half
// shell).  The stencil offsets and the LJ table are read from shared memory;
// the warp's i forces go straight to facc and its energy and virial partials
// to partial_row.  Warps never wait for one another.
template <int kForm, bool kEnergy, bool kVirial, bool kMolVir, class Smem = MixedWarpSmem>
__device__ __forceinline__ void mixed_task(
    const GridParams &g, const MixedConsts &mc, const unsigned short *st_off, int st_ncells,
    int slot, int nslots, int ntypes, const float4 *s_lj, int cell,
    const int *__restrict__ start, const float4 *__restrict__ spos,
    const int2 *__restrict__ smeta, const int *__restrict__ sidx,
    const int *__restrict__ ex_start, const int2 *__restrict__ ex,
    unsigned long long *__restrict__ facc, int n, double *__restrict__ partial_row,
    const PbcRef &pb, const double *__restrict__ com, Smem &sm,
    int *__restrict__ err, float *__restrict__ s_res, const float4 *__restrict__ spos_lo) {
  const int lane = threadIdx.x & 31;
  // the energy of the cutoff form is summed from FP64 distances: kEnergy
  // launches also stage, for each j position shifted into the i-cell frame,
  // what the FP32 staged value lacks of the FP64 one (s_res: this warp's
  // 3 x kBatch floats), from the FP32 coordinate, its rounding residual
  // (spos_lo, sorted order) and the shift; FP32 staged value + that
  // remainder = the FP64 position to ~1e-13 of a cell
  constexpr bool kExactE = kEnergy && kForm == FORM_CUTOFF;
  float *rsx = kExactE ? s_res : nullptr;
  constexpr int kBatch = Smem::kCap;  // this kernel's staging batch
  // the int32 shared sums: a staged j atom meets each of a chunk's (at most
  // 32) i atoms once per batch, each contribution within kJLimit quanta; a
  // lane's dealt i-force sums take at most kBatch / 2 contributions per batch,
  // each within kJLimit / 2
  static_assert(32.0 * (double)kJLimit < 2147483648.0, "j-force sums fit int32");
  static_assert((double)(kBatch / 2) * 0.5 * (double)kJLimit < 2147483648.0,
                "dealt i-force sums fit int32");
  float *rsy = kExactE ? rsx + kBatch : nullptr, *rsz = kExactE ? rsx + 2 * kBatch : nullptr;
  const int cx = cell % g.nx;
  const int cy = (cell / g.nx) % g.ny;
  const int cz = cell / (g.nx * g.ny);
  const int cs = start[cell], ce = start[cell + 1];

  KahanF kU;
  double accU = 0, accE = 0, accP = 0;
  double w[6] = {0, 0, 0, 0, 0, 0};
  double mw[6] = {0, 0, 0, 0, 0, 0};
  const double inv_unit = 1.0 / g.unit;

  for (int c0 = cs; c0 < ce; c0 += 32) {
    const int m = min(32, ce - c0);
    // every lane serves one of the chunk's atoms: atom ia owns the L
    // contiguous lanes whose first has sub 0 (the first 32 % m atoms one
    // lane more than the others), and each lane takes every L-th candidate
    const int base = small_quot(32, m), extra = 32 - base * m, split = extra * (base + 1);
    const bool wide = lane < split;
    const int L = wide ? base + 1 : base;
    const int la = wide ? lane : lane - split;
    const int q = small_quot(la, L);
    const int ia = wide ? q : extra + q;
    const int sub = la - q * L;
    const bool active = ia < m;
    const int i = c0 + (active ? ia : 0);
    const float4 pi = spos[i];
    const int2 mi = smeta[i];
    const int oi = sidx[i];
    const int elo = ex_start[oi], ehi = ex_start[oi + 1];
    const int ti = mi.x * ntypes;
    // the box around the chunk's i atoms
    float blo_x = pi.x, blo_y = pi.y, blo_z = pi.z, bhi_x = pi.x, bhi_y = pi.y, bhi_z = pi.z;
    for (int off = 16; off > 0; off >>= 1) {
      blo_x = fminf(blo_x, __shfl_xor_sync(0xffffffffu, blo_x, off));
      blo_y = fminf(blo_y, __shfl_xor_sync(0xffffffffu, blo_y, off));
      blo_z = fminf(blo_z, __shfl_xor_sync(0xffffffffu, blo_z, off));
      bhi_x = fmaxf(bhi_x, __shfl_xor_sync(0xffffffffu, bhi_x, off));
      bhi_y = fmaxf(bhi_y, __shfl_xor_sync(0xffffffffu, bhi_y, off));
      bhi_z = fmaxf(bhi_z, __shfl_xor_sync(0xffffffffu, bhi_z, off));
    }
    // a batch holds at most kBatch / 2 candidates per lane (the list depth)
    const int batch_cap = min(kBatch, (kBatch / 2) * base);
    long long fx = 0, fy = 0, fz = 0;
    // FP64 Coulomb energy sum of the cutoff form (see kExactE)
    double eU = 0.0;
    double pid_x = 0.0, pid_y = 0.0, pid_z = 0.0;
    if (kExactE) {
      const float4 li = spos_lo[i];
      pid_x = (double)pi.x + (double)li.x;
      pid_y = (double)pi.y + (double)li.y;
      pid_z = (double)pi.z + (double)li.z;
    }
    double Ri[3] = {0.0, 0.0, 0.0};
    if (kMolVir)
      for (int k = 0; k < 3; k++) Ri[k] = com[3 * (size_t)mi.y + k];

    int nb = 0;          // staged atoms in the current batch
    int home_lo = 0;     // staged range [home_lo, home_hi) of the home cell,
    int home_hi = 0;     // whose first entry has sorted index home_base;
    int home_base = 0;   // home-cell pairs are taken for i < j only
    auto flush_batch = [&]() {
      __syncwarp();
      int cnt = 0;
      if (active) {
        // home-cell entries t with ex_lo <= t < ex_lo + ex_n are j <= i
        const int ex_lo = home_lo;
        const unsigned ex_n =
            (unsigned)max(0, min(home_hi - home_lo, i - home_base + 1));
        const float2 nx = make_float2(-pi.x, -pi.x), ny = make_float2(-pi.y, -pi.y),
                     nz = make_float2(-pi.z, -pi.z);
        unsigned char *lst = &sm.list[0][lane];
        // the exclusion-range test only where the batch holds home-cell atoms
        // (the i < j rule); the other batches scan without it
        auto scan = [&](auto with_home) {
          constexpr bool kHome = decltype(with_home)::value;
          int t = sub;
          // two candidates per step with packed FP32 (FADD2 / FMUL2 / FFMA2)
          for (; t + L < nb; t += 2 * L) {
            const float4 a = sm.pos[t], b = sm.pos[t + L];
            const float2 dx = __fadd2_rn(make_float2(a.x, b.x), nx);
            const float2 dy = __fadd2_rn(make_float2(a.y, b.y), ny);
            const float2 dz = __fadd2_rn(make_float2(a.z, b.z), nz);
            float2 r2 = __fmul2_rn(dz, dz);
            r2 = __ffma2_rn(dy, dy, r2);
            r2 = __ffma2_rn(dx, dx, r2);
            if (r2.x <= mc.cut2 && (!kHome || (unsigned)(t - ex_lo) >= ex_n)) {
              lst[cnt * 32] = (unsigned char)t;
              cnt++;
            }
            if (r2.y <= mc.cut2 && (!kHome || (unsigned)(t + L - ex_lo) >= ex_n)) {
              lst[cnt * 32] = (unsigned char)(t + L);
              cnt++;
            }
          }
          if (t < nb) {
            const float4 a = sm.pos[t];
            const float dx = a.x - pi.x, dy = a.y - pi.y, dz = a.z - pi.z;
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            if (r2 <= mc.cut2 && (!kHome || (unsigned)(t - ex_lo) >= ex_n)) {
              lst[cnt * 32] = (unsigned char)t;
              cnt++;
            }
          }
        };
        if (home_hi > home_lo) scan(std::true_type{});
        else scan(std::false_type{});
      }
      // lists are walked in two phases when that is cheaper: every lane first
      // takes the first kmin entries of its own list (kmin = the shortest
      // active list), then the remaining entries of the longer lists are
      // dealt over the whole warp, so no lane idles while another finishes a
      // long list.  Leftovers go out in units of up to kDealUnit = 3
      // consecutive entries of one list (one search and one exchange of i
      // data per unit); a round of dealt units (shuffled i data, shared
      // i-force sums) is counted as 4 rounds of own pairs.  (Measured on the
      // 41k and 327k water boxes: units of 1, 2, 3, 4 and 6 at costs from
      // 1.5 to 8; 3 at 4 to 5 is best on both.)
      const int kmin = __reduce_min_sync(0xffffffffu, active ? cnt : 0x7fffffff);
      const int maxc = __reduce_max_sync(0xffffffffu, cnt);
      float px = 0.f, py = 0.f, pz = 0.f, pE = 0.f;
      float pw0 = 0.f, pw1 = 0.f, pw2 = 0.f, pw3 = 0.f, pw4 = 0.f, pw5 = 0.f;
      float pm0 = 0.f, pm1 = 0.f, pm2 = 0.f, pm3 = 0.f, pm4 = 0.f, pm5 = 0.f;
      int pc = 0;
      // One listed pair: staged j atom t and i atom (a4, moli, exclusion range
      // elo_..ehi_, LJ row ti_, sorted index ii, FP64 position pix..piz,
      // molecule centre rx..rz).  own: the lane's own atom (force summed in
      // px..pz); otherwise the atom of lane src (force to its shared sums).
      auto pair = [&](const int t, const bool own, const float4 a4, const int moli,
                      const int elo_, const int ehi_, const int ti_, const size_t ii,
                      const int src, const double pix, const double piy, const double piz,
                      const double rx, const double ry, const double rz) {
        const float4 pj = sm.pos[t];
        const float ddx = pj.x - a4.x, ddy = pj.y - a4.y, ddz = pj.z - a4.z;
        const float r2 = fmaf(ddx, ddx, fmaf(ddy, ddy, ddz * ddz));
        const int2 mj = sm.meta[t];
        int kind = 0;
        if (mj.y == moli) {
          kind = excl_kind(ex, elo_, ehi_, sidx[sm.gidx[t]]);
          if (kind == 2) return;
        }
        // 1/r: hardware reciprocal square root refined by one Newton-Raphson
        // step for 1/sqrt(x).
        float rinv = rsqrtf(r2);
        rinv = fmaf(0.5f * rinv, fmaf(-r2 * rinv, rinv, 1.0f), rinv);
        const float r2inv = rinv * rinv;
        float f;
        if constexpr (kForm == FORM_GENERIC) {
          // OneAtomPair / OneAtomPairTwo with any of the C1, C2, Cn switches
          // (OneAtomPair.h:62-105, OneAtomPairTwo.h:57-125)
          f = 0.0f;
          if (mc.swl.kind != SW_OFF) {
            const float4 p = s_lj[ti_ + mj.x];
            const float A = kind == 1 ? p.z : p.x;
            const float B = kind == 1 ? p.w : p.y;
            const float r6 = r2inv * r2inv * r2inv;
            float elj = fmaf(A, r6, -B) * r6;
            float flj = fmaf(12.0f * A, r6, -6.0f * B) * r6 * r2inv;
            float S, dS;
            switch_eval(mc.swl, r2, rinv, S, dS);
            f = fmaf(flj, S, -elj * dS);
            if (kEnergy) pE = fmaf(elj, S, pE);
          }
          if (mc.swc.kind != SW_OFF) {
            float qj = pj.w;
            if (kind == 1) qj *= mc.csf;
            const float ec = a4.w * qj * rinv;
            float S, dS;
            switch_eval(mc.swc, r2, rinv, S, dS);
            f += fmaf(ec * r2inv, S, -ec * dS);
            if (kEnergy) {
              const float eS = __fmul_rn(qj * rinv, S);
              if (own) kU.add(eS);
              else accU += (double)a4.w * (double)eS;
            }
          }
        } else if constexpr (kForm != FORM_CUTOFF) {
          // real-space Ewald (NonbondedFullEwaldSystemForce.h:803-823):
          // g = erfc(a r) / r, F / r = q_i q_j (g + 2a/sqrt(pi) e^{-a^2 r^2}) / r^2
          float qj = pj.w;
          if (kind == 1) qj *= mc.csf;
          const float x = mc.ea * (r2 * rinv);
          const float ex = expf(-x * x);
          float g;
          if constexpr (kForm == FORM_EWALD_POLY5) {
            const float t = __fdividef(1.0f, fmaf((float)kAsP, x, 1.0f));
            const float poly =
                t * fmaf(t, fmaf(t, fmaf(t, fmaf(t, (float)kAsA5, (float)kAsA4), (float)kAsA3),
                                 (float)kAsA2),
                         (float)kAsA1);
            g = poly * ex * rinv;
          } else {
            g = erfcf(x) * rinv;
          }
          f = a4.w * qj * fmaf(mc.ea2pi, ex, g) * r2inv;
          if (kEnergy) {
            const float eg = __fmul_rn(qj, g);
            if (own) kU.add(eg);
            else accU += (double)a4.w * (double)eg;
          }
        } else {
        const float4 p = s_lj[ti_ + mj.x];
        const float A = kind == 1 ? p.z : p.x;
        const float B = kind == 1 ? p.w : p.y;
        const float r6 = r2inv * r2inv * r2inv;
        float elj = fmaf(A, r6, -B) * r6;
        float flj = fmaf(12.0f * A, r6, -6.0f * B) * r6 * r2inv;
        {  // C2 switch, branch-free: value 1 below switchon, 0 beyond cutoff
          const float c2 = mc.rclj2 - r2;
          const float c4 = c2 * fmaf(2.0f, r2, mc.s2);
          const bool on = r2 >= mc.ron2;
          const bool in = r2 <= mc.rclj2;
          const float sv = in ? (on ? mc.s1 * (c2 * c4) : 1.0f) : 0.0f;
          const float sd = (in && on) ? mc.s3 * fmaf(c2, c2, -c4) : 0.0f;
          flj = fmaf(flj, sv, -elj * sd);
          elj = __fmul_rn(elj, sv);
        }
        float qj = pj.w;
        if (kind == 1) qj *= mc.csf;
        float fc;
        {  // C1 switched Coulomb, branch-free (zero beyond its cutoff)
          const bool inC = r2 <= mc.rcc2;
          const float ec = a4.w * qj * rinv;
          const float dist = r2 * rinv;
          const float sv = fmaf(-dist, fmaf(-r2, mc.c05_3, mc.c15_1), 1.0f);
          const float sd = fmaf(dist, mc.c15_3, -mc.c15_1 * rinv);
          fc = inC ? __fmul_rn(ec, fmaf(r2inv, sv, -sd)) : 0.f;
          if (kEnergy) {
            // q_j g(r), g = 1/r - 1.5/rc + 0.5 r^2/rc^3 (the C1-switched
            // 1/r), from the FP64 distance: the FP32 one rounds each term by
            // ~1e-7 of q_j / rc while the energy of a pair near the cutoff
            // is far smaller, and the total cancels to ~1e-4 of the pair
            // magnitudes on lattice-start boxes.  1/r from the FP32 value and
            // one Newton-Raphson step in FP64; g in FP64 keeps its absolute
            // error at ~1e-16 / r where it vanishes at the cutoff.  Computed
            // for every pair and added under the cutoff by selection: no
            // branch, so the FP64 chain overlaps the force arithmetic.
            const double ex_ = ((double)pj.x + (double)rsx[t]) - pix;
            const double ey_ = ((double)pj.y + (double)rsy[t]) - piy;
            const double ez_ = ((double)pj.z + (double)rsz[t]) - piz;
            const double r2d = fma(ex_, ex_, fma(ey_, ey_, ez_ * ez_));
            double rid = (double)rinv;
            rid = rid * fma(-0.5 * r2d, rid * rid, 1.5);
            const double gd = fma(mc.e05, r2d, rid - mc.e15);
            const double qjd = inC ? (double)qj : 0.0;
            if (own) eU = fma(qjd, gd, eU);
            else accU = fma(qjd * (double)a4.w, gd, accU);  // weighted by q_i here
          }
        }
        f = flj + fc;
        if (kEnergy) pE += elj;
        }
        // force on j in 2^-18 quanta (power-of-two scale: exact); the i
        // force, virial and molecular virial sums run in the same units.
        // (Every product that meets a sum is rounded explicitly, through
        // fmaf or __fmul_rn / __fsub_rn, so that no kernel instantiating this
        // body contracts it differently: the batched and single-system
        // kernels round every pair alike.)
        const float fq = f * kJScale;
        const float fxv = ddx * fq, fyv = ddy * fq, fzv = ddz * fq;
        if (own) {
          px = __fsub_rn(px, fxv);
          py = __fsub_rn(py, fyv);
          pz = __fsub_rn(pz, fzv);
        }
        // j force: int32 shared-memory quanta, or, for a contribution too
        // large for 32 of them to fit, straight into the int64 accumulator
        const float fm = fmaxf(fabsf(fxv), fmaxf(fabsf(fyv), fabsf(fzv)));
        // (the shared adds are unconditional, zero for a large contribution,
        // so the common path has no branch)
        const bool small = fm <= kJLimit;
        atomicAdd(&sm.jf[0][t], small ? __float2int_rn(fxv) : 0);
        atomicAdd(&sm.jf[1][t], small ? __float2int_rn(fyv) : 0);
        atomicAdd(&sm.jf[2][t], small ? __float2int_rn(fzv) : 0);
        if (!small) {
          // beyond the int64 accumulator's range (~2^31 cell units), or not
          // finite: the evaluation reports a device error
          if (!(fm < 2.8e14f)) atomicOr(err, 2);
          const size_t jg = (size_t)sm.gidx[t];
          atomicAdd(&facc[jg], (unsigned long long)__float2ll_rn(fxv * kJToGlobal));
          atomicAdd(&facc[(size_t)n + jg], (unsigned long long)__float2ll_rn(fyv * kJToGlobal));
          atomicAdd(&facc[2 * (size_t)n + jg],
                    (unsigned long long)__float2ll_rn(fzv * kJToGlobal));
        }
        if (!own) {
          // i force of another lane's atom: int32 shared quanta (at most
          // kBatch / 2 contributions per lane and batch, each within half
          // of kJLimit), else straight into the int64 accumulator
          if (fm <= 0.5f * kJLimit) {
            atomicAdd(&sm.fi[0][src], -__float2int_rn(fxv));
            atomicAdd(&sm.fi[1][src], -__float2int_rn(fyv));
            atomicAdd(&sm.fi[2][src], -__float2int_rn(fzv));
          } else {
            atomicAdd(&facc[ii], (unsigned long long)__float2ll_rn(-fxv * kJToGlobal));
            atomicAdd(&facc[(size_t)n + ii], (unsigned long long)__float2ll_rn(-fyv * kJToGlobal));
            atomicAdd(&facc[2 * (size_t)n + ii],
                      (unsigned long long)__float2ll_rn(-fzv * kJToGlobal));
          }
        }
        if (kEnergy) pc++;
        if (kVirial) {
          pw0 = fmaf(fxv, ddx, pw0); pw1 = fmaf(fxv, ddy, pw1); pw2 = fmaf(fxv, ddz, pw2);
          pw3 = fmaf(fyv, ddy, pw3); pw4 = fmaf(fyv, ddz, pw4); pw5 = fmaf(fzv, ddz, pw5);
          if (kMolVir && mj.y != moli) {
            // ScalarStructure::addVirial(fij, diff, comDiff): comDiff is the
            // minimal image of the two molecule centres (FP64), in cell units
            double cd[3];
            cd[0] = com[3 * (size_t)mj.y] - rx;
            cd[1] = com[3 * (size_t)mj.y + 1] - ry;
            cd[2] = com[3 * (size_t)mj.y + 2] - rz;
            ref_min_image(pb, cd);
            const float cx_ = (float)(cd[0] * inv_unit), cy_ = (float)(cd[1] * inv_unit),
                        cz_ = (float)(cd[2] * inv_unit);
            pm0 = fmaf(fxv, cx_, pm0); pm1 = fmaf(fxv, cy_, pm1); pm2 = fmaf(fxv, cz_, pm2);
            pm3 = fmaf(fyv, cy_, pm3); pm4 = fmaf(fyv, cz_, pm4); pm5 = fmaf(fzv, cz_, pm5);
          }
        }
      };
      int left = active ? cnt - kmin : 0;
      // leftovers are dealt in units of up to kDealUnit consecutive entries
      // of one lane's list, so that one search for the source lane and one
      // exchange of its atom's data serve several pairs
      int units = (left + kDealUnit - 1) / kDealUnit;
      int uinc = units;  // inclusive prefix of the unit counts
      for (int off = 1; off < 32; off <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, uinc, off);
        if (lane >= off) uinc += v;
      }
      int utot = __shfl_sync(0xffffffffu, uinc, 31);
      if (10 * (maxc - kmin) <= PMB200_SPREAD_COST * ((utot + 31) >> 5)) {
        utot = 0;  // one phase: each lane walks its whole list
        left = 0;
      }
      const int kown = active ? cnt - left : 0;
      for (int k = 0; k < kown; k++)
        pair(sm.list[k][lane], true, pi, mi.y, elo, ehi, ti, (size_t)i, lane, pid_x, pid_y,
             pid_z, Ri[0], Ri[1], Ri[2]);
      for (int base = 0; base < utot; base += 32) {
        const int u = base + lane;
        int src = 0;  // the lane whose leftovers hold unit u
        for (int step = 16; step > 0; step >>= 1) {
          const int v = __shfl_sync(0xffffffffu, uinc, src + step - 1);
          if (v <= u) src += step;
        }
        const int u0 = __shfl_sync(0xffffffffu, uinc, src) -
                       __shfl_sync(0xffffffffu, units, src);  // src's first unit
        const int lsrc = __shfl_sync(0xffffffffu, left, src);  // (every lane shuffles)
        const int k = kmin + kDealUnit * (u - u0);
        const int nk = u < utot ? min(kDealUnit, kmin + lsrc - k) : 0;
        float4 a4;
        a4.x = __shfl_sync(0xffffffffu, pi.x, src);
        a4.y = __shfl_sync(0xffffffffu, pi.y, src);
        a4.z = __shfl_sync(0xffffffffu, pi.z, src);
        a4.w = __shfl_sync(0xffffffffu, pi.w, src);
        const int moli = __shfl_sync(0xffffffffu, mi.y, src);
        const int elo_ = __shfl_sync(0xffffffffu, elo, src);
        const int ehi_ = __shfl_sync(0xffffffffu, ehi, src);
        const int ti_ = __shfl_sync(0xffffffffu, ti, src);
        const int ii = __shfl_sync(0xffffffffu, i, src);
        double pix = 0.0, piy = 0.0, piz = 0.0, rx = 0.0, ry = 0.0, rz = 0.0;
        if (kExactE) {
          pix = __shfl_sync(0xffffffffu, pid_x, src);
          piy = __shfl_sync(0xffffffffu, pid_y, src);
          piz = __shfl_sync(0xffffffffu, pid_z, src);
        }
        if (kMolVir) {
          rx = __shfl_sync(0xffffffffu, Ri[0], src);
          ry = __shfl_sync(0xffffffffu, Ri[1], src);
          rz = __shfl_sync(0xffffffffu, Ri[2], src);
        }
        for (int r = 0; r < nk; r++)
          pair(sm.list[k + r][src], false, a4, moli, elo_, ehi_, ti_, (size_t)ii, src, pix, piy,
               piz, rx, ry, rz);
      }
      if (utot > 0) {  // the shared i-force sums of the leftovers, per lane
        __syncwarp();
        fx += (long long)sm.fi[0][lane] << kJShift;
        fy += (long long)sm.fi[1][lane] << kJShift;
        fz += (long long)sm.fi[2][lane] << kJShift;
        sm.fi[0][lane] = sm.fi[1][lane] = sm.fi[2][lane] = 0;
      }
      fx += __float2ll_rn(px * kJToGlobal);
      fy += __float2ll_rn(py * kJToGlobal);
      fz += __float2ll_rn(pz * kJToGlobal);
      if (kEnergy) { accE += (double)pE; accP += (double)pc; }
      constexpr double kInvJ = 1.0 / (double)kJScale;  // quanta -> cell-unit forces
      if (kVirial) {
        w[0] += pw0 * kInvJ; w[1] += pw1 * kInvJ; w[2] += pw2 * kInvJ;
        w[3] += pw3 * kInvJ; w[4] += pw4 * kInvJ; w[5] += pw5 * kInvJ;
      }
      if (kMolVir) {
        mw[0] += pm0 * kInvJ; mw[1] += pm1 * kInvJ; mw[2] += pm2 * kInvJ;
        mw[3] += pm3 * kInvJ; mw[4] += pm4 * kInvJ; mw[5] += pm5 * kInvJ;
      }
      __syncwarp();
      // flush the batch's j forces to the global accumulator and clear them
      for (int t = lane; t < nb; t += 32) {
        const int j = sm.gidx[t];
#pragma unroll
        for (int q = 0; q < 3; q++) {
          const int v = sm.jf[q][t];
          if (v) atomicAdd(&facc[(size_t)q * n + j],
                           (unsigned long long)((long long)v << kJShift));
          sm.jf[q][t] = 0;
        }
      }
      nb = 0;
      home_lo = home_hi = 0;
      __syncwarp();
    };

    // This warp's share of the half-shell cells (dealt round-robin), taken
    // 32 at a time: each lane fetches one cell's atom range, a warp prefix sum
    // lays the cells end to end, and every batch is loaded with independent
    // loads (a binary search over the prefix finds each entry's cell), so the
    // L2 latency is paid once per batch rather than once per cell.
    const int first = slot, stride = nslots;
    const int nmine = first < st_ncells ? (st_ncells - first + stride - 1) / stride : 0;
    for (int g0 = 0; g0 < nmine; g0 += 32) {
      const int myq = g0 + lane;
      int cjs = 0, ccnt = 0;
      float csx = 0.f, csy = 0.f, csz = 0.f;
      double dsx = 0.0, dsy = 0.0, dsz = 0.0;  // the same shift in FP64 (energies)
      bool chome = false;
      if (myq < nmine) {
        const unsigned o = st_off[first + myq * stride];
        const int dx = (int)(o & 31u) - 8, dy = (int)((o >> 5) & 31u) - 8,
                  dz = (int)((o >> 10) & 31u) - 8;
        chome = (dx | dy | dz) == 0;
        int jx = cx + dx, jy = cy + dy, jz = cz + dz;
        bool inside = true;
        if (g.periodic) {
          // one wrap suffices: offsets reach at most ceil(rc / edge) <= n / 2
          // cells, since every box edge is at least twice the cutoff
          jx += jx < 0 ? g.nx : (jx >= g.nx ? -g.nx : 0);
          jy += jy < 0 ? g.ny : (jy >= g.ny ? -g.ny : 0);
          jz += jz < 0 ? g.nz : (jz >= g.nz ? -g.nz : 0);
        } else {
          inside = jx >= 0 && jx < g.nx && jy >= 0 && jy < g.ny && jz >= 0 && jz < g.nz;
        }
        if (inside) {
          const int jc = (jz * g.ny + jy) * g.nx + jx;
          cjs = start[jc];
          ccnt = start[jc + 1] - cjs;
        }
        if (g.tric) {
          // a lattice vector: rounded to FP32 once per cell offset
          cell_shift(g, g.m, 1.0, dx, dy, dz, dsx, dsy, dsz);
          csx = (float)dsx; csy = (float)dsy; csz = (float)dsz;
        } else {
          csx = (float)dx; csy = (float)dy * mc.ey; csz = (float)dz * mc.ez;
          dsx = csx; dsy = csy; dsz = csz;
        }
      }
      int incl = ccnt;  // inclusive prefix of the cells' atom counts
      for (int off = 1; off < 32; off <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += v;
      }
      const int total = __shfl_sync(0xffffffffu, incl, 31);
      const int excl = incl - ccnt;
      const unsigned hmask = __ballot_sync(0xffffffffu, chome && ccnt > 0);
      int h_excl = 0, h_cnt = 0, h_js = 0;
      if (hmask) {
        const int hl = __ffs(hmask) - 1;
        h_excl = __shfl_sync(0xffffffffu, excl, hl);
        h_cnt = __shfl_sync(0xffffffffu, ccnt, hl);
        h_js = __shfl_sync(0xffffffffu, cjs, hl);
      }
      // stage the cells' atoms 32 (or the batch's remaining room) at a
      // time; an atom farther than the cutoff from the box around this
      // chunk's i atoms is dropped here instead of being tested by every i
      // lane (home-cell atoms are always kept, so the home run stays whole)
      for (int f0 = 0; f0 < total;) {
        const int take = min(min(total - f0, batch_cap - nb), 32);
        const int f = f0 + lane;
        int c = 0;  // number of cells ending at or before f = f's cell
        for (int step = 16; step > 0; step >>= 1) {
          const int v = __shfl_sync(0xffffffffu, incl, c + step - 1);
          if (v <= f) c += step;
        }
        const int js_c = __shfl_sync(0xffffffffu, cjs, c);
        const int ex_c = __shfl_sync(0xffffffffu, excl, c);
        const float sx = __shfl_sync(0xffffffffu, csx, c);
        const float sy = __shfl_sync(0xffffffffu, csy, c);
        const float sz = __shfl_sync(0xffffffffu, csz, c);
        double dshx = sx, dshy = sy, dshz = sz;  // (the FP32 shift is exact unless triclinic)
        if (kExactE && g.tric) {
          dshx = __shfl_sync(0xffffffffu, dsx, c);
          dshy = __shfl_sync(0xffffffffu, dsy, c);
          dshz = __shfl_sync(0xffffffffu, dsz, c);
        }
        const bool home_atom = hmask && f >= h_excl && f < h_excl + h_cnt;
        bool keep = false;
        float4 a = make_float4(0.f, 0.f, 0.f, 0.f), p = a;
        int jg = 0;
        if (lane < take) {
          jg = js_c + (f - ex_c);
          a = spos[jg];
          p = a;
          p.x += sx; p.y += sy; p.z += sz;
          // squared distance to the box in the pair test's operation order:
          // per axis it is at most |p - x_i| for every i in the chunk, and
          // rounding is monotonic, so no pair the test accepts is dropped
          const float bx = fmaxf(fmaxf(blo_x - p.x, p.x - bhi_x), 0.f);
          const float by = fmaxf(fmaxf(blo_y - p.y, p.y - bhi_y), 0.f);
          const float bz = fmaxf(fmaxf(blo_z - p.z, p.z - bhi_z), 0.f);
          keep = home_atom || fmaf(bx, bx, fmaf(by, by, bz * bz)) <= mc.cut2;
        }
        const unsigned km = __ballot_sync(0xffffffffu, keep);
        if (keep) {
          const int slot = nb + __popc(km & ((1u << lane) - 1u));
          sm.pos[slot] = p;
          sm.meta[slot] = smeta[jg];
          sm.gidx[slot] = jg;
          if (kExactE) {  // coordinate, residual and shift in FP64, less the staged value
            const float4 lj = spos_lo[jg];
            rsx[slot] = (float)((((double)a.x + (double)lj.x) + dshx) - (double)p.x);
            rsy[slot] = (float)((((double)a.y + (double)lj.y) + dshy) - (double)p.y);
            rsz[slot] = (float)((((double)a.z + (double)lj.z) + dshz) - (double)p.z);
          }
        }
        const unsigned hm = __ballot_sync(0xffffffffu, keep && home_atom);
        if (hm) {  // the part of the home cell staged in this round
          const int fl = __ffs(hm) - 1, ll = 31 - __clz(hm);
          if (home_hi == home_lo) {
            home_lo = nb + __popc(km & ((1u << fl) - 1u));
            home_base = h_js + (f0 + fl - h_excl);
          }
          home_hi = nb + __popc(km & ((2u << ll) - 1u));
        }
        nb += __popc(km);
        f0 += take;
        if (batch_cap - nb < 16) flush_batch();
      }
    }
    if (nb > 0) flush_batch();

    // the i forces: summed over the atom's lanes [lane - sub, seg_end) into
    // its first lane (after the step with offset d, a lane holds the sum of
    // its lanes up to 2d ahead, within the atom), then the global accumulator
    const int seg_end = lane - sub + L;
    for (int off = 1; off < base + (extra ? 1 : 0); off <<= 1) {
      const long long vx = __shfl_down_sync(0xffffffffu, fx, off);
      const long long vy = __shfl_down_sync(0xffffffffu, fy, off);
      const long long vz = __shfl_down_sync(0xffffffffu, fz, off);
      if (lane + off < seg_end) { fx += vx; fy += vy; fz += vz; }
    }
    if (active && sub == 0) {
      atomicAdd(&facc[i], (unsigned long long)fx);
      atomicAdd(&facc[(size_t)n + i], (unsigned long long)fy);
      atomicAdd(&facc[2 * (size_t)n + i], (unsigned long long)fz);
    }
    if (kEnergy && active) {
      // the own-pair Coulomb sum is per i-atom: weight it by q_i (FP64)
      const double qi = (double)pi.w;
      if (kExactE) accU += qi * eU;
      else accU += qi * ((double)kU.s - (double)kU.c);
    }
    kU = KahanF();
  }
  if (kEnergy || kVirial) {
    double v[ACC_MV];
#pragma unroll
    for (int k = 0; k < ACC_MV; k++) v[k] = 0.0;
    v[ACC_ECOUL] = accU; v[ACC_ELJ] = accE; v[ACC_PAIRS] = accP;
#pragma unroll
    for (int k = 0; k < 6; k++) { v[ACC_W + k] = w[k]; v[ACC_MW + k] = mw[k]; }
    write_partial_row<kVirial ? ACC_MV : ACC_E>(v, lane, partial_row);
  }
}

// One warp per block, `slots` blocks per i-cell (block b: cell cell0 + b /
// slots, stencil entries b % slots + k * slots), so a warp that finishes early
// frees its slot for the next block instead of waiting for the cell's other
// warps.  More slots mean more, shorter warps (better balance, more per-warp
// setup); the host picks 8 for forces-only launches on sparse cells and 4
// otherwise (kMaxCellSlots bounds the partial rows).  Dynamic shared memory:
// the LJ table (ntypes^2 float4, cutoff and generic forms) and then the
// stencil offsets.  Forces-only launches are held to 72 registers, so that
// shared memory (~8.4 KB per block with the per-block reserve) sets the
// residency at 27 blocks per SM; energy launches (~10 KB) to the registers
// of 19 blocks per SM (measured on the 41k water box: 19, 20, 21, 22 blocks
// took 167, 171, 171, 179 us, the higher counts through spilled registers);
// the virial variants keep the compiler's choice.
constexpr int kMaxCellSlots = 8;
constexpr int kEnergyCellSlots = 4;  // energy / virial launches (the ones with partial rows)


// kGlobalLj: the LJ table (more than kMaxTypes types) is read from global
// memory through L1 instead of being staged in shared memory.
template <int kForm, bool kEnergy, bool kVirial, bool kMolVir, bool kGlobalLj = false>
#ifndef PMB200_ENERGY_BLOCKS
#define PMB200_ENERGY_BLOCKS 19  // resident blocks per SM asked of energy launches
#endif
__global__ void __launch_bounds__(32, kVirial ? 1 : (kEnergy ? PMB200_ENERGY_BLOCKS : 26))
k_pair_mixed(GridParams g, MixedConsts mc, const HalfStencil st, int ntypes, const float4 *__restrict__ lj32,
             const int *__restrict__ start, const float4 *__restrict__ spos,
             const int2 *__restrict__ smeta, const int *__restrict__ sidx,
             const int *__restrict__ ex_start, const int2 *__restrict__ ex,
             unsigned long long *__restrict__ facc, int n, int *__restrict__ err,
             double *__restrict__ partial, const PbcRef pb, const double *__restrict__ com,
             int slots, const float4 *__restrict__ spos_lo, int cell0) {
  extern __shared__ float4 s_dyn[];
  constexpr int kB = kEnergy ? kBatchE : kBatch;
  __shared__ MixedWarpSmemT<kB> sm;
  __shared__ float s_res[(kEnergy && kForm == FORM_CUTOFF) ? 3 * kB : 1];
  constexpr bool kLj = kForm == FORM_CUTOFF || kForm == FORM_GENERIC;
  const int nlj = (kLj && !kGlobalLj) ? ntypes * ntypes : 0;
  float4 *s_lj = s_dyn;
  unsigned short *s_st = reinterpret_cast<unsigned short *>(s_dyn + nlj);
  const int lane = threadIdx.x;
  for (int k = lane; k < nlj; k += 32) s_lj[k] = lj32[k];
  for (int k = lane; k < st.ncells; k += 32) s_st[k] = st.off[k];
  for (int t = lane; t < kB; t += 32) sm.jf[0][t] = sm.jf[1][t] = sm.jf[2][t] = 0;
  sm.fi[0][lane] = sm.fi[1][lane] = sm.fi[2][lane] = 0;
  __syncwarp();
  // a launch that overlaps the cell build's last kernel waits for it here,
  // after a prologue that reads only data written before that kernel started
  pdl_wait();
  const int cell = cell0 + (int)(blockIdx.x / slots);  // cells cell0.. (a shard's range)
  if (cell >= g.ncell) return;  // uniform per block
  mixed_task<kForm, kEnergy, kVirial, kMolVir, MixedWarpSmemT<kB>>(
      g, mc, s_st, st.ncells, blockIdx.x % slots, slots, ntypes, kGlobalLj ? lj32 : s_lj, cell,
      start,
      spos, smeta, sidx, ex_start, ex, facc, n, partial + (size_t)blockIdx.x * kNacc, pb, com,
      sm, err, s_res, spos_lo);
}

// Blocks per i-cell of a k_pair_mixed launch: 8 for forces-only launches
// when cells hold at most 18 atoms on average (measured on water boxes:
// 15 atoms per cell 4% faster than 4; 24 per cell 5% slower), else 4.
inline int mixed_cell_slots(bool energy_or_virial, int natoms, int ncell) {
  if (energy_or_virial) return kEnergyCellSlots;
  return natoms <= 18LL * ncell ? kMaxCellSlots : 4;
}

// Dynamic shared memory of a k_pair_mixed launch.
inline size_t mixed_smem_bytes(int form, int ntypes, int st_ncells) {
  const size_t lj = ((form == FORM_CUTOFF || form == FORM_GENERIC) && ntypes <= kMaxTypes)
                        ? sizeof(float4) * (size_t)ntypes * ntypes : 0;
  return lj + ((sizeof(unsigned short) * (size_t)st_ncells + 15) & ~(size_t)15);
}

// Fixed-point force accumulator (sorted order, [3][n], 2^-32 quanta in cell
// units) -> FP64 forces in the caller's atom order, accumulated or
// overwritten.
__global__ void k_finalize(int n, const unsigned long long *__restrict__ facc,
                           const int *__restrict__ sidx, double scale, int accumulate,
                           double *__restrict__ forces) {
  pdl_wait();
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int o = sidx[j];
  double *fo = forces + 3 * (size_t)o;
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const double v = (double)(long long)facc[(size_t)q * n + j] * scale;
    fo[q] = accumulate ? fo[q] + v : v;
  }
}

// The reference's per-pair arithmetic in FP64 for a pair at squared
// distance r2 (A^2): OneAtomPairTwo::doOneAtomPair's LJ(C2) + Coulomb(C1)
// (OneAtomPairTwo.h:57-125) for the cutoff form, the generic switches and
// the tabulated LJ (OneAtomPair.h:56-111) for the generic form, the
// real-space Ewald term otherwise.  ti = type_i * ntypes, tj = type_j, kind
// the pair's exclusion class (1: modified), qi / qj the scaled charges.  Out:
// f = force / r, e1 the LJ energy, e2 the Coulomb energy.  Shared by the FP64
// kernels so that they round every pair alike.
template <int kForm>
__device__ __forceinline__ void fp64_pair(const Fp64Consts &mc, const double4 *__restrict__ lj64,
                                          int ti, int tj, int kind, double r2, double qi,
                                          double qj, double &f, double &e1, double &e2) {
  e1 = 0.0;
  e2 = 0.0;
  if constexpr (kForm == FORM_GENERIC) {
    f = 0.0;
    const double rd2 = 1.0 / r2;
    const double rinv = sqrt(rd2);
    if (mc.ljtab) {  // no Coulomb term beside the table
      const double4 p = lj64[ti + tj];
      lj_table_eval(mc.ljtab, mc.tfirst, mc.tlast, r2, kind == 1 ? p.z : p.x,
                    kind == 1 ? p.w : p.y, e1, f);
    } else if (mc.swl.kind != SW_OFF) {
      const double4 p = lj64[ti + tj];
      const double A = kind == 1 ? p.z : p.x;
      const double B = kind == 1 ? p.w : p.y;
      const double r6 = rd2 * rd2 * rd2;
      const double r12 = r6 * r6;
      const double r6B = B * r6, r12A = A * r12;
      e1 = r12A - r6B;
      double f1 = 12.0 * r12A * rd2 - 6.0 * r6B * rd2;
      double S, dS;
      switch_eval(mc.swl, r2, rinv, S, dS);
      f1 = f1 * S - e1 * dS;
      e1 = e1 * S;
      f += f1;
    }
    if (mc.swc.kind != SW_OFF) {
      e2 = qi * qj * rinv;
      if (kind == 1) e2 *= mc.csf;
      double f2 = e2 * rd2;
      double S, dS;
      switch_eval(mc.swc, r2, rinv, S, dS);
      f2 = f2 * S - e2 * dS;
      e2 = e2 * S;
      f += f2;
    }
  } else if constexpr (kForm != FORM_CUTOFF) {
    // NonbondedFullEwaldSystemForce::realTerm's pair arithmetic
    // (NonbondedFullEwaldSystemForce.h:803-823)
    const double r = sqrt(r2);
    double qq = qi * qj;
    if (kind == 1) qq *= mc.csf;
    if constexpr (kForm == FORM_EWALD_POLY5) {
      const double rr = 1.0 / r;
      const double ar = mc.ea * r;
      const double e = qq * exp(-ar * ar);
      const double t = 1.0 / (1.0 + kAsP * ar);
      const double poly =
          (t) * (kAsA1 + (t) * (kAsA2 + (t) * (kAsA3 + (t) * (kAsA4 + (t) * kAsA5))));
      e2 = poly * e * rr;
      f = ((e2 + mc.ea2pi * e) * rr * rr);
    } else {
      const double a = erfc(mc.ea * r) / r;
      e2 = qq * a;
      f = qq * (a + mc.ea2pi * exp(-mc.ea2 * r2)) / r2;
    }
  } else {
    const double rd2 = 1.0 / r2;
    const double4 p = lj64[ti + tj];
    const double A = kind == 1 ? p.z : p.x;
    const double B = kind == 1 ? p.w : p.y;
    const double r6 = rd2 * rd2 * rd2;
    const double r12 = r6 * r6;
    const double r6B = B * r6, r12A = A * r12;
    e1 = r12A - r6B;
    double f1 = 12.0 * r12A * rd2 - 6.0 * r6B * rd2;
    double sv = 1.0, sd = 0.0;
    if (r2 > mc.rclj2) sv = 0.0;
    else if (r2 >= mc.ron2) {
      const double c2 = mc.rclj2 - r2;
      const double c4 = c2 * (mc.s2 + 2.0 * r2);
      sv = mc.s1 * (c2 * c4);
      sd = mc.s3 * (c2 * c2 - c4);
    }
    f1 = f1 * sv - e1 * sd;
    e1 = e1 * sv;
    e2 = qi * qj * sqrt(rd2);
    if (kind == 1) e2 *= mc.csf;
    double f2 = e2 * rd2;
    if (r2 > mc.rcc2) { e2 = 0.0; f2 = 0.0; }
    else {
      const double dist = sqrt(r2);
      const double v = 1.0 - dist * (mc.c15_1 - r2 * mc.c05_3);
      const double dv = -mc.c15_1 / dist + dist * mc.c15_3;
      f2 = f2 * v - e2 * dv;
      e2 = e2 * v;
    }
    f = f1 + f2;
  }
}

// ---------------------------------------------------------------------------
// Plain FP64 pair kernel: the same cell-pair walk and lane mapping as the
// mixed kernel, with the reference's FP64 per-pair arithmetic
// (OneAtomPairTwo::doOneAtomPair) in Angstrom, forces summed in FP64.
// ---------------------------------------------------------------------------
template <int kForm, bool kEnergy, bool kVirial, bool kMolVir>
__global__ void __launch_bounds__(128)
k_pair_fp64(GridParams g, Fp64Consts mc, const Stencil st, int ntypes, const double4 *__restrict__ lj64,
            const int *__restrict__ start, const double4 *__restrict__ spos,
            const int2 *__restrict__ smeta, const int *__restrict__ sidx,
            const int *__restrict__ ex_start, const int2 *__restrict__ ex,
            double *__restrict__ forces, int accumulate, double *__restrict__ partial,
            const PbcRef pb, const double *__restrict__ com, int cell0 = 0,
            int ncells = 1 << 30) {
  const int lane = threadIdx.x & 31;
  // one warp per i-cell of [cell0, cell0 + ncells)
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int cell = cell0 + wid;
  if (wid >= ncells || cell >= g.ncell) return;
  const int cx = cell % g.nx;
  const int cy = (cell / g.nx) % g.ny;
  const int cz = cell / (g.nx * g.ny);
  const int cs = start[cell], ce = start[cell + 1];
  double accC = 0, accE = 0, accP = 0;
  double w[6] = {0, 0, 0, 0, 0, 0};
  double mw[6] = {0, 0, 0, 0, 0, 0};
  for (int c0 = cs; c0 < ce; c0 += 32) {
    const int m = min(32, ce - c0);
    const int L = lanes_per_atom(m);
    const int ia = lane / L;
    const int sub = lane % L;
    const bool active = ia < m;
    const int i = c0 + (active ? ia : 0);
    const double4 pi = spos[i];
    const int2 mi = smeta[i];
    const int oi = sidx[i];
    const int elo = ex_start[oi], ehi = ex_start[oi + 1];
    const int ti = mi.x * ntypes;
    double fx = 0, fy = 0, fz = 0;
    double Ri[3] = {0.0, 0.0, 0.0};
    if (kMolVir)
      for (int k = 0; k < 3; k++) Ri[k] = com[3 * (size_t)mi.y + k];
    for (int r = 0; r < g.nrows; r++) {
      const Row row = st.rows[r];
      int jy = cy + row.dy, jz = cz + row.dz;
      if (!g.periodic && (jy < 0 || jy >= g.ny || jz < 0 || jz >= g.nz)) continue;
      while (jy < 0) jy += g.ny;
      while (jy >= g.ny) jy -= g.ny;
      while (jz < 0) jz += g.nz;
      while (jz >= g.nz) jz -= g.nz;
      const int rowbase = (jz * g.ny + jy) * g.nx;
      for (int dx = row.dxlo; dx <= row.dxhi; dx++) {
        int jx = cx + dx;
        if (!g.periodic && (jx < 0 || jx >= g.nx)) continue;
        jx += jx < 0 ? g.nx : (jx >= g.nx ? -g.nx : 0);  // |dx| <= n / 2: one wrap
        const int jc = rowbase + jx;
        const int js = start[jc], je = start[jc + 1];
        double sx, sy, sz;  // the neighbour cell's shift (A)
        cell_shift(g, g.ec, 1.0, dx, row.dy, row.dz, sx, sy, sz);
        for (int j = js + sub; j < je; j += L) {
          const double4 pj = spos[j];
          const double ddx = (pj.x + sx) - pi.x;
          const double ddy = (pj.y + sy) - pi.y;
          const double ddz = (pj.z + sz) - pi.z;
          const double r2 = ddx * ddx + ddy * ddy + ddz * ddz;
          if (!(r2 <= mc.cut2) || j == i || !active) continue;
          const int2 mj = smeta[j];
          int kind = 0;
          if (mj.y == mi.y) {
            kind = excl_kind(ex, elo, ehi, sidx[j]);
            if (kind == 2) continue;
          }
          double f, e1, e2;
          fp64_pair<kForm>(mc, lj64, ti, mj.x, kind, r2, pi.w, pj.w, f, e1, e2);
          fx -= ddx * f; fy -= ddy * f; fz -= ddz * f;
          if (kEnergy) { accE += e1; accC += e2; accP += 1.0; }
          if (kVirial) {
            const double fxv = ddx * f, fyv = ddy * f, fzv = ddz * f;
            w[0] += fxv * ddx; w[1] += fxv * ddy; w[2] += fxv * ddz;
            w[3] += fyv * ddy; w[4] += fyv * ddz; w[5] += fzv * ddz;
            if (kMolVir && mj.y != mi.y) {
              double cd[3];
              for (int q = 0; q < 3; q++) cd[q] = com[3 * (size_t)mj.y + q] - Ri[q];
              ref_min_image(pb, cd);
              mw[0] += fxv * cd[0]; mw[1] += fxv * cd[1]; mw[2] += fxv * cd[2];
              mw[3] += fyv * cd[1]; mw[4] += fyv * cd[2]; mw[5] += fzv * cd[2];
            }
          }
        }
      }
    }
    for (int off = 1; off < L; off <<= 1) {
      fx += __shfl_xor_sync(0xffffffffu, fx, off);
      fy += __shfl_xor_sync(0xffffffffu, fy, off);
      fz += __shfl_xor_sync(0xffffffffu, fz, off);
    }
    if (active && sub == 0) {
      double *fo = forces + 3 * (size_t)oi;
      if (accumulate) { fo[0] += fx; fo[1] += fy; fo[2] += fz; }
      else { fo[0] = fx; fo[1] = fy; fo[2] = fz; }
    }
  }
  if (kEnergy || kVirial) {
    double v[ACC_MV];
#pragma unroll
    for (int k = 0; k < ACC_MV; k++) v[k] = 0.0;
    v[ACC_ECOUL] = accC; v[ACC_ELJ] = accE; v[ACC_PAIRS] = accP;
#pragma unroll
    for (int k = 0; k < 6; k++) { v[ACC_W + k] = w[k]; v[ACC_MW + k] = mw[k]; }
    write_partial_row<kVirial ? ACC_MV : ACC_E>(v, lane, partial + (size_t)cell * kNacc);
  }
}

// ---------------------------------------------------------------------------
// FP64 pair kernel on the half shell (the evaluation kernel of FP64
// contexts): the mixed kernel's task split -- one warp per block, each warp
// one i-cell and one share of the half-shell cell offsets (the same
// HalfStencil; home-cell pairs taken for i < j) -- with fp64_pair's
// arithmetic and each pair evaluated once, its force added to both atoms
// (Newton's third law, as NonbondedCutoffForce's cell-pair loop does).  The
// warp stages the atoms of its cells (positions in the i-cell frame, FP64)
// kB64 at a time in shared memory, leaving out those farther than the
// cutoff from the box around the chunk's i atoms (no pair of theirs is
// within it), and every i atom meets every staged atom.  The lanes of i atom ia
// take the batch in blocks of L entries, block (ia + k) mod nsteps at step k,
// so that at each step no two lanes touch the same staged atom: j forces are
// summed in shared memory without atomics, in step order, and i forces in
// registers.  Both reach the global accumulator as exact two-word
// fixed-point numbers (fix2_split: multiples of 2^-20 and of 2^-68
// kcal/mol/A), whose integer sums are the same in any order: the results are
// deterministic.  Accumulator acc[6][n] int64, sorted order, words {hi x,
// hi y, hi z, lo x, lo y, lo z}.  Energy and virial partials: one row per
// block.
constexpr int kB64 = 64;
constexpr double kFix2Hi = 1048576.0;            // 2^20
constexpr double kFix2Lo = 281474976710656.0;    // 2^48 (below 2^-20)
constexpr double kFix2Max = 6.0e10;              // < 2^36 kcal/mol/A
struct Fp64WarpSmem {
  double4 pos[kB64];  // staged j: position in the i-cell frame (A), charge
  int2 meta[kB64];    // type, molecule
  int jidx[kB64];     // sorted index; bit 31: an atom of the home cell
  double jf[3][kB64]; // j force sums of the batch
};

// v = (hi + lo 2^-48) 2^-20 exactly: hi = rint(v 2^20); the remainder
// v 2^20 - hi (exact, |.| <= 1/2) scaled by 2^48 and rounded (error <= 2^-69
// kcal/mol/A).  A summed force component of kFix2Max or more (or not finite)
// makes the evaluation report a device error: below it every word sum stays
// within int64 for up to 2^13 such contributions.
__device__ __forceinline__ void fix2_add(unsigned long long *__restrict__ acc, size_t n, size_t j,
                                         int q, double v, int *__restrict__ err) {
  if (!(fabs(v) < kFix2Max)) {
    atomicOr(err, 2);
    return;
  }
  const double s = v * kFix2Hi;
  const double h = rint(s);
  const long long hi = (long long)h;
  const long long lo = __double2ll_rn((s - h) * kFix2Lo);
  if (hi) atomicAdd(&acc[(size_t)q * n + j], (unsigned long long)hi);
  if (lo) atomicAdd(&acc[(size_t)(3 + q) * n + j], (unsigned long long)lo);
}

#ifndef PMB200_FP64_BLOCKS
// resident blocks per SM asked of the FP64 kernel (measured on the 41k water
// box with energies: 20 and 24 blocks 0.439 ms, 28 blocks 0.426 ms)
#define PMB200_FP64_BLOCKS 28
#endif
template <int kForm, bool kEnergy, bool kVirial, bool kMolVir>
__global__ void __launch_bounds__(32, kVirial ? 1 : PMB200_FP64_BLOCKS)
k_pair_fp64_half(GridParams g, Fp64Consts mc, const HalfStencil st, int slots, int ntypes,
                 const double4 *__restrict__ lj64, const int *__restrict__ start,
                 const double4 *__restrict__ spos, const int2 *__restrict__ smeta,
                 const int *__restrict__ sidx, const int *__restrict__ ex_start,
                 const int2 *__restrict__ ex, unsigned long long *__restrict__ acc, int n,
                 double *__restrict__ partial, const PbcRef pb, const double *__restrict__ com,
                 int *__restrict__ err) {
  __shared__ Fp64WarpSmem sm;
  const int lane = threadIdx.x;
  const int cell = (int)(blockIdx.x / slots), slot = (int)(blockIdx.x % slots);
  if (cell >= g.ncell) return;  // uniform per block
  const int cx = cell % g.nx;
  const int cy = (cell / g.nx) % g.ny;
  const int cz = cell / (g.nx * g.ny);
  const int cs = start[cell], ce = start[cell + 1];
  for (int t = lane; t < kB64; t += 32) sm.jf[0][t] = sm.jf[1][t] = sm.jf[2][t] = 0.0;
  double accC = 0, accE = 0, accP = 0;
  double w[6] = {0, 0, 0, 0, 0, 0};
  double mw[6] = {0, 0, 0, 0, 0, 0};
  for (int c0 = cs; c0 < ce; c0 += 32) {
    const int m = min(32, ce - c0);
    const int L = lanes_per_atom(m);
    const int ia = lane / L;
    const int sub = lane % L;
    const bool active = ia < m;
    const int i = c0 + (active ? ia : 0);
    const double4 pi = spos[i];
    const int2 mi = smeta[i];
    const int oi = sidx[i];
    const int elo = ex_start[oi], ehi = ex_start[oi + 1];
    const int ti = mi.x * ntypes;
    double fx = 0, fy = 0, fz = 0;
    double Ri[3] = {0.0, 0.0, 0.0};
    if (kMolVir)
      for (int k = 0; k < 3; k++) Ri[k] = com[3 * (size_t)mi.y + k];
    // the box around the chunk's i atoms
    double blo_x = pi.x, blo_y = pi.y, blo_z = pi.z, bhi_x = pi.x, bhi_y = pi.y, bhi_z = pi.z;
    for (int off = 16; off > 0; off >>= 1) {
      blo_x = fmin(blo_x, __shfl_xor_sync(0xffffffffu, blo_x, off));
      blo_y = fmin(blo_y, __shfl_xor_sync(0xffffffffu, blo_y, off));
      blo_z = fmin(blo_z, __shfl_xor_sync(0xffffffffu, blo_z, off));
      bhi_x = fmax(bhi_x, __shfl_xor_sync(0xffffffffu, bhi_x, off));
      bhi_y = fmax(bhi_y, __shfl_xor_sync(0xffffffffu, bhi_y, off));
      bhi_z = fmax(bhi_z, __shfl_xor_sync(0xffffffffu, bhi_z, off));
    }
    int nb = 0;
    // every i atom of the chunk against the nb staged atoms, then the j
    // forces out and the batch emptied
    auto process = [&]() {
      __syncwarp();
      const int nblk = (nb + L - 1) / L;
      const int nsteps = max(nblk, m);  // >= m: the atoms' blocks differ at every step
      for (int k = 0; k < nsteps; k++) {
        int blk = ia + k;
        if (blk >= nsteps) blk -= nsteps;
        const int t = blk * L + sub;
        if (active && t < nb) {
          const int jw = sm.jidx[t];
          const int j = jw & 0x7fffffff;
          const double4 pj = sm.pos[t];
          const double ddx = pj.x - pi.x;
          const double ddy = pj.y - pi.y;
          const double ddz = pj.z - pi.z;
          const double r2 = ddx * ddx + ddy * ddy + ddz * ddz;
          const int2 mj = sm.meta[t];
          int kind = (jw < 0 && j <= i) ? 2 : 0;  // home cell: pairs i < j only
          if (kind == 0 && r2 <= mc.cut2 && mj.y == mi.y) kind = excl_kind(ex, elo, ehi, sidx[j]);
          if (kind != 2 && r2 <= mc.cut2) {
            double f, e1, e2;
            fp64_pair<kForm>(mc, lj64, ti, mj.x, kind, r2, pi.w, pj.w, f, e1, e2);
            const double fxv = ddx * f, fyv = ddy * f, fzv = ddz * f;
            fx -= fxv; fy -= fyv; fz -= fzv;
            sm.jf[0][t] += fxv;
            sm.jf[1][t] += fyv;
            sm.jf[2][t] += fzv;
            if (kEnergy) { accE += e1; accC += e2; accP += 1.0; }
            if (kVirial) {
              w[0] += fxv * ddx; w[1] += fxv * ddy; w[2] += fxv * ddz;
              w[3] += fyv * ddy; w[4] += fyv * ddz; w[5] += fzv * ddz;
              if (kMolVir && mj.y != mi.y) {
                double cd[3];
                for (int qq = 0; qq < 3; qq++) cd[qq] = com[3 * (size_t)mj.y + qq] - Ri[qq];
                ref_min_image(pb, cd);
                mw[0] += fxv * cd[0]; mw[1] += fxv * cd[1]; mw[2] += fxv * cd[2];
                mw[3] += fyv * cd[1]; mw[4] += fyv * cd[2]; mw[5] += fzv * cd[2];
              }
            }
          }
        }
        __syncwarp();
      }
      for (int t = lane; t < nb; t += 32) {
        const size_t j = (size_t)(sm.jidx[t] & 0x7fffffff);
#pragma unroll
        for (int qq = 0; qq < 3; qq++) {
          const double v = sm.jf[qq][t];
          if (v != 0.0) fix2_add(acc, (size_t)n, j, qq, v, err);
          sm.jf[qq][t] = 0.0;
        }
      }
      nb = 0;
      __syncwarp();
    };
    for (int q = slot; q < st.ncells; q += slots) {
      const unsigned o = st.off[q];
      const int dx = (int)(o & 31u) - 8, dy = (int)((o >> 5) & 31u) - 8,
                dz = (int)((o >> 10) & 31u) - 8;
      const int homebit = (dx | dy | dz) == 0 ? (int)0x80000000u : 0;
      int jx = cx + dx, jy = cy + dy, jz = cz + dz;
      if (g.periodic) {
        // one wrap suffices: offsets reach at most ceil(rc / edge) <= n / 2
        jx += jx < 0 ? g.nx : (jx >= g.nx ? -g.nx : 0);
        jy += jy < 0 ? g.ny : (jy >= g.ny ? -g.ny : 0);
        jz += jz < 0 ? g.nz : (jz >= g.nz ? -g.nz : 0);
      } else if (jx < 0 || jx >= g.nx || jy < 0 || jy >= g.ny || jz < 0 || jz >= g.nz) {
        continue;  // uniform per warp
      }
      const int jc = (jz * g.ny + jy) * g.nx + jx;
      const int js = start[jc], cnt = start[jc + 1] - js;
      double sx, sy, sz;  // the neighbour cell's shift (A)
      cell_shift(g, g.ec, 1.0, dx, dy, dz, sx, sy, sz);
      for (int f0 = 0; f0 < cnt;) {
        const int take = min(min(cnt - f0, kB64 - nb), 32);
        bool keep = false;
        double4 p = make_double4(0.0, 0.0, 0.0, 0.0);
        const int j = js + f0 + lane;
        if (lane < take) {
          p = spos[j];
          p.x += sx; p.y += sy; p.z += sz;
          // squared distance to the box in the pair test's operation order:
          // per axis at most |p - x_i| for every i in the chunk, and rounding
          // is monotonic, so no pair the test accepts is dropped
          const double bx = fmax(fmax(blo_x - p.x, p.x - bhi_x), 0.0);
          const double by = fmax(fmax(blo_y - p.y, p.y - bhi_y), 0.0);
          const double bz = fmax(fmax(blo_z - p.z, p.z - bhi_z), 0.0);
          keep = bx * bx + by * by + bz * bz <= mc.cut2;
        }
        const unsigned km = __ballot_sync(0xffffffffu, keep);
        if (keep) {
          const int slot = nb + __popc(km & ((1u << lane) - 1u));
          sm.pos[slot] = p;
          sm.meta[slot] = smeta[j];
          sm.jidx[slot] = j | homebit;
        }
        nb += __popc(km);
        f0 += take;
        if (nb > kB64 - 32) process();  // less than a full round of room left
      }
    }
    if (nb > 0) process();
    for (int off = 1; off < L; off <<= 1) {
      fx += __shfl_xor_sync(0xffffffffu, fx, off);
      fy += __shfl_xor_sync(0xffffffffu, fy, off);
      fz += __shfl_xor_sync(0xffffffffu, fz, off);
    }
    if (active && sub == 0) {
      fix2_add(acc, (size_t)n, (size_t)i, 0, fx, err);
      fix2_add(acc, (size_t)n, (size_t)i, 1, fy, err);
      fix2_add(acc, (size_t)n, (size_t)i, 2, fz, err);
    }
  }
  if (kEnergy || kVirial) {
    double v[ACC_MV];
#pragma unroll
    for (int k = 0; k < ACC_MV; k++) v[k] = 0.0;
    v[ACC_ECOUL] = accC; v[ACC_ELJ] = accE; v[ACC_PAIRS] = accP;
#pragma unroll
    for (int k = 0; k < 6; k++) { v[ACC_W + k] = w[k]; v[ACC_MW + k] = mw[k]; }
    write_partial_row<kVirial ? ACC_MV : ACC_E>(v, lane, partial + (size_t)blockIdx.x * kNacc);
  }
}

// The FP64 half-shell kernel's accumulator (sorted order, fix2 words
// [6][n]) -> forces in the caller's atom order, accumulated or overwritten.
__global__ void k_finalize64(int n, const unsigned long long *__restrict__ acc,
                             const int *__restrict__ sidx, int accumulate,
                             double *__restrict__ forces) {
  pdl_wait();
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  double *fo = forces + 3 * (size_t)sidx[j];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const double hi = (double)(long long)acc[(size_t)q * n + j];
    const double lo = (double)(long long)acc[(size_t)(3 + q) * n + j];
    const double v = (hi + lo * (1.0 / kFix2Lo)) * (1.0 / kFix2Hi);
    fo[q] = accumulate ? fo[q] + v : v;
  }
}

// ---------------------------------------------------------------------------
// FP64 derivative kernel of the cutoff LJ(C2) + Coulomb(C1) energy for the
// differentiable form.  Same full-shell cell walk and lane mapping as
// k_pair_fp64 (every pair is visited from both of its atoms).  Per pair, in
// the variable s = r^2 (d = x_j - x_i, minimum image):
//   U(s) = S(s) (A s^-6 - B s^-3) + f q_i q_j phi(s),
//   phi = s^-1/2 - 1.5/rc + 0.5 s/rc^3 (C1-shifted Coulomb), S the C2 switch
//   (C2SwitchingFunction.h:42-53 as a function of s), f = coulombScalingFactor
//   for modified pairs (A14/B14 then too), 1 otherwise.
// Gradient of U with respect to x_j: 2 U_s d; Hessian block
// K = 2 U_s I + 4 U_ss d d^T.
//
// DERIV_PARAMS: dq[i] = dE/dq_i = sum_j f q_j phi; per LJ table entry (a, b)
//   dE/dA = sum S s^-6, dE/dB = -sum S s^-3 (entries 2, 3: the modified
//   pairs' A14, B14), each unordered pair split half to (a, b), half to
//   (b, a) -- the derivative with respect to the table as the pair loop reads
//   it.
// DERIV_VJP: for a direction w (3n), hv = H w (hv_i = sum_j K (w_i - w_j)),
//   and the derivatives of w . grad E = sum_pairs 2 U_s d.(w_j - w_i) with
//   respect to q_i (dq) and to the table entries (tpart), as above.
// Table sums go through shared memory to one column entry per block of
// tpart ([ntypes^2 * 4][gridDim.x]); k_reduce_columns adds them up.
// ---------------------------------------------------------------------------
enum DerivMode { DERIV_PARAMS = 0, DERIV_VJP = 1 };

// One pair's terms in s = r^2: the LJ energy E = A s^-6 - B s^-3 and its
// s-derivatives, the C2 switch S and its derivatives (polynomials in s), f q_j
// and the C1-shifted Coulomb phi with its derivatives (zero beyond rc).
// Shared by the derivative kernels, so that they round every pair alike.
struct DerivTerms {
  double is, is3, is6, E, Es, Ess, S, Ss, Sss, qf, phi, phis, phiss;
};
__device__ __forceinline__ DerivTerms deriv_terms(const Fp64Consts &mc,
                                                  const double4 *__restrict__ lj64, int tab,
                                                  int kind, double s, double qj) {
  DerivTerms u;
  const double4 p = lj64[tab];
  const double A = kind == 1 ? p.z : p.x;
  const double B = kind == 1 ? p.w : p.y;
  // one reciprocal square root serves both 1/s and s^-1/2 (the Coulomb
  // terms): 1/s as its square, within 2 ulp of the quotient
  const double ir = rsqrt(s);
  u.is = ir * ir;
  u.is3 = u.is * u.is * u.is;
  u.is6 = u.is3 * u.is3;
  u.E = A * u.is6 - B * u.is3;
  u.Es = (-6.0 * A * u.is6 + 3.0 * B * u.is3) * u.is;
  u.Ess = (42.0 * A * u.is6 - 12.0 * B * u.is3) * u.is * u.is;
  u.S = 1.0; u.Ss = 0.0; u.Sss = 0.0;
  if (s > mc.rclj2) {
    u.S = 0.0;
  } else if (s >= mc.ron2) {
    const double c2 = mc.rclj2 - s;
    u.S = mc.s1 * c2 * c2 * (mc.s2 + 2.0 * s);
    u.Ss = 2.0 * mc.s1 * c2 * (c2 - mc.s2 - 2.0 * s);
    u.Sss = 2.0 * mc.s1 * (mc.s2 + 2.0 * s - 4.0 * c2);
  }
  u.qf = qj * (kind == 1 ? mc.csf : 1.0);  // f q_j
  u.phi = 0.0; u.phis = 0.0; u.phiss = 0.0;
  if (s <= mc.rcc2) {
    u.phi = ir - mc.c15_1 + mc.c05_3 * s;
    u.phis = -0.5 * ir * u.is + mc.c05_3;
    u.phiss = 0.75 * ir * u.is * u.is;
  }
  return u;
}

// kParams: also the parameter derivatives (dq, the table partials); a
// VJP launch without them computes H w alone.  In VJP mode w is read in the
// sorted order (ws[j] = w of sorted atom j, gathered by k_gather_sorted).
template <int kMode, bool kParams = true>
__global__ void __launch_bounds__(128)
k_deriv_fp64(GridParams g, Fp64Consts mc, const Stencil st, int ntypes,
             const double4 *__restrict__ lj64, const int *__restrict__ start,
             const double4 *__restrict__ spos, const int2 *__restrict__ smeta,
             const int *__restrict__ sidx, const int *__restrict__ ex_start,
             const int2 *__restrict__ ex, const double4 *__restrict__ ws, double *__restrict__ hv,
             double *__restrict__ dq, double *__restrict__ tpart) {
  extern __shared__ double s_tab[];  // ntypes^2 * 4
  const int nt4 = ntypes * ntypes * 4;
  for (int k = threadIdx.x; k < nt4; k += blockDim.x) s_tab[k] = 0.0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int cell = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (cell < g.ncell) {
    const int cx = cell % g.nx;
    const int cy = (cell / g.nx) % g.ny;
    const int cz = cell / (g.nx * g.ny);
    const int cs = start[cell], ce = start[cell + 1];
    for (int c0 = cs; c0 < ce; c0 += 32) {
      const int m = min(32, ce - c0);
      const int L = lanes_per_atom(m);
      const int ia = lane / L;
      const int sub = lane % L;
      const bool active = ia < m;
      const int i = c0 + (active ? ia : 0);
      const double4 pi = spos[i];
      const int2 mi = smeta[i];
      const int oi = sidx[i];
      const int elo = ex_start[oi], ehi = ex_start[oi + 1];
      const int ti = mi.x * ntypes;
      double wi[3] = {0.0, 0.0, 0.0};
      if (kMode == DERIV_VJP) {
        const double4 wv = ws[i];
        wi[0] = wv.x; wi[1] = wv.y; wi[2] = wv.z;
      }
      double hx = 0, hy = 0, hz = 0, gq = 0;
      // table derivatives of this lane's plain pairs, per j type, in
      // registers (with few types the block's shared sums would see every
      // lane add to the same entry); modified pairs and larger tables go to
      // the shared sums directly
      constexpr int kRegTypes = 4;
      const bool regtab = kParams && ntypes <= kRegTypes;
      double ta[kRegTypes] = {0.0, 0.0, 0.0, 0.0}, tb[kRegTypes] = {0.0, 0.0, 0.0, 0.0};
      auto table_add = [&](int tj, int kind_, int tab_, double va, double vb) {
        if (regtab && kind_ == 0) {
#pragma unroll
          for (int k = 0; k < kRegTypes; k++)
            if (k == tj) { ta[k] += va; tb[k] += vb; }
        } else {
          atomicAdd(&s_tab[tab_], va);
          atomicAdd(&s_tab[tab_ + 1], vb);
        }
      };
      for (int r = 0; r < g.nrows; r++) {
        const Row row = st.rows[r];
        int jy = cy + row.dy, jz = cz + row.dz;
        if (!g.periodic && (jy < 0 || jy >= g.ny || jz < 0 || jz >= g.nz)) continue;
        while (jy < 0) jy += g.ny;
        while (jy >= g.ny) jy -= g.ny;
        while (jz < 0) jz += g.nz;
        while (jz >= g.nz) jz -= g.nz;
        const int rowbase = (jz * g.ny + jy) * g.nx;
        for (int dx = row.dxlo; dx <= row.dxhi; dx++) {
          int jx = cx + dx;
          if (!g.periodic && (jx < 0 || jx >= g.nx)) continue;
          jx += jx < 0 ? g.nx : (jx >= g.nx ? -g.nx : 0);  // |dx| <= n / 2: one wrap
          const int jc = rowbase + jx;
          const int js = start[jc], je = start[jc + 1];
          double sx, sy, sz;  // the neighbour cell's shift (A)
          cell_shift(g, g.ec, 1.0, dx, row.dy, row.dz, sx, sy, sz);
          for (int j = js + sub; j < je; j += L) {
            const double4 pj = spos[j];
            const double ddx = (pj.x + sx) - pi.x;
            const double ddy = (pj.y + sy) - pi.y;
            const double ddz = (pj.z + sz) - pi.z;
            const double s = ddx * ddx + ddy * ddy + ddz * ddz;
            if (!(s <= mc.cut2) || !(s > 0.0) || j == i || !active) continue;
            const int2 mj = smeta[j];
            int kind = 0;
            if (mj.y == mi.y) {
              kind = excl_kind(ex, elo, ehi, sidx[j]);
              if (kind == 2) continue;
            }
            const DerivTerms u = deriv_terms(mc, lj64, ti + mj.x, kind, s, pj.w);
            const double E = u.E, Es = u.Es, Ess = u.Ess, S = u.S, Ss = u.Ss, Sss = u.Sss;
            const double is = u.is, is3 = u.is3, is6 = u.is6;
            const double qf = u.qf, phi = u.phi, phis = u.phis, phiss = u.phiss;
            const int tab = (ti + mj.x) * 4 + (kind == 1 ? 2 : 0);
            if (kMode == DERIV_PARAMS) {
              gq += qf * phi;
              table_add(mj.x, kind, tab, 0.5 * S * is6, -0.5 * S * is3);
            } else {
              const double4 wj = ws[j];
              const double dl0 = wi[0] - wj.x, dl1 = wi[1] - wj.y, dl2 = wi[2] - wj.z;
              const double dd = ddx * dl0 + ddy * dl1 + ddz * dl2;  // d . (w_i - w_j)
              const double Us = Ss * E + S * Es + pi.w * qf * phis;
              const double Uss = Sss * E + 2.0 * Ss * Es + S * Ess + pi.w * qf * phiss;
              const double a = 2.0 * Us, b = 4.0 * Uss * dd;
              hx += a * dl0 + b * ddx;
              hy += a * dl1 + b * ddy;
              hz += a * dl2 + b * ddz;
              if (kParams) {
                const double T = -2.0 * dd;  // 2 d . (w_j - w_i)
                gq += qf * phis * T;
                table_add(mj.x, kind, tab, 0.5 * T * (Ss * is6 - 6.0 * S * is6 * is),
                          0.5 * T * (-Ss * is3 + 3.0 * S * is3 * is));
              }
            }
          }
        }
      }
      for (int off = 1; off < L; off <<= 1) {
        gq += __shfl_xor_sync(0xffffffffu, gq, off);
        if (kMode == DERIV_VJP) {
          hx += __shfl_xor_sync(0xffffffffu, hx, off);
          hy += __shfl_xor_sync(0xffffffffu, hy, off);
          hz += __shfl_xor_sync(0xffffffffu, hz, off);
        }
      }
      if (regtab && active) {  // the lane's register sums into the block's table
        for (int k = 0; k < ntypes; k++) {
          if (ta[k] != 0.0) atomicAdd(&s_tab[(ti + k) * 4], ta[k]);
          if (tb[k] != 0.0) atomicAdd(&s_tab[(ti + k) * 4 + 1], tb[k]);
        }
      }
      if (active && sub == 0) {
        if (kParams) dq[oi] = gq;
        if (kMode == DERIV_VJP) {
          hv[3 * (size_t)oi] = hx;
          hv[3 * (size_t)oi + 1] = hy;
          hv[3 * (size_t)oi + 2] = hz;
        }
      }
    }
  }
  if (kParams) {
    __syncthreads();
    for (int k = threadIdx.x; k < nt4; k += blockDim.x)
      tpart[(size_t)k * gridDim.x + blockIdx.x] = s_tab[k];
  }
}

// ---------------------------------------------------------------------------
// The derivative kernel on the half shell: k_pair_fp64_half's task split --
// one warp per block, `slots` warps per i-cell, each a share of the
// half-shell cell offsets (home-cell pairs i < j) -- its staging (j atoms in
// the i-cell frame, kB64 at a time, with their direction in DERIV_VJP mode;
// those farther than the cutoff from the box around the chunk's i atoms left
// out) and its conflict-free block rotation, with deriv_terms' per-pair
// arithmetic.  Each pair is evaluated once and its terms go to both atoms:
// DERIV_VJP: K (w_i - w_j), K = 2 U_s I + 4 U_ss d d^T, to hv_i and, K being
//   even in d = x_j - x_i, its negative to hv_j;
// kParams: c = f phi (DERIV_PARAMS) or f phi_s T, T = 2 d.(w_j - w_i) (even
//   in d too): q_j c to dq_i and q_i c to dq_j; the table terms (halved) to
//   the entries (a, b) and (b, a) of the pair's types -- the terms of
//   k_deriv_fp64's two visits of the pair.
// hv and dq reach acc (sorted order, cleared by the cell build: words
// {hi x, hi y, hi z, lo x, lo y, lo z} of hv, then {hi, lo} of dq) as the
// exact two-word fixed point of fix2_add, so they do not depend on the order
// of the sums; k_finalize64 and k_finalize_q write them in the caller's order.
// Table sums (kParams; at most kDerivRegTypes types, summed per lane in
// registers by j type, modified pairs in shared memory) leave one column
// entry per block: tpart[entry][block], added up by k_reduce_columns.
// ---------------------------------------------------------------------------
constexpr int kDerivRegTypes = 4;
constexpr int kDerivTab = kDerivRegTypes * kDerivRegTypes * 4;
struct DerivWarpSmem {
  double4 pos[kB64];    // staged j: position in the i-cell frame (A), charge
  double4 w[kB64];      // its direction (w.w unused; DERIV_VJP)
  int2 meta[kB64];      // type, molecule
  int jidx[kB64];       // sorted index; bit 31: an atom of the home cell
  double jh[3][kB64];   // the batch's hv_j sums
  double jq[kB64];      // the batch's dq_j sums
  double tab[kDerivTab];  // the block's table sums
};

// v into the two-word fixed-point words rhi, rlo of atom j (fix2_add's split)
__device__ __forceinline__ void fix2_add_rows(unsigned long long *__restrict__ acc, size_t n,
                                              size_t j, int rhi, int rlo, double v,
                                              int *__restrict__ err) {
  if (!(fabs(v) < kFix2Max)) {
    atomicOr(err, 2);
    return;
  }
  const double s = v * kFix2Hi;
  const double h = rint(s);
  const long long hi = (long long)h;
  const long long lo = __double2ll_rn((s - h) * kFix2Lo);
  if (hi) atomicAdd(&acc[(size_t)rhi * n + j], (unsigned long long)hi);
  if (lo) atomicAdd(&acc[(size_t)rlo * n + j], (unsigned long long)lo);
}

#ifndef PMB200_HVP_BLOCKS
// resident blocks per SM asked of the Hessian-vector product kernel
// (measured on the 41k water box: 12, 16, 20, 24 blocks 0.468, 0.473, 0.455,
// 0.446 ms per product)
#define PMB200_HVP_BLOCKS 24
#endif
#ifndef PMB200_DERIV_PARAM_BLOCKS
// the same with parameter derivatives (41k box, 16 / 20 / 24 blocks: dE/dparams
// 0.478 / 0.430 / 0.431 ms, a product with them 0.634 / 0.622 / 0.754 ms)
#define PMB200_DERIV_PARAM_BLOCKS 20
#endif
template <int kMode, bool kParams>
__global__ void __launch_bounds__(32, kParams ? PMB200_DERIV_PARAM_BLOCKS : PMB200_HVP_BLOCKS)
k_deriv_fp64_half(GridParams g, Fp64Consts mc, const HalfStencil st, int slots, int ntypes,
                  const double4 *__restrict__ lj64, const int *__restrict__ start,
                  const double4 *__restrict__ spos, const int2 *__restrict__ smeta,
                  const int *__restrict__ sidx, const int *__restrict__ ex_start,
                  const int2 *__restrict__ ex, const double4 *__restrict__ ws,
                  unsigned long long *__restrict__ acc, int n, double *__restrict__ tpart,
                  int *__restrict__ err) {
  constexpr bool kVjp = kMode == DERIV_VJP;
  __shared__ DerivWarpSmem sm;
  const int lane = threadIdx.x;
  const int cell = (int)(blockIdx.x / slots), slot = (int)(blockIdx.x % slots);
  if (cell >= g.ncell) return;  // uniform per block
  const int cx = cell % g.nx;
  const int cy = (cell / g.nx) % g.ny;
  const int cz = cell / (g.nx * g.ny);
  const int cs = start[cell], ce = start[cell + 1];
  for (int t = lane; t < kB64; t += 32) {
    sm.jh[0][t] = sm.jh[1][t] = sm.jh[2][t] = 0.0;
    sm.jq[t] = 0.0;
  }
  if (kParams)
    for (int t = lane; t < kDerivTab; t += 32) sm.tab[t] = 0.0;
  for (int c0 = cs; c0 < ce; c0 += 32) {
    const int m = min(32, ce - c0);
    const int L = lanes_per_atom(m);
    const int ia = lane / L;
    const int sub = lane % L;
    const bool active = ia < m;
    const int i = c0 + (active ? ia : 0);
    const double4 pi = spos[i];
    const double4 wi = kVjp ? ws[i] : make_double4(0.0, 0.0, 0.0, 0.0);
    const int2 mi = smeta[i];
    const int oi = sidx[i];
    const int elo = ex_start[oi], ehi = ex_start[oi + 1];
    const int ti = mi.x * ntypes;
    double hx = 0, hy = 0, hz = 0, gq = 0;
    // the lane's plain pairs' table terms by j type
    double ta[kDerivRegTypes] = {0.0, 0.0, 0.0, 0.0}, tb[kDerivRegTypes] = {0.0, 0.0, 0.0, 0.0};
    // the box around the chunk's i atoms
    double blo_x = pi.x, blo_y = pi.y, blo_z = pi.z, bhi_x = pi.x, bhi_y = pi.y, bhi_z = pi.z;
    for (int off = 16; off > 0; off >>= 1) {
      blo_x = fmin(blo_x, __shfl_xor_sync(0xffffffffu, blo_x, off));
      blo_y = fmin(blo_y, __shfl_xor_sync(0xffffffffu, blo_y, off));
      blo_z = fmin(blo_z, __shfl_xor_sync(0xffffffffu, blo_z, off));
      bhi_x = fmax(bhi_x, __shfl_xor_sync(0xffffffffu, bhi_x, off));
      bhi_y = fmax(bhi_y, __shfl_xor_sync(0xffffffffu, bhi_y, off));
      bhi_z = fmax(bhi_z, __shfl_xor_sync(0xffffffffu, bhi_z, off));
    }
    int nb = 0;
    // every i atom of the chunk against the nb staged atoms (atom ia's lanes
    // take block (ia + k) mod nsteps at step k: no two lanes meet one staged
    // atom in a step), then the j sums out and the batch emptied
    auto process = [&]() {
      __syncwarp();
      const int nblk = (nb + L - 1) / L;
      const int nsteps = max(nblk, m);
      for (int k = 0; k < nsteps; k++) {
        int blk = ia + k;
        if (blk >= nsteps) blk -= nsteps;
        const int t = blk * L + sub;
        if (active && t < nb) {
          const int jw = sm.jidx[t];
          const int j = jw & 0x7fffffff;
          const double4 pj = sm.pos[t];
          const double ddx = pj.x - pi.x;
          const double ddy = pj.y - pi.y;
          const double ddz = pj.z - pi.z;
          const double s = ddx * ddx + ddy * ddy + ddz * ddz;
          const int2 mj = sm.meta[t];
          int kind = (jw < 0 && j <= i) ? 2 : 0;  // home cell: pairs i < j only
          const bool near = s <= mc.cut2 && s > 0.0;
          if (kind == 0 && near && mj.y == mi.y) kind = excl_kind(ex, elo, ehi, sidx[j]);
          if (kind != 2 && near) {
            const DerivTerms u = deriv_terms(mc, lj64, ti + mj.x, kind, s, pj.w);
            double T = 0.0;
            if (kVjp) {
              const double4 wj = sm.w[t];
              const double dl0 = wi.x - wj.x, dl1 = wi.y - wj.y, dl2 = wi.z - wj.z;
              const double dd = ddx * dl0 + ddy * dl1 + ddz * dl2;  // d . (w_i - w_j)
              const double Us = u.Ss * u.E + u.S * u.Es + pi.w * u.qf * u.phis;
              const double Uss =
                  u.Sss * u.E + 2.0 * u.Ss * u.Es + u.S * u.Ess + pi.w * u.qf * u.phiss;
              const double a = 2.0 * Us, b = 4.0 * Uss * dd;
              const double vx = a * dl0 + b * ddx, vy = a * dl1 + b * ddy,
                           vz = a * dl2 + b * ddz;
              hx += vx; hy += vy; hz += vz;
              sm.jh[0][t] -= vx;
              sm.jh[1][t] -= vy;
              sm.jh[2][t] -= vz;
              T = -2.0 * dd;
            }
            if (kParams) {
              const double c = kVjp ? u.phis * T : u.phi;
              gq += u.qf * c;                                      // f q_j c
              sm.jq[t] += pi.w * (kind == 1 ? mc.csf : 1.0) * c;  // f q_i c
              double va, vb;
              if (kVjp) {
                va = 0.5 * T * (u.Ss * u.is6 - 6.0 * u.S * u.is6 * u.is);
                vb = 0.5 * T * (-u.Ss * u.is3 + 3.0 * u.S * u.is3 * u.is);
              } else {
                va = 0.5 * u.S * u.is6;
                vb = -0.5 * u.S * u.is3;
              }
              if (kind == 0) {
#pragma unroll
                for (int q = 0; q < kDerivRegTypes; q++)
                  if (q == mj.x) { ta[q] += va; tb[q] += vb; }
              } else {  // a modified pair: entries 2, 3 of both orders
                const int e1 = (ti + mj.x) * 4 + 2, e2 = (mj.x * ntypes + mi.x) * 4 + 2;
                atomicAdd(&sm.tab[e1], va);
                atomicAdd(&sm.tab[e1 + 1], vb);
                atomicAdd(&sm.tab[e2], va);
                atomicAdd(&sm.tab[e2 + 1], vb);
              }
            }
          }
        }
        __syncwarp();
      }
      for (int t = lane; t < nb; t += 32) {
        const size_t j = (size_t)(sm.jidx[t] & 0x7fffffff);
        if (kVjp) {
#pragma unroll
          for (int qq = 0; qq < 3; qq++) {
            const double v = sm.jh[qq][t];
            if (v != 0.0) fix2_add_rows(acc, (size_t)n, j, qq, 3 + qq, v, err);
            sm.jh[qq][t] = 0.0;
          }
        }
        if (kParams) {
          const double v = sm.jq[t];
          if (v != 0.0) fix2_add_rows(acc, (size_t)n, j, 6, 7, v, err);
          sm.jq[t] = 0.0;
        }
      }
      nb = 0;
      __syncwarp();
    };
    for (int q = slot; q < st.ncells; q += slots) {
      const unsigned o = st.off[q];
      const int dx = (int)(o & 31u) - 8, dy = (int)((o >> 5) & 31u) - 8,
                dz = (int)((o >> 10) & 31u) - 8;
      const int homebit = (dx | dy | dz) == 0 ? (int)0x80000000u : 0;
      int jx = cx + dx, jy = cy + dy, jz = cz + dz;
      if (g.periodic) {
        // one wrap suffices: offsets reach at most ceil(rc / edge) <= n / 2
        jx += jx < 0 ? g.nx : (jx >= g.nx ? -g.nx : 0);
        jy += jy < 0 ? g.ny : (jy >= g.ny ? -g.ny : 0);
        jz += jz < 0 ? g.nz : (jz >= g.nz ? -g.nz : 0);
      } else if (jx < 0 || jx >= g.nx || jy < 0 || jy >= g.ny || jz < 0 || jz >= g.nz) {
        continue;  // uniform per warp
      }
      const int jc = (jz * g.ny + jy) * g.nx + jx;
      const int js = start[jc], cnt = start[jc + 1] - js;
      double sx, sy, sz;  // the neighbour cell's shift (A)
      cell_shift(g, g.ec, 1.0, dx, dy, dz, sx, sy, sz);
      for (int f0 = 0; f0 < cnt;) {
        const int take = min(min(cnt - f0, kB64 - nb), 32);
        bool keep = false;
        double4 p = make_double4(0.0, 0.0, 0.0, 0.0);
        const int j = js + f0 + lane;
        if (lane < take) {
          p = spos[j];
          p.x += sx; p.y += sy; p.z += sz;
          // squared distance to the box (no pair the test accepts is dropped:
          // per axis at most |p - x_i| for every i of the chunk)
          const double bx = fmax(fmax(blo_x - p.x, p.x - bhi_x), 0.0);
          const double by = fmax(fmax(blo_y - p.y, p.y - bhi_y), 0.0);
          const double bz = fmax(fmax(blo_z - p.z, p.z - bhi_z), 0.0);
          keep = bx * bx + by * by + bz * bz <= mc.cut2;
        }
        const unsigned km = __ballot_sync(0xffffffffu, keep);
        if (keep) {
          const int slot_ = nb + __popc(km & ((1u << lane) - 1u));
          sm.pos[slot_] = p;
          if (kVjp) sm.w[slot_] = ws[j];
          sm.meta[slot_] = smeta[j];
          sm.jidx[slot_] = j | homebit;
        }
        nb += __popc(km);
        f0 += take;
        if (nb > kB64 - 32) process();  // less than a full round of room left
      }
    }
    if (nb > 0) process();
    for (int off = 1; off < L; off <<= 1) {
      if (kVjp) {
        hx += __shfl_xor_sync(0xffffffffu, hx, off);
        hy += __shfl_xor_sync(0xffffffffu, hy, off);
        hz += __shfl_xor_sync(0xffffffffu, hz, off);
      }
      if (kParams) gq += __shfl_xor_sync(0xffffffffu, gq, off);
    }
    if (active && sub == 0) {
      if (kVjp) {
        fix2_add_rows(acc, (size_t)n, (size_t)i, 0, 3, hx, err);
        fix2_add_rows(acc, (size_t)n, (size_t)i, 1, 4, hy, err);
        fix2_add_rows(acc, (size_t)n, (size_t)i, 2, 5, hz, err);
      }
      if (kParams) fix2_add_rows(acc, (size_t)n, (size_t)i, 6, 7, gq, err);
    }
    if (kParams && active) {  // the lane's register sums, to both orders
#pragma unroll
      for (int q = 0; q < kDerivRegTypes; q++) {
        if (q >= ntypes) break;
        if (ta[q] != 0.0) {
          atomicAdd(&sm.tab[(ti + q) * 4], ta[q]);
          atomicAdd(&sm.tab[(q * ntypes + mi.x) * 4], ta[q]);
        }
        if (tb[q] != 0.0) {
          atomicAdd(&sm.tab[(ti + q) * 4 + 1], tb[q]);
          atomicAdd(&sm.tab[(q * ntypes + mi.x) * 4 + 1], tb[q]);
        }
      }
    }
  }
  if (kParams) {
    __syncwarp();
    const int nt4 = ntypes * ntypes * 4;
    for (int k = lane; k < nt4; k += 32) tpart[(size_t)k * gridDim.x + blockIdx.x] = sm.tab[k];
  }
}

// dq from the derivative accumulator's words {hi, lo} (rows 6, 7), in the
// caller's atom order.
__global__ void k_finalize_q(int n, const unsigned long long *__restrict__ acc,
                             const int *__restrict__ sidx, double *__restrict__ dq) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const double hi = (double)(long long)acc[6 * (size_t)n + j];
  const double lo = (double)(long long)acc[7 * (size_t)n + j];
  dq[sidx[j]] = (hi + lo * (1.0 / kFix2Lo)) * (1.0 / kFix2Hi);
}

// ws[j] = w[3 sidx[j] ..] for the sorted atoms j (the direction of a
// Hessian-vector product, read per pair in cell order).
__global__ void k_gather_sorted(int n, const int *__restrict__ sidx, const double *__restrict__ w,
                                double4 *__restrict__ ws) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const size_t o = 3 * (size_t)sidx[j];
  ws[j] = make_double4(w[o], w[o + 1], w[o + 2], 0.0);
}

// out[k] = sum over rows r of part[r][k], rows added in order (deterministic).
__global__ void k_reduce_columns(int rows, int cols, const double *__restrict__ part,
                                 double *__restrict__ out) {
  // one block per column (part[col][row]): strided per-thread sums, then a
  // fixed tree, so the order of the additions is the same every launch
  __shared__ double red[256];
  const int k = blockIdx.x;
  if (k >= cols) return;
  const double *col = part + (size_t)k * rows;
  double acc = 0.0;
  for (int r = threadIdx.x; r < rows; r += blockDim.x) acc += col[r];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[k] = red[0];
}

// ---------------------------------------------------------------------------
// Molecular virial support: molecule centres of mass from the raw positions
// (mass-weighted, Kahan-compensated like molecularCenterOfMass,
// protomol/src/protomol/topology/TopologyUtilities.cpp:645-672).
// ---------------------------------------------------------------------------
__global__ void k_com(int nmol, const int *__restrict__ mstart, const int *__restrict__ matoms,
                      const double *__restrict__ mass, const double *__restrict__ pos,
                      double *__restrict__ com) {
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nmol) return;
  const int lo = mstart[m], hi = mstart[m + 1];
  if (lo == hi) { com[3 * m] = com[3 * m + 1] = com[3 * m + 2] = 0.0; return; }
  int a = matoms[lo];
  double w = mass[a], sw = w;
  double c[3], e[3] = {0, 0, 0};
  for (int k = 0; k < 3; k++) c[k] = pos[3 * a + k] * w;
  for (int t = lo + 1; t < hi; t++) {
    a = matoms[t];
    w = mass[a];
    sw += w;
    for (int k = 0; k < 3; k++) {
      const double x = pos[3 * a + k] * w;
      const double y = x - e[k];
      const double tt = c[k] + y;
      e[k] = (tt - c[k]) - y;
      c[k] = tt;
    }
  }
  for (int k = 0; k < 3; k++) com[3 * m + k] = c[k] / sw;
}

// Deterministic two-stage reduction of the per-cell partials.  Stage 1:
// block b sums cells [b*span, (b+1)*span) in a fixed tree order into
// red[b][ACC_MV]; stage 2 (one block) sums the blocks in order and forms
// out[20] = {COULOMB, LENNARDJONES, virial[9], molvirial[9]} and the unique
// pair count.  mixed != 0: the Coulomb energy comes from the three-sum form
// with the C1 constants (cell units) applied here in FP64.
constexpr int kRedBlocks = 64;

// k_reduce1's work for block b of kRedBlocks (256 threads): the first ns
// slots of rows [b * span, (b + 1) * span) summed, written to red[b][.]
__device__ __forceinline__ void reduce1_block(int b, int nrows, const double *__restrict__ partial,
                                              double *__restrict__ red, int ns,
                                              double (*sh)[ACC_MV]) {
  // each thread sums its rows' first ns slots; warp shuffles, then the
  // block's warps in order (fixed order: deterministic)
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int span = (nrows + kRedBlocks - 1) / kRedBlocks;
  const int lo = b * span, hi = min(nrows, lo + span);
  double v[ACC_MV];
#pragma unroll
  for (int k = 0; k < ACC_MV; k++) v[k] = 0.0;
  for (int c = lo + t; c < hi; c += blockDim.x)
#pragma unroll
    for (int k = 0; k < ACC_MV; k++)
      if (k < ns) v[k] += partial[(size_t)c * kNacc + k];
#pragma unroll
  for (int k = 0; k < ACC_MV; k++)
    if (k < ns) {
      const double s = warp_sum_mask(v[k], 32);
      if (lane == 0) sh[w][k] = s;
    }
  __syncthreads();
  if (t < ns) {
    double acc = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) acc += sh[q][t];
    red[b * ACC_MV + t] = acc;
  }
}

// k_reduce2's work (one block): the kRedBlocks block totals summed and the
// results written (red read through L2: written by other blocks of the same
// launch in k_finalize_reduce).
__device__ __forceinline__ void reduce2_block(int nred, const double *red, double visit,
                                              double *__restrict__ out,
                                              double *__restrict__ pairs_out, int ns,
                                              double *col) {
  // each of the first ns slots summed over the blocks in block order by one
  // warp (fixed order: deterministic); slots beyond ns are zero
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int k = w; k < ACC_MV; k += (int)(blockDim.x >> 5)) {
    double acc = 0.0;
    if (k < ns)
      for (int b = lane; b < nred; b += 32) acc += __ldcg(red + b * ACC_MV + k);
    acc = warp_sum_mask(acc, 32);
    if (lane == 0) col[k] = acc;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  double r[ACC_MV];
  for (int k = 0; k < ACC_MV; k++) r[k] = col[k];
  // visit = 1 / (times each pair was evaluated)
  out[0] = visit * r[ACC_ECOUL];
  out[1] = visit * r[ACC_ELJ];
  // symmetric atomic virial from xx xy xz yy yz zz
  // Both tables hold xx xy xz yy yz zz.  The reference stores the molecular
  // virial symmetrised from the upper triangle too (ScalarStructure::
  // addVirial(f, diff, comDiff) adds f_x c_y to both XY and YX,
  // protomol/src/protomol/type/ScalarStructure.cpp:77-110).
  const int map[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
  for (int k = 0; k < 9; k++) {
    out[2 + k] = visit * r[ACC_W + map[k]];
    out[11 + k] = visit * r[ACC_MW + map[k]];
  }
  if (pairs_out) *pairs_out = visit * r[ACC_PAIRS];
}

// Launched with kRedBlocks blocks of 256 threads.
__global__ void k_reduce1(int nrows, const double *__restrict__ partial,
                          double *__restrict__ red, int ns) {
  __shared__ double sh[8][ACC_MV];
  reduce1_block(blockIdx.x, nrows, partial, red, ns, sh);
}

// One block of 256 threads; nred = kRedBlocks.
__global__ void k_reduce2(int nred, const double *__restrict__ red, double visit,
                          double *__restrict__ out, double *__restrict__ pairs_out, int ns) {
  __shared__ double col[ACC_MV];
  reduce2_block(nred, red, visit, out, pairs_out, ns, col);
}

// k_finalize, k_reduce1 and k_reduce2 of one evaluation in one launch (the
// energy and virial evaluations of the mixed kernels): every block finalizes
// its 256 atoms; blocks 0 .. kRedBlocks - 1 also do k_reduce1's work for
// their index, and the last of them to finish (an arrival counter that
// atomicInc wraps back to zero for the next launch) does k_reduce2's -- the
// same sums in the same order, so the results equal those of the three
// kernels bit for bit, without two launches and their gaps.  Launch:
// max(ceil(n / 256), kRedBlocks) blocks of 256 threads.
// f32 (host-buffer calls of mixed contexts, or null): the forces are written
// there in FP32 (the FP64 values rounded once) instead of to `forces`, and
// the 20 result words and the device error flag `err` to `tail` after them,
// for one copy back to the host.
__global__ void __launch_bounds__(256)
k_finalize_reduce(int n, const unsigned long long *__restrict__ facc,
                  const int *__restrict__ sidx, double scale, int accumulate,
                  double *__restrict__ forces, int nrows, const double *__restrict__ partial,
                  double *red, unsigned *__restrict__ arrivals, double visit,
                  double *__restrict__ out, double *__restrict__ pairs_out, int ns,
                  float *__restrict__ f32, double *__restrict__ tail, const int *err) {
  pdl_wait();
  __shared__ double sh[8][ACC_MV];
  __shared__ double col[ACC_MV];
  __shared__ unsigned s_arrived;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) {
    const int o = sidx[j];
    if (f32) {
#pragma unroll
      for (int q = 0; q < 3; q++)
        f32[3 * (size_t)o + q] = (float)((double)(long long)facc[(size_t)q * n + j] * scale);
    } else {
      double *fo = forces + 3 * (size_t)o;
#pragma unroll
      for (int q = 0; q < 3; q++) {
        const double v = (double)(long long)facc[(size_t)q * n + j] * scale;
        fo[q] = accumulate ? fo[q] + v : v;
      }
    }
  }
  if (blockIdx.x >= kRedBlocks) return;  // uniform per block
  reduce1_block(blockIdx.x, nrows, partial, red, ns, sh);
  // this block's totals visible device-wide before its arrival is counted
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_arrived = atomicInc(arrivals, kRedBlocks - 1);
  __syncthreads();
  if (s_arrived != kRedBlocks - 1) return;  // uniform per block
  __threadfence();
  reduce2_block(kRedBlocks, red, visit, out, pairs_out, ns, col);
  if (tail && threadIdx.x == 0) {  // (out was written by this thread)
    for (int k = 0; k < 20; k++) tail[k] = out[k];
    *reinterpret_cast<int *>(tail + 20) = *(const volatile int *)err;
  }
}

// Leapfrog kick + drift (LeapfrogIntegrator::doKickdoDrift without modifiers,
// protomol/src/protomol/integrator/leapfrog/LeapfrogIntegrator.cpp:72-85):
// v += F * kick / m; x += v * h.  drift == 0 gives a kick only.
__global__ void k_kick_drift(int n, double *__restrict__ pos, double *__restrict__ vel,
                             const double *__restrict__ frc, const double *__restrict__ mass,
                             double kick, double h, int drift) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * n) return;
  const int i = t / 3;
  double v = vel[t] + frc[t] * kick / mass[i];
  vel[t] = v;
  if (drift) pos[t] += v * h;
}

// ---------------------------------------------------------------------------
// Rigid water: SETTLE (Miyamoto & Kollman, J. Comput. Chem. 13, 952 (1992)),
// the analytic constraint of a 3-site water, in FP64.  Canonical triangle
// about the centre of mass: O (0, ra, 0), H1 (-rc, -rb, 0), H2 (rc, -rb, 0);
// the new orientation is solved in the frame whose z axis is normal to the
// old molecular plane.
// ---------------------------------------------------------------------------
struct SettleParams {
  double mo, mh, ra, rb, rc;
};

__device__ __forceinline__ void d_cross(const double a[3], const double b[3], double o[3]) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
__device__ __forceinline__ double d_dot(const double a[3], const double b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
__device__ __forceinline__ void d_unit(double a[3]) {
  const double r = sqrt(d_dot(a, a));
  a[0] /= r; a[1] /= r; a[2] /= r;
}

// old: A0 B0 C0 (constrained); in/out: A1 B1 C1 (unconstrained -> constrained)
__device__ void settle_water(const SettleParams &sp, const double *A0, const double *B0,
                             const double *C0, double *A1, double *B1, double *C1) {
  const double M = sp.mo + 2.0 * sp.mh;
  double com[3], a1[3], b1[3], c1[3], b0[3], c0[3], ex[3], ey[3], ez[3];
  for (int k = 0; k < 3; k++) {
    com[k] = (sp.mo * A1[k] + sp.mh * B1[k] + sp.mh * C1[k]) / M;
    a1[k] = A1[k] - com[k];
    b1[k] = B1[k] - com[k];
    c1[k] = C1[k] - com[k];
    b0[k] = B0[k] - A0[k];
    c0[k] = C0[k] - A0[k];
  }
  d_cross(b0, c0, ez);
  d_cross(a1, ez, ex);
  d_cross(ez, ex, ey);
  d_unit(ex); d_unit(ey); d_unit(ez);
  const double xb0 = d_dot(ex, b0), yb0 = d_dot(ey, b0);
  const double xc0 = d_dot(ex, c0), yc0 = d_dot(ey, c0);
  const double za1 = d_dot(ez, a1);
  const double xb1 = d_dot(ex, b1), yb1 = d_dot(ey, b1), zb1 = d_dot(ez, b1);
  const double xc1 = d_dot(ex, c1), yc1 = d_dot(ey, c1), zc1 = d_dot(ez, c1);
  const double sphi = za1 / sp.ra, cphi = sqrt(1.0 - sphi * sphi);
  const double spsi = (zb1 - zc1) / (2.0 * sp.rc * cphi), cpsi = sqrt(1.0 - spsi * spsi);
  const double ya2 = sp.ra * cphi, xb2 = -sp.rc * cpsi;
  const double t1 = -sp.rb * cphi, t2 = sp.rc * spsi * sphi;
  const double yb2 = t1 - t2, yc2 = t1 + t2;
  const double al = xb2 * (xb0 - xc0) + yb0 * yb2 + yc0 * yc2;
  const double be = xb2 * (yc0 - yb0) + xb0 * yb2 + xc0 * yc2;
  const double ga = xb0 * yb1 - xb1 * yb0 + xc0 * yc1 - xc1 * yc0;
  const double ab = al * al + be * be;
  const double sth = (al * ga - be * sqrt(ab - ga * ga)) / ab, cth = sqrt(1.0 - sth * sth);
  const double xa3 = -ya2 * sth, ya3 = ya2 * cth, za3 = za1;
  const double xb3 = xb2 * cth - yb2 * sth, yb3 = xb2 * sth + yb2 * cth, zb3 = zb1;
  const double xc3 = -xb2 * cth - yc2 * sth, yc3 = -xb2 * sth + yc2 * cth, zc3 = zc1;
  for (int k = 0; k < 3; k++) {
    A1[k] = com[k] + xa3 * ex[k] + ya3 * ey[k] + za3 * ez[k];
    B1[k] = com[k] + xb3 * ex[k] + yb3 * ey[k] + zb3 * ez[k];
    C1[k] = com[k] + xc3 * ex[k] + yc3 * ey[k] + zc3 * ez[k];
  }
}

// Kick + drift with rigid waters: unit u < nwater is a water (one thread:
// kick, drift, SETTLE, v = (x_new - x_old) / h); the rest are free atoms.
__global__ void k_kick_drift_settle(int nwater, const int *__restrict__ widx, int nfree,
                                    const int *__restrict__ fidx, double *__restrict__ pos,
                                    double *__restrict__ vel, const double *__restrict__ frc,
                                    const double *__restrict__ mass, double kick, double h,
                                    SettleParams sp) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u < nwater) {
    int at[3] = {widx[3 * u], widx[3 * u + 1], widx[3 * u + 2]};
    double x0[3][3], x1[3][3];
    for (int a = 0; a < 3; a++) {
      const int i = at[a];
      for (int k = 0; k < 3; k++) {
        const double x = pos[3 * i + k];
        const double v = vel[3 * i + k] + frc[3 * i + k] * kick / mass[i];
        x0[a][k] = x;
        x1[a][k] = x + v * h;
      }
    }
    settle_water(sp, x0[0], x0[1], x0[2], x1[0], x1[1], x1[2]);
    for (int a = 0; a < 3; a++) {
      const int i = at[a];
      for (int k = 0; k < 3; k++) {
        pos[3 * i + k] = x1[a][k];
        vel[3 * i + k] = (x1[a][k] - x0[a][k]) / h;
      }
    }
  } else if (u < nwater + nfree) {
    const int i = fidx[u - nwater];
    for (int k = 0; k < 3; k++) {
      const double v = vel[3 * i + k] + frc[3 * i + k] * kick / mass[i];
      vel[3 * i + k] = v;
      pos[3 * i + k] += v * h;
    }
  }
}

// FP32 FMA throughput probe: 8 independent FMA chains per thread.
__global__ void k_fma_peak(int iters, float seed, float *__restrict__ sink) {
  float a0 = seed + threadIdx.x, a1 = a0 + 1.f, a2 = a0 + 2.f, a3 = a0 + 3.f;
  float a4 = a0 + 4.f, a5 = a0 + 5.f, a6 = a0 + 6.f, a7 = a0 + 7.f;
  const float m = 0.999999f, b = 1e-7f;
  for (int k = 0; k < iters; k++) {
#pragma unroll
    for (int u = 0; u < 16; u++) {
      a0 = fmaf(a0, m, b); a1 = fmaf(a1, m, b); a2 = fmaf(a2, m, b); a3 = fmaf(a3, m, b);
      a4 = fmaf(a4, m, b); a5 = fmaf(a5, m, b); a6 = fmaf(a6, m, b); a7 = fmaf(a7, m, b);
    }
  }
  const float r = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (r == 12345.678f) sink[threadIdx.x] = r;
}

}  // namespace pmb200
