// Supercluster pair kernel of the mixed cutoff form (LJ(C2) + Coulomb(C1),
// OneAtomPairTwo::doOneAtomPair, OneAtomPairTwo.h:57-125): the pair set of
// NonbondedCutoffSystemForce::evaluate (NonbondedCutoffSystemForce.h:42-53),
// evaluated as 4 x 4 atom tiles of nearby clusters.
//
// Layout, rebuilt on the device at every evaluation:
//   * the box is cut into super-columns along x and y (about the edge of a
//     cube holding 32 atoms) and each column into 1 A slabs; a counting
//     sort by (column, slab, index) orders every column's atoms by height;
//   * each column's atoms are cut, bottom to top, into superclusters of 32
//     slots (the last one padded); a supercluster's atoms are split in halves
//     by height, then by y, then by x: eight clusters of four atoms (2 x 2 x
//     2), so that clusters are compact;
//   * every atom is stored twice in FP32, as its offset in A from its
//     cluster's lattice corner (j side) and from its supercluster's lattice
//     corner (i side); the lattice step divides the box edge, so the image
//     offset between two clusters is an integer number of lattice steps,
//     applied once per list entry;
//   * per supercluster, a list of the clusters whose bounding box comes
//     within the cutoff of one of its eight clusters (each unordered cluster
//     pair once: the cluster of higher index is listed, a cluster's own pairs
//     i < j), with an 8-bit mask of the clusters it meets and, per cluster, a
//     16-bit mask of the atom pairs left after exclusions.
// The pair kernel takes a list chunk per warp; lane = 16 h + 4 a + b
// evaluates i atom a of each masked cluster against j atom b of entry e + h,
// every pair tested against the exact cutoff; j forces are summed over the
// four i lanes by shuffles and added once per entry, i forces stay in FP32
// registers for the chunk.  Every global sum is an int64 fixed-point sum
// (2^-32 kcal/mol/A): deterministic.  The Coulomb energy is q_i q_j g(r) in
// FP64 from FP64 distances (the FP32 coordinates plus their rounding
// residuals, the image offset in FP64), g the C1-switched 1/r, as in the
// search kernel; the LJ energy in FP64 from the same 1/r.
#pragma once

namespace pmb200 {

constexpr int kScAtoms = 32;      // slots per supercluster
constexpr int kScCap = 640;       // list entries per supercluster
constexpr int kScChunk = 16;      // entries per warp task
constexpr int kScMaxCols = 128;   // column offsets of the stencil
constexpr int kScTaskSups = 4096; // superclusters per round of the task kernel
constexpr float kScFar = 1.0e4f;  // pad slots' coordinate (beyond any cutoff)
constexpr float kScForceLim = 2.0e9f;  // |F| (kcal/mol/A) within the int64 2^-32 range

struct ScGrid {
  int nsx, nsy, nsz, ncol;  // super-columns along x, y; slabs along z
  int m[3];                 // lattice steps per box edge
  int nsup_max, nslot_max;
  double boxmin[3], boxlen[3];
  double colw[2], slabw;    // column widths, slab thickness (A)
  double h[3];              // lattice step boxlen / m (A)
  float hf[3];              // the same in FP32
  float L[3];               // box edges (FP32, for box tests)
  float zmax_ext;           // largest supercluster height for which the z image is unique
  float rlist2;             // squared cutoff of the box tests (with a margin)
};

struct ScStencil {          // column offsets (dx, dy) within the cutoff
  int n;
  short2 off[kScMaxCols];
};

struct __align__(16) ScEntry {
  unsigned c;       // j cluster
  unsigned imask;   // the supercluster's clusters that meet it
  unsigned shift;   // image offset j - i in lattice steps, 10 bits per axis, +512
  unsigned pad;
  unsigned ex[4];   // per i cluster k, 16 bits (a * 4 + b): pair a-b allowed
};

// A control word written by an earlier kernel of the evaluation: read once,
// coherently, where the code reads it (never moved ahead of a wait on that
// kernel).
__device__ __forceinline__ int sc_ctl(const int *p) { return *(const volatile int *)p; }

__device__ __forceinline__ void sc_wrap(const double *x, const ScGrid &g, double w[3],
                                        bool &ok) {
#pragma unroll
  for (int a = 0; a < 3; a++) {
    double v = x[a];
    if (!isfinite(v)) {
      ok = false;
      v = g.boxmin[a];
    }
    double t = v - g.boxmin[a];
    t -= g.boxlen[a] * floor(t / g.boxlen[a]);
    if (t >= g.boxlen[a]) t = 0.0;  // (a value just below a multiple of the edge)
    w[a] = t;
  }
}

// Cell of every atom in the (column, slab) grid, z fastest, and its slot
// among the cell's atoms (counting-sort keys).
__global__ void k_sc_index(int n, const double *__restrict__ pos, ScGrid g,
                           int *__restrict__ cell_of, int *__restrict__ count,
                           int *__restrict__ slot, int *__restrict__ err) {
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  bool ok = true;
  double w[3];
  sc_wrap(pos + 3 * (size_t)i, g, w, ok);
  if (!ok) atomicOr(err, 1);
  const int cx = min(max((int)(w[0] / g.colw[0]), 0), g.nsx - 1);
  const int cy = min(max((int)(w[1] / g.colw[1]), 0), g.nsy - 1);
  const int cz = min(max((int)(w[2] / g.slabw), 0), g.nsz - 1);
  const int cid = (cx * g.nsy + cy) * g.nsz + cz;
  cell_of[i] = cid;
  slot[i] = atomicAdd(&count[cid], 1);
}

// Inclusive block scan of one int per thread (warp shuffles, then the warp
// totals by the first warp); sh holds 32 ints.
__device__ __forceinline__ int sc_block_scan(int x, int *sh) {
  const int t = threadIdx.x, lane = t & 31, w = t >> 5, nw = blockDim.x >> 5;
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
  return x + (w > 0 ? sh[w - 1] : 0);
}

// Superclusters per column: supbase[col] = first supercluster of the column
// (exclusive prefix of ceil(atoms / 32)); ctl[0] = their number, ctl[1] (the
// task count) and ctl[2] (the task counter) cleared.  One block.
__global__ void k_sc_columns(int ncol, int nsz, const int *__restrict__ start,
                             int *__restrict__ supbase, int *__restrict__ ctl) {
  pdl_wait();
  pdl_trigger();  // (after the wait: see k_sc_tasks)
  __shared__ int sh[32];
  const int T = blockDim.x, t = threadIdx.x;
  const int span = (ncol + T - 1) / T;
  const int lo = t * span, hi = min(ncol, lo + span);
  int s = 0;
  for (int c = lo; c < hi; c++) s += (start[(c + 1) * nsz] - start[c * nsz] + 31) >> 5;
  const int incl = sc_block_scan(s, sh);
  int base = incl - s;
  for (int c = lo; c < hi; c++) {
    supbase[c] = base;
    base += (start[(c + 1) * nsz] - start[c * nsz] + 31) >> 5;
  }
  if (t == T - 1) {
    supbase[ncol] = incl;
    ctl[0] = incl;
    ctl[1] = 0;
    ctl[2] = 0;
  }
}

// The column of supercluster s: the last column whose first supercluster is
// not beyond s (empty columns share their successor's first index).
__device__ __forceinline__ int sc_column(const int *supbase, int ncol, int s) {
  int lo = 0, hi = ncol;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (sc_ctl(supbase + mid) <= s) lo = mid;
    else hi = mid;
  }
  return lo;
}

// One warp per supercluster: the 2 x 2 x 2 split, the slot arrays, cluster
// boxes and lattice corners, the molecule signature of each cluster, the
// supercluster's box; the slots' force accumulator cleared.
constexpr int kScBuildWarps = 4;
__global__ void __launch_bounds__(32 * kScBuildWarps)
k_sc_build(ScGrid g, const double *__restrict__ pos, const int *__restrict__ start,
           const int *__restrict__ sidx, const int2 *__restrict__ smeta,
           const int *__restrict__ supbase, const int *__restrict__ ctl,
           const double *__restrict__ q, int *__restrict__ satom, int *__restrict__ stype,
           int *__restrict__ smol, float4 *__restrict__ xi, float4 *__restrict__ xj,
           float4 *__restrict__ xilo, float4 *__restrict__ xjlo, float4 *__restrict__ clo,
           float4 *__restrict__ chi, int4 *__restrict__ corg, int2 *__restrict__ cmol,
           int4 *__restrict__ sorg, float4 *__restrict__ sbox,
           unsigned long long *__restrict__ facc, int *__restrict__ err) {
  pdl_wait();
  pdl_trigger();  // (after the wait: see k_sc_tasks)
  __shared__ double s_w[kScBuildWarps][3][32];
  __shared__ int s_at[kScBuildWarps][32];
  __shared__ int2 s_me[kScBuildWarps][32];
  const int lane = threadIdx.x & 31, wb = threadIdx.x >> 5;
  const int s = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (s >= sc_ctl(ctl)) return;  // uniform per warp
  const int col = sc_column(supbase, g.ncol, s);
  const int a0 = start[col * g.nsz] + kScAtoms * (s - supbase[col]);
  const int m = min(kScAtoms, start[(col + 1) * g.nsz] - a0);
  const bool real = lane < m;
  int atom = -1;
  int2 me = make_int2(0, -1);
  double w[3] = {0.0, 0.0, 0.0};
  if (real) {
    atom = sidx[a0 + lane];
    me = smeta[a0 + lane];
    bool ok = true;
    sc_wrap(pos + 3 * (size_t)atom, g, w, ok);
  }
  const float INF = __int_as_float(0x7f800000);
  const float ky = real ? (float)w[1] : INF, kx = real ? (float)w[0] : INF;
  // lanes 0-15 hold the lower half by height (slab order); rank by y within
  // the half, then by x within each group of eight (ties by lane)
  const int hz = lane >> 4;
  int ry = 0;
  for (int o = 0; o < 16; o++) {
    const int src = (hz << 4) + o;
    const float v = __shfl_sync(0xffffffffu, ky, src);
    ry += (v < ky) || (v == ky && src < lane);
  }
  const int grp = (hz << 1) + (ry >> 3);
  int rx = 0;
  for (int o = 0; o < 32; o++) {
    const float v = __shfl_sync(0xffffffffu, kx, o);
    const int go = __shfl_sync(0xffffffffu, grp, o);
    rx += go == grp && ((v < kx) || (v == kx && o < lane));
  }
  const int p = (grp << 3) + rx;  // slot: cluster p >> 2, atom p & 3
  s_w[wb][0][p] = w[0];
  s_w[wb][1][p] = w[1];
  s_w[wb][2][p] = w[2];
  s_at[wb][p] = atom;
  s_me[wb][p] = me;
  __syncwarp();
  // from here lane = slot
  atom = s_at[wb][lane];
  me = s_me[wb][lane];
  const bool rs = atom >= 0;
  for (int a = 0; a < 3; a++) w[a] = s_w[wb][a][lane];
  float lo[3], hi[3];
  int og[3];
  double dlo[3];
  for (int a = 0; a < 3; a++) {
    lo[a] = rs ? (float)w[a] : INF;
    hi[a] = rs ? (float)w[a] : -INF;
    dlo[a] = rs ? w[a] : 1e300;
    for (int off = 1; off < 4; off <<= 1) {
      lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], off));
      hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], off));
      dlo[a] = fmin(dlo[a], __shfl_xor_sync(0xffffffffu, dlo[a], off));
    }
    // the cluster's lattice corner: from its lowest FP64 coordinate
    og[a] = dlo[a] < 1e299 ? min((int)floor(dlo[a] / g.h[a]), g.m[a] - 1) : 0;
  }
  int os[3];
  for (int a = 0; a < 3; a++) {
    int v = dlo[a] < 1e299 ? og[a] : 0x7fffffff;
    for (int off = 4; off < 32; off <<= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, off));
    os[a] = v == 0x7fffffff ? 0 : v;
  }
  // the cluster's molecule signature: bit (molecule mod 64) of each atom
  // (two clusters can share a molecule only where their signatures meet)
  unsigned long long sig = rs ? 1ull << (me.y & 63) : 0ull;
  for (int off = 1; off < 4; off <<= 1) sig |= __shfl_xor_sync(0xffffffffu, sig, off);
  float xlo = lo[0], xhi = hi[0], ylo = lo[1], yhi = hi[1], zlo = lo[2], zhi = hi[2];
  for (int off = 4; off < 32; off <<= 1) {
    xlo = fminf(xlo, __shfl_xor_sync(0xffffffffu, xlo, off));
    xhi = fmaxf(xhi, __shfl_xor_sync(0xffffffffu, xhi, off));
    ylo = fminf(ylo, __shfl_xor_sync(0xffffffffu, ylo, off));
    yhi = fmaxf(yhi, __shfl_xor_sync(0xffffffffu, yhi, off));
    zlo = fminf(zlo, __shfl_xor_sync(0xffffffffu, zlo, off));
    zhi = fmaxf(zhi, __shfl_xor_sync(0xffffffffu, zhi, off));
  }
  const size_t sl = (size_t)s * kScAtoms + lane;
  const float qv = rs ? (float)q[atom] : 0.f;
  float4 vi, vj, li = make_float4(0.f, 0.f, 0.f, 0.f), lj = li;
  if (rs) {
    double ri[3], rj[3];
    for (int a = 0; a < 3; a++) {
      ri[a] = w[a] - os[a] * g.h[a];
      rj[a] = w[a] - og[a] * g.h[a];
    }
    vi = make_float4((float)ri[0], (float)ri[1], (float)ri[2], qv);
    vj = make_float4((float)rj[0], (float)rj[1], (float)rj[2], qv);
    li = make_float4((float)(ri[0] - (double)vi.x), (float)(ri[1] - (double)vi.y),
                     (float)(ri[2] - (double)vi.z), 0.f);
    lj = make_float4((float)(rj[0] - (double)vj.x), (float)(rj[1] - (double)vj.y),
                     (float)(rj[2] - (double)vj.z), 0.f);
  } else {
    // pads: i and j copies far apart on opposite sides, so that no pair with
    // a pad (pad-pad included) comes within a cutoff
    vi = make_float4(kScFar, kScFar, kScFar, 0.f);
    vj = make_float4(-kScFar, -kScFar, -kScFar, 0.f);
  }
  satom[sl] = atom;
  stype[sl] = rs ? me.x : 0;
  smol[sl] = me.y;
  xi[sl] = vi;
  xj[sl] = vj;
  if (xilo) {
    xilo[sl] = li;
    xjlo[sl] = lj;
  }
  const size_t nsl = (size_t)g.nslot_max;
  facc[sl] = 0;
  facc[nsl + sl] = 0;
  facc[2 * nsl + sl] = 0;
  if ((lane & 3) == 0) {
    const size_t cl = (size_t)s * 8 + (lane >> 2);
    clo[cl] = make_float4(lo[0], lo[1], lo[2], 0.f);
    chi[cl] = make_float4(hi[0], hi[1], hi[2], 0.f);
    corg[cl] = make_int4(og[0], og[1], og[2], 0);
    cmol[cl] = make_int2((int)(unsigned)sig, (int)(unsigned)(sig >> 32));
  }
  if (lane == 0) {
    sorg[s] = make_int4(os[0], os[1], os[2], 0);
    sbox[2 * (size_t)s] = make_float4(xlo, ylo, zlo, 0.f);
    sbox[2 * (size_t)s + 1] = make_float4(xhi, yhi, zhi, 0.f);
    // the z image of a listed cluster is chosen by the nearer centre: unique
    // while every supercluster is low enough
    if (zhi - zlo > g.zmax_ext) atomicOr(err, 16);
  }
}

__device__ __forceinline__ float sc_gap2(float alo, float ahi, float blo, float bhi) {
  const float d = fmaxf(0.f, fmaxf(blo - ahi, alo - bhi));
  return d * d;
}

// One block of kScListWarps warps per supercluster: its cluster list
// (entries written at s * kScCap, count in cnt[s]).  The stencil's columns
// that this supercluster lists are dealt to the warps in turn, each into its own shared-memory
// buffer; the buffers are then concatenated in warp order (a fixed order,
// so the lists, the tasks and every sum over them are the same on every
// run).  (With one warp per supercluster, the chain of dependent loads over
// all its columns took ~150 us on the 41k box.)
constexpr int kScListWarps = 4;
constexpr int kScWarpCap = 192;  // entries per warp buffer
constexpr size_t kScListSmem = sizeof(ScEntry) * kScListWarps * kScWarpCap;
__global__ void __launch_bounds__(32 * kScListWarps)
k_sc_list(ScGrid g, const ScStencil st, const int *__restrict__ supbase,
          const int *__restrict__ ctl, const float4 *__restrict__ clo,
          const float4 *__restrict__ chi, const int4 *__restrict__ corg,
          const int2 *__restrict__ cmol, const int4 *__restrict__ sorg,
          const float4 *__restrict__ sbox, const int *__restrict__ satom,
          const int *__restrict__ smol, const int *__restrict__ ex_start,
          const int2 *__restrict__ ex, ScEntry *__restrict__ ent, int *__restrict__ cnt,
          int *__restrict__ err) {
  pdl_wait();
  pdl_trigger();  // (after the wait: see k_sc_tasks)
  extern __shared__ __align__(16) unsigned char s_raw[];
  ScEntry *s_ent = reinterpret_cast<ScEntry *>(s_raw);
  __shared__ float4 s_lo[8], s_hi[8];
  __shared__ int2 s_mr[8];
  __shared__ int s_at[32], s_mo[32];
  __shared__ int s_cnt[kScListWarps];
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  const int s = blockIdx.x;
  if (s >= sc_ctl(ctl)) return;  // uniform per block
  if (threadIdx.x < 8) {
    s_lo[threadIdx.x] = clo[(size_t)s * 8 + threadIdx.x];
    s_hi[threadIdx.x] = chi[(size_t)s * 8 + threadIdx.x];
    s_mr[threadIdx.x] = cmol[(size_t)s * 8 + threadIdx.x];
  }
  if (threadIdx.x < 32) {
    s_at[threadIdx.x] = satom[(size_t)s * kScAtoms + threadIdx.x];
    s_mo[threadIdx.x] = smol[(size_t)s * kScAtoms + threadIdx.x];
  }
  __syncthreads();
  const float4 bl = sbox[2 * (size_t)s], bh = sbox[2 * (size_t)s + 1];
  const int4 os = sorg[s];
  const int col = sc_column(supbase, g.ncol, s);
  const int cx = col / g.nsy, cy = col % g.nsy;
  const float zc = 0.5f * (bl.z + bh.z);
  int count = 0;
  ScEntry *out = s_ent + wp * kScWarpCap;
  int valid = 0;  // the columns this supercluster lists, dealt to the warps in turn
  for (int q = 0; q < st.n; q++) {
    int nx = cx + st.off[q].x, ny = cy + st.off[q].y;
    int imx = 0, imy = 0;
    if (nx < 0) { nx += g.nsx; imx = -1; } else if (nx >= g.nsx) { nx -= g.nsx; imx = 1; }
    if (ny < 0) { ny += g.nsy; imy = -1; } else if (ny >= g.nsy) { ny -= g.nsy; imy = 1; }
    const int col2 = nx * g.nsy + ny;
    if (col2 < col) continue;  // that column lists the pairs with this one
    if (valid++ % kScListWarps != wp) continue;
    const float shx = imx * g.L[0], shy = imy * g.L[1];
    const int s0 = col2 == col ? s : supbase[col2], s1 = supbase[col2 + 1];
    for (int b0 = s0; b0 < s1; b0 += 32) {
      // superclusters of the column whose box comes within the cutoff of
      // this one's (z image by the nearer centre; x, y by the column offset)
      const int sj = b0 + lane;
      bool near = false;
      int imz = 0;
      if (sj < s1) {
        const float4 jl = sbox[2 * (size_t)sj], jh = sbox[2 * (size_t)sj + 1];
        imz = -(int)rintf((0.5f * (jl.z + jh.z) - zc) / g.L[2]);
        const float shz = imz * g.L[2];
        const float d2 = sc_gap2(bl.x, bh.x, jl.x + shx, jh.x + shx) +
                         sc_gap2(bl.y, bh.y, jl.y + shy, jh.y + shy) +
                         sc_gap2(bl.z, bh.z, jl.z + shz, jh.z + shz);
        near = d2 < g.rlist2;
      }
      unsigned nm = __ballot_sync(0xffffffffu, near);
      while (nm) {
        // four superclusters per pass: lane = 8 gi + k takes cluster k of the
        // gi-th remaining one
        unsigned rest = nm;
        for (int r = 0; r < (lane >> 3); r++) rest &= rest - 1u;
        const int pick = rest ? __ffs((int)rest) - 1 : -1;
        for (int r = 0; r < 4 && nm; r++) nm &= nm - 1u;
        const int izs = __shfl_sync(0xffffffffu, imz, pick >= 0 ? pick : 0);
        unsigned imask = 0;
        unsigned words[8];
#pragma unroll
        for (int k = 0; k < 8; k++) words[k] = 0xFFFFu;
        int c = -1;
        int4 oc = make_int4(0, 0, 0, 0);
        if (pick >= 0) {
          c = (b0 + pick) * 8 + (lane & 7);
          // everything the candidate needs, in one round of loads
          const float4 jl = clo[c], jh = chi[c];
          const int2 jm = cmol[c];
          oc = corg[c];
          const int4 a4 = *reinterpret_cast<const int4 *>(satom + (size_t)c * 4);
          const int4 m4 = *reinterpret_cast<const int4 *>(smol + (size_t)c * 4);
          const float shz = izs * g.L[2];
#pragma unroll
          for (int k = 0; k < 8; k++) {
            if (c < s * 8 + k) continue;
            const float4 il = s_lo[k], ih = s_hi[k];
            const float d2 = sc_gap2(il.x, ih.x, jl.x + shx, jh.x + shx) +
                             sc_gap2(il.y, ih.y, jl.y + shy, jh.y + shy) +
                             sc_gap2(il.z, ih.z, jl.z + shz, jh.z + shz);
            if (d2 < g.rlist2) imask |= 1u << k;
          }
          if (imask) {
            const int jat[4] = {a4.x, a4.y, a4.z, a4.w};
            const int jmo[4] = {m4.x, m4.y, m4.z, m4.w};
#pragma unroll
            for (int k = 0; k < 8; k++) {
              if (!((imask >> k) & 1u)) continue;
              const bool self = c == s * 8 + k;
              const int2 im = s_mr[k];
              if (!self && !((im.x & jm.x) | (im.y & jm.y))) continue;  // no common molecule
              // pairs of one molecule (pads hold molecule -1 and never match
              // a real atom's)
              unsigned same = 0;
              for (int a = 0; a < 4; a++) {
                const int mi = s_mo[k * 4 + a];
                for (int b = 0; b < 4; b++)
                  same |= (mi == jmo[b] && mi >= 0) ? 1u << (a * 4 + b) : 0u;
              }
              unsigned wd = self ? 0x08CEu /* bits a * 4 + b with b > a */ : 0xFFFFu;
              wd &= ~same;
              while (same) {  // same-molecule pairs: allowed unless excluded
                const int bit = __ffs((int)same) - 1;
                same &= same - 1u;
                if (self && (bit & 3) <= (bit >> 2)) continue;
                const int ai = s_at[k * 4 + (bit >> 2)], aj = jat[bit & 3];
                if (excl_kind(ex, ex_start[ai], ex_start[ai + 1], aj) == 0) wd |= 1u << bit;
              }
              words[k] = wd;
            }
          }
        }
        const unsigned has = __ballot_sync(0xffffffffu, imask != 0);
        if (imask) {
          const int slot = count + __popc(has & ((1u << lane) - 1u));
          if (slot < kScWarpCap) {
            const int sx = oc.x - os.x + imx * g.m[0] + 512;
            const int sy = oc.y - os.y + imy * g.m[1] + 512;
            const int sz = oc.z - os.z + izs * g.m[2] + 512;
            if (sx < 0 || sx > 1023 || sy < 0 || sy > 1023 || sz < 0 || sz > 1023)
              atomicOr(err, 32);
            ScEntry e;
            e.c = (unsigned)c;
            e.imask = imask;
            e.shift = (unsigned)(sx & 1023) | ((unsigned)(sy & 1023) << 10) |
                      ((unsigned)(sz & 1023) << 20);
            e.pad = 0;
#pragma unroll
            for (int k = 0; k < 4; k++) e.ex[k] = (words[2 * k] & 0xFFFFu) | (words[2 * k + 1] << 16);
            out[slot] = e;
          }
        }
        count += __popc(has);
      }
    }
  }
  if (lane == 0) s_cnt[wp] = count;
  __syncthreads();
  // concatenate the warps' buffers in warp order
  int base = 0, total = 0;
  bool over = false;
  for (int v = 0; v < kScListWarps; v++) {
    const int cv = s_cnt[v];
    over = over || cv > kScWarpCap;
    if (v < wp) base += min(cv, kScWarpCap);
    total += min(cv, kScWarpCap);
  }
  const int mine = min(count, kScWarpCap);
  ScEntry *dst = ent + (size_t)s * kScCap;
  for (int i = lane; i < mine; i += 32)
    if (base + i < kScCap) dst[base + i] = out[i];
  if (threadIdx.x == 0) {
    if (over || total > kScCap) atomicOr(err, 8);
    cnt[s] = min(total, kScCap);
  }
}

// Tasks (supercluster, first entry, end) of at most kScChunk entries, in
// supercluster order; ctl[1] = their number.  One block.
// Every kernel of the chain signals its dependent only once its own
// predecessor is complete: the persistent pair kernel fills every SM slot
// while it waits, and launched earlier it kept the list kernel's blocks from
// the SMs (a step then took twice as long).
__global__ void __launch_bounds__(1024)
k_sc_tasks(const int *__restrict__ cnt, int *__restrict__ ctl, int4 *__restrict__ tasks) {
  pdl_wait();
  pdl_trigger();  // (after the wait: the pair kernel's blocks may now take the SMs)
  __shared__ int sh[32];
  __shared__ int s_base[kScTaskSups + 1];
  __shared__ int s_cnt[kScTaskSups];
  const int ns = sc_ctl(ctl);
  const int T = blockDim.x, t = threadIdx.x;
  int done = 0;  // tasks of the superclusters before this round
  // rounds of kScTaskSups superclusters: their task counts scanned, then
  // the tasks written by the whole block (task i of the round found by a
  // binary search over the round's prefix)
  for (int r0 = 0; r0 < ns; r0 += kScTaskSups) {
    const int nr = min(kScTaskSups, ns - r0);
    const int per = (kScTaskSups + T - 1) / T;
    int sum = 0;
    int mine[4];
    for (int q = 0; q < per; q++) {
      const int sI = t * per + q;
      const int cv = sI < nr ? cnt[r0 + sI] : 0;
      if (sI < nr) s_cnt[sI] = cv;
      mine[q] = (cv + kScChunk - 1) / kScChunk;
      sum += mine[q];
    }
    const int incl = sc_block_scan(sum, sh);
    int b = incl - sum;
    for (int q = 0; q < per; q++) {
      const int sI = t * per + q;
      if (sI < nr) s_base[sI] = b;
      b += mine[q];
    }
    if (t == T - 1) s_base[nr] = incl;
    __syncthreads();
    const int total = s_base[nr];
    for (int i = t; i < total; i += T) {
      int lo = 0, hi = nr;  // the last supercluster whose first task is <= i
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (s_base[mid] <= i) lo = mid;
        else hi = mid;
      }
      const int sI = r0 + lo, q = i - s_base[lo];
      const int e0 = sI * kScCap, e1 = e0 + s_cnt[lo];
      const int e = e0 + q * kScChunk;
      tasks[done + i] = make_int4(sI, e, min(e1, e + kScChunk), 0);
    }
    done += total;
    __syncthreads();
  }
  if (t == 0) ctl[1] = done;
}

// Persistent pair kernel: each one-warp block takes tasks from the counter
// ctl[2] until the ctl[1] tasks are done.  LJ table (A, B in A units) from
// the FP64 copy; at most kMaxTypes types.
#ifndef PMB200_SC_BLOCKS
#define PMB200_SC_BLOCKS 24
#endif
#ifndef PMB200_SC_BLOCKS_E
#define PMB200_SC_BLOCKS_E 20
#endif
// kFull: both switches end at the pair cutoff (a pair that passes the
// cutoff test is within both), so no per-switch range selects are needed.
template <bool kEnergy, bool kFull>
__global__ void __launch_bounds__(32, kEnergy ? PMB200_SC_BLOCKS_E : PMB200_SC_BLOCKS)
k_sc_pair(MixedConsts mc, int ntypes, const double4 *__restrict__ lj64,
          const int4 *__restrict__ tasks, int *__restrict__ ctl,
          const float4 *__restrict__ xi, const float4 *__restrict__ xj,
          const int *__restrict__ stype, const ScEntry *__restrict__ ent,
          const float4 *__restrict__ xilo, const float4 *__restrict__ xjlo, ScGrid g,
          unsigned long long *__restrict__ facc, double *__restrict__ partial,
          int *__restrict__ err) {
  __shared__ float4 s_lj[kMaxTypes * kMaxTypes];
  // energy launches: A and B in FP64 (the LJ total is a small difference of
  // its repulsive and attractive sums -- 1/16 of either on water boxes -- so
  // the FP32 rounding of A and B, shared by every pair of a type pair, or a
  // bias of the FP32 1/r would not average out: the LJ energy is evaluated
  // in FP64 from the FP64 1/r the Coulomb energy uses)
  __shared__ double2 s_ljd[kEnergy ? kMaxTypes * kMaxTypes : 1];
  __shared__ float4 s_xi[32];
  __shared__ int s_row[32];
  __shared__ double s_d[3][32];
  const int lane = threadIdx.x;
  for (int k = lane; k < ntypes * ntypes; k += 32) {
    const double4 p = lj64[k];
    const float a = (float)p.x, b = (float)p.y;
    s_lj[k] = make_float4(a, b, (float)(12.0 * p.x), (float)(6.0 * p.y));
    if (kEnergy) s_ljd[k] = make_double2(p.x, p.y);
  }
  pdl_wait();
  const size_t nsl = (size_t)g.nslot_max;
  const int h = lane >> 4, ti = (lane >> 2) & 3, tj = lane & 3;
  const unsigned pbit = 1u << (ti * 4 + tj);
  const int ntask = sc_ctl(ctl + 1);
  const uint4 *e4 = reinterpret_cast<const uint4 *>(ent);
  // (a task is claimed when the previous one is done: claiming the next one
  // early, to hide the counter's latency, measured slower -- warps still busy
  // hold tasks that idle warps could take at the end)
  for (;;) {
    int task = 0;
    if (lane == 0) task = atomicAdd(&ctl[2], 1);
    task = __shfl_sync(0xffffffffu, task, 0);
    if (task >= ntask) break;
    const int4 tk = tasks[task];
    const int s = tk.x;
    __syncwarp();
    const float4 xis = xi[(size_t)s * kScAtoms + lane];
    s_xi[lane] = xis;
    s_row[lane] = stype[(size_t)s * kScAtoms + lane] * ntypes;
    if (kEnergy) {
      const float4 l = xilo[(size_t)s * kScAtoms + lane];
      s_d[0][lane] = (double)xis.x + (double)l.x;
      s_d[1][lane] = (double)xis.y + (double)l.y;
      s_d[2][lane] = (double)xis.z + (double)l.z;
    }
    __syncwarp();
    double eU = 0.0, eL = 0.0;
    int npair = 0;
    float fi[8][3];
#pragma unroll
    for (int k = 0; k < 8; k++) fi[k][0] = fi[k][1] = fi[k][2] = 0.f;
    for (int e = tk.y; e < tk.z; e += 2) {
      const int my = e + h;
      const bool valid = my < tk.z;
      uint4 a = make_uint4(0u, 0u, 0u, 0u), b = make_uint4(0u, 0u, 0u, 0u);
      if (valid) {
        a = e4[2 * (size_t)my];
        b = e4[2 * (size_t)my + 1];
      }
      const unsigned im = a.y;
      const unsigned um = im | __shfl_xor_sync(0xffffffffu, im, 16);
      const size_t js = (size_t)a.x * 4 + tj;
      float4 pj = xj[js];
      const int tjt = stype[js];
      const int kx = (int)(a.z & 1023u) - 512, ky = (int)((a.z >> 10) & 1023u) - 512,
                kz = (int)((a.z >> 20) & 1023u) - 512;
      double pdx = 0.0, pdy = 0.0, pdz = 0.0;
      if (kEnergy) {
        const float4 l = xjlo[js];
        pdx = ((double)pj.x + (double)l.x) + kx * g.h[0];
        pdy = ((double)pj.y + (double)l.y) + ky * g.h[1];
        pdz = ((double)pj.z + (double)l.z) + kz * g.h[2];
      }
      pj.x += (float)kx * g.hf[0];
      pj.y += (float)ky * g.hf[1];
      pj.z += (float)kz * g.hf[2];
      const unsigned exs[4] = {b.x, b.y, b.z, b.w};
      float fjx = 0.f, fjy = 0.f, fjz = 0.f;
#pragma unroll
      for (int k = 0; k < 8; k++) {
        if (um & (1u << k)) {  // uniform over the warp
          const float4 pi = s_xi[k * 4 + ti];
          const int row = s_row[k * 4 + ti];
          const unsigned exw = exs[k >> 1] >> ((k & 1) * 16);
          const float ddx = pj.x - pi.x, ddy = pj.y - pi.y, ddz = pj.z - pi.z;
          const float r2 = fmaf(ddx, ddx, fmaf(ddy, ddy, ddz * ddz));
          const bool ok = ((im >> k) & 1u) && (exw & pbit) && r2 <= mc.cut2;
          float rinv = rsqrtf(r2);
          rinv = fmaf(0.5f * rinv, fmaf(-r2 * rinv, rinv, 1.0f), rinv);
          const float r2inv = rinv * rinv;
          const float4 p = s_lj[row + tjt];
          const float r6 = r2inv * r2inv * r2inv;
          const float elj = fmaf(p.x, r6, -p.y) * r6;
          float flj = fmaf(p.z, r6, -p.w) * r6 * r2inv;
          float svl;
          {  // C2 switch, branch-free: value 1 below switchon, 0 beyond cutoff
            const float c2 = mc.rclj2 - r2;
            const float c4 = c2 * fmaf(2.0f, r2, mc.s2);
            const bool on = r2 >= mc.ron2;
            const bool in = kFull || r2 <= mc.rclj2;
            svl = in ? (on ? mc.s1 * (c2 * c4) : 1.0f) : 0.0f;
            const float sd = (in && on) ? mc.s3 * fmaf(c2, c2, -c4) : 0.0f;
            flj = fmaf(flj, svl, -elj * sd);
          }
          float fc;
          {  // C1 switched Coulomb, branch-free (zero beyond its cutoff):
             // E S = q q (1/r - 1.5/rc + 0.5 r^2/rc^3), so F S - E dS over r
             // is q q (1/r^3 - 1/rc^3)
            const bool inC = kFull || r2 <= mc.rcc2;
            const float qq = pi.w * pj.w;
            fc = inC ? __fmul_rn(qq, fmaf(r2inv, rinv, -2.0f * mc.c05_3)) : 0.f;
            if (kEnergy) {
              // q_i q_j g(r) from the FP64 distance (as the search kernel)
              const double ex_ = pdx - s_d[0][k * 4 + ti];
              const double ey_ = pdy - s_d[1][k * 4 + ti];
              const double ez_ = pdz - s_d[2][k * 4 + ti];
              const double r2d = fma(ex_, ex_, fma(ey_, ey_, ez_ * ez_));
              double rid = (double)rinv;
              rid = rid * fma(-0.5 * r2d, rid * rid, 1.5);
              const double gd = fma(mc.e05, r2d, rid - mc.e15);
              // (selected, not multiplied by zero: a masked pair's terms
              // need not be finite)
              const double eu = fma((double)qq, gd, eU);
              eU = (ok && inC) ? eu : eU;
              // LJ: (A s^-6 - B s^-3) S with s^-1 = (1/r)^2 in FP64
              const double2 ab = s_ljd[row + tjt];
              const double i2 = rid * rid;
              const double i6 = i2 * i2 * i2;
              const double el = fma(fma(ab.x, i6, -ab.y) * i6, (double)svl, eL);
              eL = ok ? el : eL;
            }
          }
          if (kEnergy) npair += ok ? 1 : 0;
          const float f = ok ? flj + fc : 0.f;
          const float fx = __fmul_rn(ddx, f), fy = __fmul_rn(ddy, f), fz = __fmul_rn(ddz, f);
          fi[k][0] = __fsub_rn(fi[k][0], fx);
          fi[k][1] = __fsub_rn(fi[k][1], fy);
          fi[k][2] = __fsub_rn(fi[k][2], fz);
          fjx = __fadd_rn(fjx, fx);
          fjy = __fadd_rn(fjy, fy);
          fjz = __fadd_rn(fjz, fz);
        }
      }
      fjx += __shfl_xor_sync(0xffffffffu, fjx, 4);
      fjy += __shfl_xor_sync(0xffffffffu, fjy, 4);
      fjz += __shfl_xor_sync(0xffffffffu, fjz, 4);
      fjx += __shfl_xor_sync(0xffffffffu, fjx, 8);
      fjy += __shfl_xor_sync(0xffffffffu, fjy, 8);
      fjz += __shfl_xor_sync(0xffffffffu, fjz, 8);
      if (ti == 0 && valid) {
        if (!(fmaxf(fabsf(fjx), fmaxf(fabsf(fjy), fabsf(fjz))) < kScForceLim)) atomicOr(err, 2);
        atomicAdd(&facc[js], (unsigned long long)__float2ll_rn(fjx * 4294967296.0f));
        atomicAdd(&facc[nsl + js], (unsigned long long)__float2ll_rn(fjy * 4294967296.0f));
        atomicAdd(&facc[2 * nsl + js], (unsigned long long)__float2ll_rn(fjz * 4294967296.0f));
      }
    }
#pragma unroll
    for (int k = 0; k < 8; k++) {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        float v = fi[k][c];
        v += __shfl_xor_sync(0xffffffffu, v, 1);
        v += __shfl_xor_sync(0xffffffffu, v, 2);
        v += __shfl_xor_sync(0xffffffffu, v, 16);
        fi[k][c] = v;
      }
    }
    if (tj == 0 && h == 0) {
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const size_t is = (size_t)s * kScAtoms + k * 4 + ti;
        if (!(fmaxf(fabsf(fi[k][0]), fmaxf(fabsf(fi[k][1]), fabsf(fi[k][2]))) < kScForceLim))
          atomicOr(err, 2);
#pragma unroll
        for (int c = 0; c < 3; c++)
          atomicAdd(&facc[(size_t)c * nsl + is],
                    (unsigned long long)__float2ll_rn(fi[k][c] * 4294967296.0f));
      }
    }
    if (kEnergy) {
      double pc = (double)npair;
      for (int off = 16; off > 0; off >>= 1) {
        eU += __shfl_xor_sync(0xffffffffu, eU, off);
        eL += __shfl_xor_sync(0xffffffffu, eL, off);
        pc += __shfl_xor_sync(0xffffffffu, pc, off);
      }
      if (lane == 0) {
        double *row = partial + (size_t)task * kNacc;
        row[ACC_ECOUL] = eU;
        row[ACC_ELJ] = eL;
        row[ACC_PAIRS] = pc;
      }
    }
  }
}

// Forces back to the original order: forces[atom] (+)= facc[slot] 2^-32.
__global__ void k_sc_finalize(const int *__restrict__ ctl, int nslot_max,
                              const int *__restrict__ satom,
                              const unsigned long long *__restrict__ facc, int accumulate,
                              double *__restrict__ forces) {
  pdl_wait();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= sc_ctl(ctl) * kScAtoms) return;
  const int a = satom[p];
  if (a < 0) return;
  double *fo = forces + 3 * (size_t)a;
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const double v = (double)(long long)facc[(size_t)q * nslot_max + p] * kFixInv;
    fo[q] = accumulate ? fo[q] + v : v;
  }
}

// k_reduce1 over a row count held on the device (the task count).
__global__ void k_sc_reduce1(const int *__restrict__ nrows, const double *__restrict__ partial,
                             double *__restrict__ red, int ns) {
  __shared__ double sh[8][ACC_MV];
  const int nr = sc_ctl(nrows);
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int span = (nr + gridDim.x - 1) / gridDim.x;
  const int lo = blockIdx.x * span, hi = min(nr, lo + span);
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
    red[blockIdx.x * ACC_MV + t] = acc;
  }
}

}  // namespace pmb200
