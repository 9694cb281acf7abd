// Cluster-pair ("tile") variant of the mixed pair kernel, cutoff form
// (LJ(C2) + Coulomb(C1), OneAtomPairTwo::doOneAtomPair, OneAtomPairTwo.h:
// 57-125) and the real-space Ewald forms.
//
// The same grid, cell sort and half-shell stencil as k_pair_mixed; within a
// cell the atoms are sorted by height (k_rank_gather's z order), so that
// every run of kTile consecutive atoms of a cell is a compact cluster.  A
// warp takes one i-cell and one share of the stencil offsets (as
// k_pair_mixed); for each i-cluster of its cell it tests the bounding boxes
// of the j-clusters of its neighbour cells against the i-cluster's box (one
// test per cluster pair, not per atom pair), keeps those within the cutoff
// in a shared-memory list, and then evaluates the kept cluster pairs two at
// a time: lane = 16 h + 4 a + b takes i atom a and j atom b of list entry
// e + h.  Every atom pair of a tile is tested against the exact cutoff
// (the pair set is the search kernel's); pairs beyond it, excluded pairs,
// padding lanes and home-cell pairs with j <= i are masked.  The j forces of
// a step are summed over the tile's four i lanes by shuffles and added to
// the int64 fixed-point accumulator (2^-32 quanta) by one lane per j atom;
// i forces are summed per lane in FP32 (in 2^-18 quanta) for kTileFlush
// steps at a time, then folded into int64 and finally combined over the
// atom's lanes.  Every global sum is an integer sum: deterministic.
// Energies: the LJ energy in FP32 per lane (into FP64 per flush), the
// cutoff form's Coulomb energy as q_j g(r) in FP64 from FP64 distances (as
// the search kernel), the Ewald forms' in FP32 (Kahan).
#pragma once

namespace pmb200 {

constexpr int kTile = 4;          // atoms per cluster
constexpr int kTileCap = 96;      // cluster-pair entries per list batch (per warp)
constexpr int kTileFlush = 8;     // steps between i-force folds into int64

struct __align__(16) TileWarpSmem {
  int js[kTileCap];     // j-cluster's first sorted index | (atoms - 1) << 29
  float sx[kTileCap];   // the j cell's shift into the i-cell frame (cell units)
  float sy[kTileCap];
  float sz[kTileCap];
  unsigned char home[kTileCap];  // 1: the i-cell itself (pairs j > i only)
};

// Bounding boxes of the clusters of one cell (cell units, the cell's frame):
// written at the first sorted index of each cluster.  One warp per cell.
__global__ void k_cluster_boxes(int ncell, const int *__restrict__ start,
                                const float4 *__restrict__ spos, float4 *__restrict__ blo,
                                float4 *__restrict__ bhi) {
  pdl_wait();
  const int lane = threadIdx.x & 31;
  const int cell = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (cell >= ncell) return;
  const int s = start[cell], e = start[cell + 1];
  for (int c0 = s + kTile * lane; c0 < e; c0 += kTile * 32) {
    const int c1 = min(c0 + kTile, e);
    float4 lo = spos[c0], hi = lo;
    for (int k = c0 + 1; k < c1; k++) {
      const float4 p = spos[k];
      lo.x = fminf(lo.x, p.x); lo.y = fminf(lo.y, p.y); lo.z = fminf(lo.z, p.z);
      hi.x = fmaxf(hi.x, p.x); hi.y = fmaxf(hi.y, p.y); hi.z = fmaxf(hi.z, p.z);
    }
    blo[c0] = lo;
    bhi[c0] = hi;
  }
}

template <int kForm, bool kEnergy>
__global__ void __launch_bounds__(32, kEnergy ? 16 : 20)
k_pair_tiles(GridParams g, MixedConsts mc, const HalfStencil st, int ntypes,
             const float4 *__restrict__ lj32, const int *__restrict__ start,
             const float4 *__restrict__ spos, const int2 *__restrict__ smeta,
             const int *__restrict__ sidx, const int *__restrict__ ex_start,
             const int2 *__restrict__ ex, const float4 *__restrict__ blo,
             const float4 *__restrict__ bhi, unsigned long long *__restrict__ facc, int n,
             int *__restrict__ err, double *__restrict__ partial, int slots,
             const float4 *__restrict__ spos_lo) {
  extern __shared__ float4 s_dyn[];
  __shared__ TileWarpSmem sm;
  constexpr bool kExactE = kEnergy && kForm == FORM_CUTOFF;
  const int nlj = kForm == FORM_CUTOFF ? ntypes * ntypes : 0;
  float4 *s_lj = s_dyn;
  unsigned short *s_st = reinterpret_cast<unsigned short *>(s_dyn + nlj);
  const int lane = threadIdx.x;
  for (int k = lane; k < nlj; k += 32) s_lj[k] = lj32[k];
  for (int k = lane; k < st.ncells; k += 32) s_st[k] = st.off[k];
  __syncwarp();
  pdl_wait();
  const int cell = (int)(blockIdx.x / slots), slot = (int)(blockIdx.x % slots);
  if (cell >= g.ncell) return;  // uniform per block
  const int cx = cell % g.nx;
  const int cy = (cell / g.nx) % g.ny;
  const int cz = cell / (g.nx * g.ny);
  const int cs = start[cell], ce = start[cell + 1];
  const int h = lane >> 4, a = (lane >> 2) & 3, b = lane & 3;
  double accU = 0.0, accE = 0.0, accP = 0.0;
  KahanF kU;
  for (int g0 = cs; g0 < ce; g0 += kTile) {
    // this i-cluster: atoms g0 .. g0 + ni - 1
    const int ni = min(kTile, ce - g0);
    const bool ivalid = a < ni;
    const int i = g0 + (ivalid ? a : 0);
    const float4 pi = spos[i];
    const int2 mi = smeta[i];
    const int oi = sidx[i];
    const int elo = ex_start[oi], ehi = ex_start[oi + 1];
    const int ti = mi.x * ntypes;
    const float4 ilo = blo[g0], ihi = bhi[g0];
    double pid_x = 0.0, pid_y = 0.0, pid_z = 0.0;
    if (kExactE) {
      const float4 li = spos_lo[i];
      pid_x = (double)pi.x + (double)li.x;
      pid_y = (double)pi.y + (double)li.y;
      pid_z = (double)pi.z + (double)li.z;
    }
    double eU = 0.0;
    float px = 0.f, py = 0.f, pz = 0.f, pE = 0.f;
    long long fx = 0, fy = 0, fz = 0;
    int nsteps = 0, pc = 0;
    int nl = 0;  // list entries
    // the kept cluster pairs, two per step
    auto process = [&]() {
      __syncwarp();
      for (int e0 = 0; e0 < nl; e0 += 2) {
        const int e = e0 + h;
        const bool evalid = e < nl;
        const int jw = sm.js[evalid ? e : e0];
        const int j0 = jw & 0x1fffffff, nj = (jw >> 29) + 1;
        const bool jvalid = evalid && b < nj;
        const int j = j0 + (jvalid ? b : 0);
        const float4 pj0 = spos[j];
        const float shx = sm.sx[evalid ? e : e0], shy = sm.sy[evalid ? e : e0],
                    shz = sm.sz[evalid ? e : e0];
        const float pjx = pj0.x + shx, pjy = pj0.y + shy, pjz = pj0.z + shz;
        const float ddx = pjx - pi.x, ddy = pjy - pi.y, ddz = pjz - pi.z;
        const float r2 = fmaf(ddx, ddx, fmaf(ddy, ddy, ddz * ddz));
        const int2 mj = smeta[j];
        bool use = ivalid && jvalid && r2 <= mc.cut2 &&
                   !(sm.home[evalid ? e : e0] && j <= i);
        int kind = 0;
        if (__any_sync(0xffffffffu, use && mj.y == mi.y)) {
          if (use && mj.y == mi.y) {
            kind = excl_kind(ex, elo, ehi, sidx[j]);
            if (kind == 2) use = false;
          }
        }
        float fxv = 0.f, fyv = 0.f, fzv = 0.f;
        if (use) {
          float rinv = rsqrtf(r2);
          rinv = fmaf(0.5f * rinv, fmaf(-r2 * rinv, rinv, 1.0f), rinv);
          const float r2inv = rinv * rinv;
          float f;
          float qj = pj0.w;
          if (kind == 1) qj *= mc.csf;
          if constexpr (kForm == FORM_CUTOFF) {
            const float4 p = s_lj[ti + mj.x];
            const float A = kind == 1 ? p.z : p.x;
            const float B = kind == 1 ? p.w : p.y;
            const float r6 = r2inv * r2inv * r2inv;
            float elj = fmaf(A, r6, -B) * r6;
            float flj = fmaf(12.0f * A, r6, -6.0f * B) * r6 * r2inv;
            {  // C2 switch: value 1 below switchon, 0 beyond the LJ cutoff
              const float c2 = mc.rclj2 - r2;
              const float c4 = c2 * fmaf(2.0f, r2, mc.s2);
              const bool on = r2 >= mc.ron2;
              const bool in = r2 <= mc.rclj2;
              const float sv = in ? (on ? mc.s1 * (c2 * c4) : 1.0f) : 0.0f;
              const float sd = (in && on) ? mc.s3 * fmaf(c2, c2, -c4) : 0.0f;
              flj = fmaf(flj, sv, -elj * sd);
              elj = __fmul_rn(elj, sv);
            }
            float fc;
            {  // C1 switched Coulomb, zero beyond its cutoff
              const bool inC = r2 <= mc.rcc2;
              const float ec = pi.w * qj * rinv;
              const float dist = r2 * rinv;
              const float sv = fmaf(-dist, fmaf(-r2, mc.c05_3, mc.c15_1), 1.0f);
              const float sd = fmaf(dist, mc.c15_3, -mc.c15_1 * rinv);
              fc = inC ? __fmul_rn(ec, fmaf(r2inv, sv, -sd)) : 0.f;
              if (kEnergy) {
                // q_j g(r) from the FP64 distance (see mixed_task)
                const float4 lj = spos_lo[j];
                const double ex_ = (((double)pj0.x + (double)lj.x) + (double)shx) - pid_x;
                const double ey_ = (((double)pj0.y + (double)lj.y) + (double)shy) - pid_y;
                const double ez_ = (((double)pj0.z + (double)lj.z) + (double)shz) - pid_z;
                const double r2d = fma(ex_, ex_, fma(ey_, ey_, ez_ * ez_));
                double rid = (double)rinv;
                rid = rid * fma(-0.5 * r2d, rid * rid, 1.5);
                const double gd = fma(mc.e05, r2d, rid - mc.e15);
                eU = fma(inC ? (double)qj : 0.0, gd, eU);
              }
            }
            f = flj + fc;
            if (kEnergy) pE += elj;
          } else {
            // real-space Ewald (NonbondedFullEwaldSystemForce.h:803-823)
            const float x = mc.ea * (r2 * rinv);
            const float exf = expf(-x * x);
            float gg;
            if constexpr (kForm == FORM_EWALD_POLY5) {
              const float t = __fdividef(1.0f, fmaf((float)kAsP, x, 1.0f));
              const float poly =
                  t * fmaf(t, fmaf(t, fmaf(t, fmaf(t, (float)kAsA5, (float)kAsA4),
                                           (float)kAsA3),
                                   (float)kAsA2),
                           (float)kAsA1);
              gg = poly * exf * rinv;
            } else {
              gg = erfcf(x) * rinv;
            }
            f = pi.w * qj * fmaf(mc.ea2pi, exf, gg) * r2inv;
            if (kEnergy) kU.add(__fmul_rn(qj, gg));
          }
          const float fq = f * kJScale;
          fxv = ddx * fq; fyv = ddy * fq; fzv = ddz * fq;
          px = __fsub_rn(px, fxv);
          py = __fsub_rn(py, fyv);
          pz = __fsub_rn(pz, fzv);
          if (kEnergy) pc++;
        }
        // j force of the step: summed over the tile's four i lanes
        for (int off = 4; off <= 8; off <<= 1) {
          fxv += __shfl_xor_sync(0xffffffffu, fxv, off);
          fyv += __shfl_xor_sync(0xffffffffu, fyv, off);
          fzv += __shfl_xor_sync(0xffffffffu, fzv, off);
        }
        if (a == 0 && jvalid) {
          const float fm = fmaxf(fabsf(fxv), fmaxf(fabsf(fyv), fabsf(fzv)));
          if (!(fm < 2.8e14f)) atomicOr(err, 2);
          if (fm > 0.f) {
            atomicAdd(&facc[j], (unsigned long long)__float2ll_rn(fxv * kJToGlobal));
            atomicAdd(&facc[(size_t)n + j], (unsigned long long)__float2ll_rn(fyv * kJToGlobal));
            atomicAdd(&facc[2 * (size_t)n + j],
                      (unsigned long long)__float2ll_rn(fzv * kJToGlobal));
          }
        }
        if (++nsteps == kTileFlush) {
          nsteps = 0;
          fx += __float2ll_rn(px * kJToGlobal);
          fy += __float2ll_rn(py * kJToGlobal);
          fz += __float2ll_rn(pz * kJToGlobal);
          px = py = pz = 0.f;
          if (kEnergy) { accE += (double)pE; pE = 0.f; }
        }
      }
      nl = 0;
      __syncwarp();
    };
    // candidate j-clusters of this warp's stencil share, 32 at a time
    const int first = slot, stride = slots;
    const int nmine = first < st.ncells ? (st.ncells - first + stride - 1) / stride : 0;
    for (int q0 = 0; q0 < nmine; q0 += 32) {
      const int myq = q0 + lane;
      int cjs = 0, cje = 0, ccnt = 0;  // the cell's first cluster start, end, cluster count
      float csx = 0.f, csy = 0.f, csz = 0.f;
      bool chome = false;
      if (myq < nmine) {
        const unsigned o = s_st[first + myq * stride];
        const int dx = (int)(o & 31u) - 8, dy = (int)((o >> 5) & 31u) - 8,
                  dz = (int)((o >> 10) & 31u) - 8;
        chome = (dx | dy | dz) == 0;
        int jx = cx + dx, jy = cy + dy, jz = cz + dz;
        bool inside = true;
        if (g.periodic) {
          jx += jx < 0 ? g.nx : (jx >= g.nx ? -g.nx : 0);
          jy += jy < 0 ? g.ny : (jy >= g.ny ? -g.ny : 0);
          jz += jz < 0 ? g.nz : (jz >= g.nz ? -g.nz : 0);
        } else {
          inside = jx >= 0 && jx < g.nx && jy >= 0 && jy < g.ny && jz >= 0 && jz < g.nz;
        }
        if (inside) {
          const int jc = (jz * g.ny + jy) * g.nx + jx;
          cjs = chome ? g0 : start[jc];  // home cell: from the i-cluster on (j > i pairs)
          cje = start[jc + 1];
          ccnt = (cje - cjs + kTile - 1) / kTile;
        }
        csx = (float)dx; csy = (float)dy * mc.ey; csz = (float)dz * mc.ez;
      }
      int incl = ccnt;  // inclusive prefix of the cells' cluster counts
      for (int off = 1; off < 32; off <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += v;
      }
      const int total = __shfl_sync(0xffffffffu, incl, 31);
      for (int f0 = 0; f0 < total; f0 += 32) {
        const int f = f0 + lane;
        int c = 0;  // the cell of candidate f
        for (int step = 16; step > 0; step >>= 1) {
          const int v = __shfl_sync(0xffffffffu, incl, c + step - 1);
          if (v <= f) c += step;
        }
        const int js_c = __shfl_sync(0xffffffffu, cjs, c);
        const int je_c = __shfl_sync(0xffffffffu, cje, c);
        const int ex_c = __shfl_sync(0xffffffffu, incl - ccnt, c);
        const float sx = __shfl_sync(0xffffffffu, csx, c);
        const float sy = __shfl_sync(0xffffffffu, csy, c);
        const float sz = __shfl_sync(0xffffffffu, csz, c);
        const bool home = __shfl_sync(0xffffffffu, chome ? 1 : 0, c) != 0;
        bool keep = false;
        int jw = 0;
        if (f < total) {
          const int j0 = js_c + kTile * (f - ex_c);
          const int nj = min(kTile, je_c - j0);
          const float4 jl = blo[j0], jh = bhi[j0];
          // gap between the boxes in the i-cell frame, in the pair test's
          // operation order (monotonic rounding: no pair within the cutoff
          // is dropped)
          const float gx = fmaxf(fmaxf((jl.x + sx) - ihi.x, ilo.x - (jh.x + sx)), 0.f);
          const float gy = fmaxf(fmaxf((jl.y + sy) - ihi.y, ilo.y - (jh.y + sy)), 0.f);
          const float gz = fmaxf(fmaxf((jl.z + sz) - ihi.z, ilo.z - (jh.z + sz)), 0.f);
          keep = fmaf(gx, gx, fmaf(gy, gy, gz * gz)) <= mc.cut2;
          jw = j0 | ((nj - 1) << 29);
        }
        const unsigned km = __ballot_sync(0xffffffffu, keep);
        if (keep) {
          const int s = nl + __popc(km & ((1u << lane) - 1u));
          sm.js[s] = jw;
          sm.sx[s] = sx; sm.sy[s] = sy; sm.sz[s] = sz;
          sm.home[s] = home ? 1 : 0;
        }
        nl += __popc(km);
        if (nl > kTileCap - 32) process();
      }
    }
    if (nl > 0) process();
    // i forces: the atom's eight lanes (b, h) combined, then the accumulator
    fx += __float2ll_rn(px * kJToGlobal);
    fy += __float2ll_rn(py * kJToGlobal);
    fz += __float2ll_rn(pz * kJToGlobal);
    for (int off = 1; off <= 16; off <<= 1) {
      if (off == 4 || off == 8) continue;  // (a: another atom)
      fx += __shfl_xor_sync(0xffffffffu, fx, off);
      fy += __shfl_xor_sync(0xffffffffu, fy, off);
      fz += __shfl_xor_sync(0xffffffffu, fz, off);
    }
    if (ivalid && b == 0 && h == 0) {
      atomicAdd(&facc[i], (unsigned long long)fx);
      atomicAdd(&facc[(size_t)n + i], (unsigned long long)fy);
      atomicAdd(&facc[2 * (size_t)n + i], (unsigned long long)fz);
    }
    if (kEnergy) {
      accE += (double)pE;
      accP += (double)pc;
      if (ivalid) {
        const double qi = (double)pi.w;
        if (kExactE) accU += qi * eU;
        else accU += qi * ((double)kU.s - (double)kU.c);
      }
      kU = KahanF();
    }
  }
  if (kEnergy) {
    double v[ACC_MV];
#pragma unroll
    for (int k = 0; k < ACC_MV; k++) v[k] = 0.0;
    v[ACC_ECOUL] = accU; v[ACC_ELJ] = accE; v[ACC_PAIRS] = accP;
    write_partial_row<ACC_E>(v, lane, partial + (size_t)blockIdx.x * kNacc);
  }
}

}  // namespace pmb200
