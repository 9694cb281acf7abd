// Batched evaluation of many independent periodic systems of uneven size:
// one counting sort over every atom of the batch, one persistent pair
// kernel over a task list (system, cell, part of the cell's stencil), one
// fixed-point finalize and one per-system reduction.
//
// Layout in HBM (N atoms and C cells over all systems, systems back to back):
//   sys[S]            BatchSys: each system's grid, constants, offsets
//   atom_sys[N]       system of each atom (caller order)
//   type/mol/q[N]     per atom; molecule ids stay system-local
//   ex_start[N+1]/ex  exclusion CSR over batch-wide atom indices
//   stencils[...]     each system's half-shell offsets, back to back
//   lj32[...]         each system's LJ table in its own cell units
//   cell arrays [C]   cell_count/cell_start over batch-wide cell ids
//   tasks[T]          int4 {system, cell (system-local), part, parts}
//   partial[T][NACC]  per-task energy / virial partials
//   rows_start[S+1], rows[T]: each system's task rows (fixed order)
#pragma once
#include "pmb200_kernels.cuh"

namespace pmb200 {

struct BatchSys {
  GridParams g;
  MixedConsts mc;
  PbcRef pb;
  double fscale;         // fixed point -> force: 2^-32 / cell edge
  float qscale32;        // 1 / sqrt(cell edge)
  int cell0, atom0, natoms;
  int st0, st_n;         // stencil slice
  int lj0, ntypes;       // LJ table slice
};

__global__ void k_cell_index_batch(int N, const double *__restrict__ pos,
                                   const BatchSys *__restrict__ sys,
                                   const int *__restrict__ atom_sys, int *__restrict__ cell_of,
                                   int *__restrict__ cell_count, int *__restrict__ slot,
                                   float4 *__restrict__ rel32, const double *__restrict__ q,
                                   int *__restrict__ err, float4 *__restrict__ rel_lo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const BatchSys &b = sys[atom_sys[i]];
  int c[3];
  double r[3];
  if (!locate_cell(pos + 3 * (size_t)i, b.g, c, r)) atomicOr(err, 1);
  const int cid = b.cell0 + (c[2] * b.g.ny + c[1]) * b.g.nx + c[0];
  cell_of[i] = cid;
  slot[i] = atomicAdd(&cell_count[cid], 1);
  const double inv = 1.0 / b.g.unit;
  const double v[3] = {r[0] * inv, r[1] * inv, r[2] * inv};
  const float h[3] = {(float)v[0], (float)v[1], (float)v[2]};
  rel32[i] = make_float4(h[0], h[1], h[2], (float)q[i] * b.qscale32);
  if (rel_lo)  // the FP32 coordinates' rounding residuals (energy evaluations)
    rel_lo[i] = make_float4((float)(v[0] - (double)h[0]), (float)(v[1] - (double)h[1]),
                            (float)(v[2] - (double)h[2]), 0.f);
}

// Persistent pair kernel, one warp per block: each warp takes tasks (system,
// i-cell, stencil part, parts) from a global counter until the list is
// exhausted and never waits for another warp; a task's system parameters,
// stencil and LJ table are staged in the warp's shared memory when the system
// changes.  Dynamic shared memory: lj_max float4 LJ records, then st_max
// stencil offsets (the largest of any system in the batch).
template <int kForm, bool kEnergy, bool kVirial>
__global__ void __launch_bounds__(32, (kEnergy || kVirial) ? 1 : 24)
k_pair_mixed_batch(const BatchSys *__restrict__ sys, const int4 *__restrict__ tasks, int ntasks,
                   int *__restrict__ counter, const unsigned short *__restrict__ stencils,
                   const float4 *__restrict__ lj32, const int *__restrict__ start,
                   const float4 *__restrict__ spos, const int2 *__restrict__ smeta,
                   const int *__restrict__ sidx, const int *__restrict__ ex_start,
                   const int2 *__restrict__ ex, unsigned long long *__restrict__ facc, int N,
                   double *__restrict__ partial, int *__restrict__ err,
                   const float4 *__restrict__ spos_lo, int lj_max) {
  extern __shared__ float4 s_dyn[];
  __shared__ MixedWarpSmem sm;
  __shared__ BatchSys s_sys;
  __shared__ float s_res[(kEnergy && kForm == FORM_CUTOFF) ? 3 * kBatch : 1];
  float4 *s_lj = s_dyn;
  unsigned short *s_st = reinterpret_cast<unsigned short *>(s_dyn + lj_max);
  const int lane = threadIdx.x;
  for (int t = lane; t < kBatch; t += 32) sm.jf[0][t] = sm.jf[1][t] = sm.jf[2][t] = 0;
  sm.fi[0][lane] = sm.fi[1][lane] = sm.fi[2][lane] = 0;
  int loaded = -1;
  for (;;) {
    int t = 0;
    if (lane == 0) t = atomicAdd(counter, 1);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= ntasks) break;  // uniform per warp
    const int4 tk = tasks[t];
    if (tk.x != loaded) {
      // stage the system: parameters (as 32-bit words), stencil, LJ table
      __syncwarp();
      const int *src = reinterpret_cast<const int *>(&sys[tk.x]);
      int *dst = reinterpret_cast<int *>(&s_sys);
      for (int k = lane; k < (int)(sizeof(BatchSys) / sizeof(int)); k += 32) dst[k] = src[k];
      const BatchSys &gs = sys[tk.x];
      for (int k = lane; k < gs.st_n; k += 32) s_st[k] = stencils[gs.st0 + k];
      if (kForm == FORM_CUTOFF || kForm == FORM_GENERIC)
        for (int k = lane; k < gs.ntypes * gs.ntypes; k += 32) s_lj[k] = lj32[gs.lj0 + k];
      loaded = tk.x;
      __syncwarp();
    }
    // the task's stencil entries: part + k * parts
    mixed_task<kForm, kEnergy, kVirial, false>(
        s_sys.g, s_sys.mc, s_st, s_sys.st_n, tk.z, tk.w, s_sys.ntypes, s_lj, tk.y,
        start + s_sys.cell0, spos, smeta, sidx, ex_start, ex, facc, N,
        partial + (size_t)t * kNacc, s_sys.pb, nullptr, sm, err,
        (kEnergy && kForm == FORM_CUTOFF) ? s_res : nullptr, spos_lo);
  }
}

// Fixed point (sorted order) -> FP64 forces in caller order, each atom at
// its own system's scale.
__global__ void k_finalize_batch(int N, const unsigned long long *__restrict__ facc,
                                 const int *__restrict__ sidx, const int *__restrict__ atom_sys,
                                 const BatchSys *__restrict__ sys, int accumulate,
                                 double *__restrict__ forces) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  const int o = sidx[j];
  const double scale = sys[atom_sys[o]].fscale;
  double *fo = forces + 3 * (size_t)o;
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const double v = (double)(long long)facc[(size_t)q * N + j] * scale;
    fo[q] = accumulate ? fo[q] + v : v;
  }
}

// One warp per system: its task rows summed in list order (deterministic),
// then the same outputs as k_reduce2 (out[s][20]: COULOMB, LENNARDJONES,
// virial 9, molecular virial 9 (zero)); pairs[s] = in-cutoff pair count.
__global__ void k_reduce_batch(int nsys, const int *__restrict__ rows_start,
                               const int *__restrict__ rows, const double *__restrict__ partial,
                               const BatchSys *__restrict__ sys, double *__restrict__ out,
                               double *__restrict__ pairs, int ns) {
  const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (s >= nsys) return;
  double acc = 0.0;  // lane k < ns sums slot k (the slots the launch filled; the rest 0)
  if (lane < ns)
    for (int r = rows_start[s]; r < rows_start[s + 1]; r++)
      acc += partial[(size_t)rows[r] * kNacc + lane];
  double v[ACC_MV];
#pragma unroll
  for (int k = 0; k < ACC_MV; k++) v[k] = __shfl_sync(0xffffffffu, acc, k);
  if (lane != 0) return;
  double *o = out + 20 * (size_t)s;
  o[0] = v[ACC_ECOUL];
  o[1] = v[ACC_ELJ];
  const int map[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
  for (int k = 0; k < 9; k++) {
    o[2 + k] = v[ACC_W + map[k]];
    o[11 + k] = 0.0;
  }
  if (pairs) pairs[s] = v[ACC_PAIRS];
}

}  // namespace pmb200
