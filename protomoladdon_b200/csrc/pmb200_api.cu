// libpmb200: host side of the C ABI declared in include/pmb200.h.
//
// One context = one periodic system on one GPU: device copies of the
// topology, the cell grid for the current box, per-evaluation buffers and a
// CUDA stream.  An evaluation is
//   k_cell_index -> k_scan -> k_scatter -> k_rank_gather   (counting sort)
//   k_pair_mixed | k_pair_fp64                            (forces, partials)
//   [k_com -> k_molvir] -> k_reduce                        (energies, virial)
// all on the context's stream.
#include "../../include/pmb200.h"
#include "pmb200_kernels.cuh"
#include "pmb200_tiles.cuh"
#include "pmb200_clusters.cuh"

#include <algorithm>
#include <cmath>
#include <limits>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

using namespace pmb200;

// page-locked result words of a host-buffer evaluation: 20 doubles (energies,
// virial, molecular virial) and the device error flag behind them
constexpr int kPinOut = 21;

struct pmb200_ctx {
  pmb200_params p{};
  std::string err;
  // pair potential: FORM_CUTOFF, or the Ewald real-space term with its
  // parameters and the alpha / cutoff derived from them
  int form = FORM_CUTOFF;
  double ew_alpha_in = 0.0, ew_accuracy = 0.0;
  double ew_alpha = 0.0, ew_rc = 0.0;
  // generic form: switch kind and {switchon, cutoff, order, switchoff} per
  // potential (LJ, Coulomb)
  int sw_kind[2] = {0, 0};
  double sw_par[2][4] = {};
  // mixed kernel warps per i-cell for forces-only and for energy / virial
  // launches (0: mixed_cell_slots' choice; set by pmb200_autotune)
  int slots_f = 0, slots_e = 0;
  // mixed pair kernel for energy and for forces-only launches: the
  // cluster-pair (tile) kernel where it applies (pmb200_set_pair_kernel,
  // pmb200_autotune), else the search kernel
  bool tiles_e = false, tiles_f = false;
  float4 *d_cblo = nullptr, *d_cbhi = nullptr;  // cluster boxes (tile kernel)
  // supercluster pair kernel (pmb200_clusters.cuh) for energy and forces-only
  // launches, where it applies (sc_ok: mixed cutoff form, orthogonal
  // periodic box wide enough, at most kMaxTypes types, no modified pairs)
  bool clu_e = false, clu_f = false, sc_ok = false;
  bool has_modified = false;  // the exclusion list holds modified (1-4) pairs
  ScGrid sg{};
  ScStencil sst{};
  MixedConsts mca{};          // the pair constants in A
  int sc_grid_e = 0, sc_grid_f = 0;  // persistent pair-kernel blocks
  bool sc_full = false;       // both switch cutoffs equal the pair cutoff
  double sc_side = 1.0;       // column width / edge of a cube of 32 atoms (pmb200_autotune)
  int sc_ncell_alloc = 0, sc_ncol_alloc = 0, sc_nsup_alloc = 0;
  bool sc_count_zero = false;
  int *d_sc_count = nullptr, *d_sc_start = nullptr, *d_sc_supbase = nullptr;
  int *d_sc_ctl = nullptr, *d_sc_atom = nullptr, *d_sc_type = nullptr, *d_sc_mol = nullptr;
  int *d_sc_cnt = nullptr;
  float4 *d_sc_xi = nullptr, *d_sc_xj = nullptr, *d_sc_xilo = nullptr, *d_sc_xjlo = nullptr;
  float4 *d_sc_clo = nullptr, *d_sc_chi = nullptr, *d_sc_sbox = nullptr;
  int4 *d_sc_corg = nullptr, *d_sc_sorg = nullptr, *d_sc_tasks = nullptr;
  int2 *d_sc_cmol = nullptr;
  ScEntry *d_sc_ent = nullptr;
  unsigned long long *d_sc_facc = nullptr;
  double *d_sc_part = nullptr;
  // tabulated LJ (LennardJonesTableForce under UniversalSwitchingFunction):
  // the FP64 grid on the device (null: analytic LJ)
  double4 *d_ljtab = nullptr;
  int tab_first = 0, tab_last = 0;
  // vacuum boundaries: the box is only the cell domain (no wrap, no images)
  bool vacuum = false, vacuum_pending = false;
  // the box as last given (re-applied when an Ewald default alpha changes)
  bool box_given = false;
  double box_e[3][3] = {}, box_origin[3] = {};
  cudaStream_t stream = nullptr;
  // topology
  int n = 0, ntypes = 0, nmol = 0;
  bool have_topo = false, have_box = false, have_mass = false;
  double csf = 1.0;
  std::vector<double> h_lj;  // ntypes^2 * 4
  int *d_type = nullptr, *d_mol = nullptr;
  double *d_q = nullptr, *d_mass = nullptr;
  int *d_ex_start = nullptr;
  int2 *d_ex = nullptr;
  int *d_mstart = nullptr, *d_matoms = nullptr;
  float4 *d_lj32 = nullptr;
  double4 *d_lj64 = nullptr;
  // grid
  GridParams g{};
  MixedConsts mc{};
  Fp64Consts fc{};
  PbcRef pb{};
  std::vector<Row> rows;
  Stencil stencil{};       // full shell (FP64 kernel)
  HalfStencil half{};      // half shell by cell (mixed kernel, Newton's third law)
  int ncell_alloc = 0;
  int *d_count = nullptr, *d_start = nullptr, *d_err = nullptr;
  double *d_partial = nullptr;
  // per-atom buffers
  int n_alloc = 0;
  int *d_cell_of = nullptr, *d_slot = nullptr, *d_tmp = nullptr, *d_sidx = nullptr;
  float4 *d_rel32 = nullptr, *d_spos32 = nullptr;
  float4 *d_rel_lo = nullptr, *d_spos_lo = nullptr;  // FP32 coordinate residuals
  double4 *d_rel64 = nullptr, *d_spos64 = nullptr;
  int2 *d_smeta = nullptr;
  // force accumulator, sorted order: [3][n] 2^-32 quanta (mixed) or [6][n]
  // two-word fixed point (FP64 evaluation kernel)
  unsigned long long *d_facc = nullptr;
  // d_count holds zeros between evaluations (k_scan clears it after reading);
  // false after a launch sequence broke off, when the next build clears it
  bool count_zero = false;
  double *d_com = nullptr;
  // derivative kernels: per-block table rows and scratch outputs
  double *d_tpart = nullptr, *d_gq = nullptr, *d_glj = nullptr;
  size_t tpart_alloc = 0, gq_alloc = 0, glj_alloc = 0;
  double4 *d_wsorted = nullptr;  // a Hessian-vector product's direction, sorted order
  size_t ws_alloc = 0;
  double *d_pairs = nullptr, *d_out = nullptr, *d_red = nullptr;
  unsigned *d_redctr = nullptr;  // k_finalize_reduce's arrival counter (wraps to 0)
  // rigid waters (SETTLE) for the device integrator
  int nwater = 0, nfree = 0;
  int *d_widx = nullptr, *d_fidx = nullptr;
  SettleParams sp{};
  // host-buffer evaluation scratch: device copies and pinned staging
  double *d_hpos = nullptr, *d_hfrc = nullptr;
  // host-buffer calls of mixed contexts read the forces back in FP32
  float *d_hf32 = nullptr;
  double *h_pin_pos = nullptr, *h_pin_frc = nullptr, *h_pin_out = nullptr;
  int n_pin = 0;
  // leapfrog graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  const void *graph_key[4] = {nullptr, nullptr, nullptr, nullptr};
  double graph_dt = 0.0;
  // one-step graph (pmb200_step_device)
  cudaGraph_t sgraph = nullptr;
  cudaGraphExec_t sgraph_exec = nullptr;
  const void *sgraph_key[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  double sgraph_dt = 0.0;
  unsigned sgraph_flags = 0;
  // host-buffer evaluation graph (pmb200_eval): copy in, evaluate, copy out
  cudaGraph_t hgraph = nullptr;
  cudaGraphExec_t hgraph_exec = nullptr;
  const void *hgraph_src = nullptr;
  unsigned hgraph_flags = 0;
  // pair-kernel timing
  int timing = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // the LJ table was last set on the device (pmb200_update_params_device):
  // h_lj is refreshed from d_lj64 after ev_lj before a host consumer reads it
  bool lj_dev_newer = false;
  cudaEvent_t ev_lj = nullptr;
};

namespace {

int fail(pmb200_ctx *c, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

#define CK(call)                                                                 \
  do {                                                                           \
    cudaError_t e_ = (call);                                                     \
    if (e_ != cudaSuccess)                                                       \
      return fail(c, PMB200_ECUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

template <class T>
void dfree(T *&p) {
  if (p) cudaFree((void *)p);
  p = nullptr;
}

template <class T>
cudaError_t dalloc(T *&p, size_t count) {
  dfree(p);
  if (count == 0) count = 1;
  return cudaMalloc((void **)&p, sizeof(T) * count);
}

void release_graph(pmb200_ctx *c) {
  if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
  if (c->graph) cudaGraphDestroy(c->graph);
  c->graph_exec = nullptr;
  c->graph = nullptr;
  for (auto &k : c->graph_key) k = nullptr;
  if (c->sgraph_exec) cudaGraphExecDestroy(c->sgraph_exec);
  if (c->sgraph) cudaGraphDestroy(c->sgraph);
  c->sgraph_exec = nullptr;
  c->sgraph = nullptr;
  for (auto &k : c->sgraph_key) k = nullptr;
  if (c->hgraph_exec) cudaGraphExecDestroy(c->hgraph_exec);
  if (c->hgraph) cudaGraphDestroy(c->hgraph);
  c->hgraph_exec = nullptr;
  c->hgraph = nullptr;
  c->hgraph_src = nullptr;
}

double rc_max(const pmb200_params &p) { return std::max(p.cutoff_lj, p.cutoff_coul); }

// Warps per i-cell of the context's mixed launches.
int ctx_slots(const pmb200_ctx *c, bool energy_or_virial) {
  const int s = energy_or_virial ? c->slots_e : c->slots_f;
  return s > 0 ? s : mixed_cell_slots(energy_or_virial, c->n, c->g.ncell);
}

// Pair cutoff of the context's potential.
double ctx_rc(const pmb200_ctx *c) {
  if (c->form == FORM_GENERIC) {
    double r = 0.0;
    for (int k = 0; k < 2; k++)
      if (c->sw_kind[k] != SW_OFF) r = std::max(r, c->sw_par[k][1]);
    return r;
  }
  return c->form == FORM_CUTOFF ? rc_max(c->p) : c->ew_rc;
}

// Cn polynomial coefficients (CnSwitchingFunction.cpp:9-31), rows by order
// 2, 3, 4, (5: all zero in the reference), 6.
const double kCnValue[5][7] = {{10., -15., 6., 0, 0, 0, 0},
                               {35., -84., 70., -20., 0, 0, 0},
                               {126., -420., 540., -315., 70., 0, 0},
                               {0, 0, 0, 0, 0, 0, 0},
                               {1716., -9009., 20020., -24024., 16380., -6006., 924.0}};
const double kCnDeriv[5][7] = {{30., -60., 30., 0, 0, 0, 0},
                               {140., -420., 420., -140., 0, 0, 0},
                               {630., -2520., 3780., -2520., 630., 0, 0},
                               {0, 0, 0, 0, 0, 0, 0},
                               {12012., -72072., 180180., -240240., 180180., -72072., 12012.0}};

double binomial(int n, int k) {
  double b = 1.0;
  for (int i = 1; i <= k; i++) b = b * (n - k + i) / i;
  return b;
}

// The Bernstein form used on the device reproduces the reference's power
// tables: expanding sum_j binom(2n+1, n+1+j) t^(n+1+j) (1-t)^(n-j) gives
// kCnValue's row (checked once per process, on the host).
bool cn_tables_agree() {
  for (int n : {2, 3, 4, 6}) {
    double poly[14] = {0};
    for (int j = 0; j <= n; j++) {
      const double b = binomial(2 * n + 1, n + 1 + j);
      for (int m = 0; m <= n - j; m++)  // (1-t)^(n-j) = sum_m binom(n-j, m) (-t)^m
        poly[n + 1 + j + m] += b * binomial(n - j, m) * ((m & 1) ? -1.0 : 1.0);
    }
    for (int i = 0; i <= n; i++)
      if (std::fabs(poly[n + 1 + i] - kCnValue[n - 2][i]) > 1e-9) return false;
  }
  return true;
}

// A switch's constants with lengths divided by u (1 for Angstrom).
template <class T>
SwitchSpec<T> make_switch(int kind, const double par[4], double u) {
  SwitchSpec<T> w{};
  w.kind = kind;
  if (kind == SW_OFF) return w;
  const double ron = par[0] / u, rc = par[1] / u;
  w.rc2 = (T)(rc * rc);
  w.rc = (T)rc;
  if (kind == SW_C1) {  // C1SwitchingFunction.cpp:12-16
    w.a = (T)(1.5 / rc);
    w.b = (T)(0.5 / (rc * rc * rc));
    w.c = (T)(1.5 / (rc * rc * rc));
  } else if (kind == SW_C2) {  // C2SwitchingFunction.cpp:12-18
    const double t = rc * rc - ron * ron;
    w.ron2 = (T)(ron * ron);
    w.a = (T)(1.0 / ((t * t) * t));
    w.b = (T)(rc * rc - 3.0 * ron * ron);
    w.c = (T)(4.0 / ((t * t) * t));
  } else if (kind == SW_CN) {  // CnSwitchingFunction.cpp:38-60
    const int n = (int)par[2];
    w.nord = n;
    w.ron2 = (T)(ron * ron);
    w.ron = (T)ron;
    w.inv_range = (T)(1.0 / (ron - rc));
    for (int j = 0; j <= n; j++) w.vcoef[j] = (T)binomial(2 * n + 1, n + 1 + j);
    w.dpeak = (T)kCnDeriv[n - 2][0];
  } else if (kind == SW_CMPCNCN) {  // CmpCnCnSwitchingFunction.cpp:16-33
    // order 5 is read as 2, as the reference's constructor does
    const int n = par[2] == 5.0 ? 2 : (int)par[2];
    const double roff = par[3] / u;
    w.nord = n;
    w.ron2 = (T)(ron * ron);
    w.ron = (T)ron;
    w.roff2 = (T)(roff * roff);
    w.roff = (T)roff;
    w.inv_range = roff < rc ? (T)(1.0 / (roff - rc)) : (T)0;  // empty falling part
    w.inv_in = (T)(1.0 / (roff - ron));
    for (int j = 0; j <= n; j++) w.vcoef[j] = (T)binomial(2 * n + 1, n + 1 + j);
    w.dpeak = (T)kCnDeriv[n - 2][0];
  }
  return w;
}

// The grid of LennardJonesTableForce<S, 7, double>(swf): LookupTable's
// construction (protomol/src/protomol/force/table/LookupTable.h:71-158) with
// LennardJonesLookupValues::assign (LennardJonesTableForce.h:24-34).  Grid
// points run over r^2 from lowerboundExp2(0.1) = 1/16, 128 per octave, up to
// the octave holding the switch's cutoff^2; point p holds, for the switched
// r^-12 part (A) and the switched -r^-6 part (B), the value, its derivative
// in r^2 and the cubic Hermite coefficients c, d of the interval starting at
// p (refined twice against the next point, as the reference does).  Output:
// two double4 per point ({v, g, c, d} of A, then of B); first = the biased
// exponent-and-top-mantissa hash of 1/16; last = the final point's index.
void build_lj_table(const SwitchSpec<double> &w, std::vector<double4> &tab, int &first,
                    int &last) {
  auto bits = [](double x) {
    long long b;
    std::memcpy(&b, &x, sizeof b);
    return b;
  };
  auto lb2 = [](double r) {  // MathUtilities.cpp:52-61
    double res = 1.0;
    while (res < r) res *= 2.0;
    while (res > r) res /= 2.0;
    return res;
  };
  constexpr int kN = 1 << kTabPre;
  const double lo = lb2(0.1);
  const int octaves = (int)((bits(lb2(w.rc2)) >> 52) + 1 - (bits(lo) >> 52));
  const int npt = octaves * kN + 1;
  first = (int)(bits(lo) >> kTabShift);
  last = octaves * kN;
  std::vector<double> t((size_t)8 * npt, 0.0);
  for (int i = 0; i < npt; i++) {
    const double base = lo * (double)(1 << (i / kN));
    const double del = base / (double)kN;
    const double r = base + del * (double)(i % kN);
    const double r1 = std::sqrt(r);
    double v, d;
    switch_eval(w, r, 1.0 / r1, v, d);
    // powers of 1/r1 by squaring, in the order MathUtilities.h:79-90 uses
    const double ip = 1.0 / r1;
    const double p3 = (ip * ip) * ip, p6 = p3 * p3, p4 = (ip * ip) * (ip * ip);
    const double p7 = p6 * ip;
    double *e = &t[(size_t)8 * i];
    double ev = p6 * p6, fv = 12.0 * (p7 * p7);
    e[0] = ev * v;
    e[1] = -0.5 * (fv * v - ev * d);
    ev = -p6;
    fv = -6.0 * (p4 * p4);
    e[4] = ev * v;
    e[5] = -0.5 * (fv * v - ev * d);
    if (i == 0) continue;
    const double x = lo * (double)(1 << ((i - 1) / kN)) / (double)kN;
    double *pr = &t[(size_t)8 * (i - 1)];
    for (int j = 0; j < 8; j += 4) {
      const double v1 = pr[j], g1 = pr[j + 1], v2 = e[j], g2 = e[j + 1];
      double c = (3.0 * (v2 - v1) - x * (2.0 * g1 + g2)) / (x * x);
      double dd = (-2.0 * (v2 - v1) + x * (g1 + g2)) / (x * x * x);
      for (int k = 0; k < 2; k++) {
        const double dv = (v1 - v2) + ((dd * x + c) * x + g1) * x;
        const double dg = (g1 - g2) + (3.0 * dd * x + 2.0 * c) * x;
        c -= (3.0 * dv - x * dg) / (x * x);
        dd -= (-2.0 * dv + x * dg) / (x * x * x);
      }
      pr[j + 2] = c;
      pr[j + 3] = dd;
    }
  }
  tab.resize((size_t)2 * npt);
  for (int i = 0; i < 2 * npt; i++)
    tab[i] = make_double4(t[4 * i], t[4 * i + 1], t[4 * i + 2], t[4 * i + 3]);
}

// NonbondedFullEwaldSystemForce::initialize
// (protomol/src/protomol/force/nonbonded/NonbondedFullEwaldSystemForce.h:
// 586-598): alpha (default sqrt(pi) (5.5 N / V^2)^(1/6), V = |(e1 x e2) . e3|)
// and rc = sqrt(-log(accuracy)) / alpha.
void ewald_derive(pmb200_ctx *c, double volume) {
  double alpha = c->ew_alpha_in;
  if (alpha <= 0.0) {
    const double v = volume;
    alpha = std::sqrt(M_PI) * std::pow(5.5 * (unsigned)c->n / (v * v), 1.0 / 6.0);
  }
  c->ew_alpha = alpha;
  c->ew_rc = std::sqrt(-std::log(c->ew_accuracy)) / alpha;
}

// The host copy of the LJ table, brought up to date after a device-side
// update (for the rare host consumers: box changes, batch creation).
int pull_lj(pmb200_ctx *c) {
  if (!c->lj_dev_newer) return PMB200_OK;
  CK(cudaEventSynchronize(c->ev_lj));
  const size_t t2 = (size_t)c->ntypes * c->ntypes;
  CK(cudaMemcpy(c->h_lj.data(), c->d_lj64, sizeof(double4) * t2, cudaMemcpyDeviceToHost));
  c->lj_dev_newer = false;
  return PMB200_OK;
}

// LJ tables: FP64 in Angstrom units, FP32 in cell units (A / u^12, B / u^6).
int upload_lj(pmb200_ctx *c) {
  int rc = pull_lj(c);
  if (rc) return rc;
  const int t2 = c->ntypes * c->ntypes;
  std::vector<double4> l64(t2);
  std::vector<float4> l32(t2);
  const double u = c->g.unit;
  const double u6 = std::pow(u, 6.0), u12 = u6 * u6;
  for (int k = 0; k < t2; k++) {
    const double *p = &c->h_lj[4 * k];
    l64[k] = make_double4(p[0], p[1], p[2], p[3]);
    l32[k] = make_float4((float)(p[0] / u12), (float)(p[1] / u6), (float)(p[2] / u12),
                         (float)(p[3] / u6));
  }
  CK(cudaMemcpyAsync(c->d_lj64, l64.data(), sizeof(double4) * t2, cudaMemcpyHostToDevice,
                     c->stream));
  CK(cudaMemcpyAsync(c->d_lj32, l32.data(), sizeof(float4) * t2, cudaMemcpyHostToDevice,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PMB200_OK;
}

int ensure_atom_buffers(pmb200_ctx *c) {
  if (c->n_alloc >= c->n && c->d_cell_of) return PMB200_OK;
  const size_t n = (size_t)std::max(c->n, 1);
  CK(dalloc(c->d_cell_of, n));
  CK(dalloc(c->d_slot, n));
  CK(dalloc(c->d_tmp, n));
  CK(dalloc(c->d_sidx, n));
  CK(dalloc(c->d_rel32, n));
  CK(dalloc(c->d_spos32, n));
  CK(dalloc(c->d_rel_lo, n));
  CK(dalloc(c->d_spos_lo, n));
  CK(dalloc(c->d_rel64, n));
  CK(dalloc(c->d_spos64, n));
  CK(dalloc(c->d_smeta, n));
  CK(dalloc(c->d_facc, 8 * n));  // FP64 forces: 6 words per atom; derivatives: 8
  CK(dalloc(c->d_cblo, n));
  CK(dalloc(c->d_cbhi, n));
  CK(dalloc(c->d_hpos, 3 * n));
  CK(dalloc(c->d_hfrc, 3 * n + kPinOut + 3));  // forces, then the results (pmb200_eval)
  CK(dalloc(c->d_hf32, 3 * n + 2 + 2 * (kPinOut + 3)));  // FP32 forces, then the results
  c->n_alloc = c->n;
  return PMB200_OK;
}

// Launches kernel k on st; pdl: as a programmatic dependent of the kernel
// launched just before it on st (k calls pdl_wait before it touches that
// kernel's data), so that its launch overlaps the predecessor's tail.
template <class... Exp, class... Act>
void launch_k(void (*k)(Exp...), unsigned grid, unsigned block, size_t smem, cudaStream_t st,
              bool pdl, Act &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = (pdl && PMB200_PDL) ? 1 : 0;
  cudaLaunchKernelEx(&cfg, k, std::forward<Act>(args)...);
}

// The pair kernels for the flags asked for (template instances per form),
// over the i-cells [cell0, cell0 + ncells) (all by default) into the fixed-
// point accumulator facc (the context's by default).
// pdl: the previous operation on `st` is the cell build's last kernel; the
// pair kernel is then launched as its programmatic dependent, so that its
// launch and prologue overlap that kernel's tail (it waits for it before
// reading the sorted atoms).
template <int F>
void launch_pair_mixed(pmb200_ctx *c, unsigned flags, cudaStream_t st, int cell0 = 0,
                       int ncells = -1, unsigned long long *facc = nullptr, bool pdl = false) {
  const GridParams &g = c->g;
  if (ncells < 0) ncells = g.ncell;
  if (!facc) facc = c->d_facc;
  const bool energy = (flags & PMB200_ENERGY) != 0;
  const bool virial = (flags & (PMB200_VIRIAL | PMB200_MOLVIRIAL)) != 0;
  const bool molvir = (flags & PMB200_MOLVIRIAL) != 0;
  const size_t smem = mixed_smem_bytes(F, c->ntypes, c->half.ncells);
  const int slots = ctx_slots(c, energy || virial);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(std::max(ncells, 1) * slots));
  cfg.blockDim = dim3(32);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = (pdl && PMB200_PDL) ? 1 : 0;
  // tables of more than kMaxTypes types are read through L1 (forms with LJ)
  constexpr bool kLjForm = F == FORM_CUTOFF || F == FORM_GENERIC;
  const bool big = kLjForm && c->ntypes > kMaxTypes;
#define PMB_MIXED_LAUNCH(E, V, M, G)                                                       \
  cudaLaunchKernelEx(&cfg, k_pair_mixed<F, E, V, M, G>, g, c->mc, c->half, c->ntypes,      \
                     c->d_lj32, c->d_start, c->d_spos32, c->d_smeta, c->d_sidx,             \
                     c->d_ex_start, c->d_ex, facc, c->n, c->d_err, c->d_partial, c->pb,     \
                     c->d_com, slots, c->d_spos_lo, ncells > 0 ? cell0 : g.ncell)
#define PMB_MIXED_FLAGS(G)                                                                 \
  if (molvir) PMB_MIXED_LAUNCH(true, true, true, G);                                       \
  else if (energy && virial) PMB_MIXED_LAUNCH(true, true, false, G);                       \
  else if (energy) PMB_MIXED_LAUNCH(true, false, false, G);                                \
  else if (virial) PMB_MIXED_LAUNCH(false, true, false, G);                                \
  else PMB_MIXED_LAUNCH(false, false, false, G)
  if (!big) {
    PMB_MIXED_FLAGS(false);
  } else if constexpr (kLjForm) {
    PMB_MIXED_FLAGS(true);
  }
#undef PMB_MIXED_FLAGS
#undef PMB_MIXED_LAUNCH
}

// Whether an evaluation with these flags runs on the cluster-pair kernel:
// the context asked for it, mixed precision, the cutoff or real-space Ewald
// form with its LJ table in shared memory, no virial, an orthogonal grid.
bool tiles_apply(const pmb200_ctx *c, unsigned flags) {
  return ((flags & PMB200_ENERGY) ? c->tiles_e : c->tiles_f) && c->p.precision == PMB200_MIXED &&
         (c->form == FORM_CUTOFF || c->form == FORM_EWALD_POLY5 || c->form == FORM_EWALD_EXACT) &&
         !(flags & (PMB200_VIRIAL | PMB200_MOLVIRIAL)) && c->ntypes <= kMaxTypes && !c->g.tric &&
         c->n < (1 << 29);
}

// The cluster boxes and the cluster-pair kernel (see pmb200_tiles.cuh), as
// programmatic dependents of the cell build when pdl.
template <int F>
void launch_pair_tiles(pmb200_ctx *c, unsigned flags, cudaStream_t st, bool pdl) {
  const GridParams &g = c->g;
  const bool energy = (flags & PMB200_ENERGY) != 0;
  const int slots = ctx_slots(c, energy);
  launch_k(k_cluster_boxes, (unsigned)((g.ncell + 3) / 4), 128, 0, st, pdl, g.ncell,
           (const int *)c->d_start, (const float4 *)c->d_spos32, c->d_cblo, c->d_cbhi);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(std::max(g.ncell, 1) * slots));
  cfg.blockDim = dim3(32);
  cfg.dynamicSmemBytes = mixed_smem_bytes(F, c->ntypes, c->half.ncells);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = (pdl && PMB200_PDL) ? 1 : 0;
#define PMB_TILES_LAUNCH(E)                                                                \
  cudaLaunchKernelEx(&cfg, k_pair_tiles<F, E>, g, c->mc, c->half, c->ntypes, c->d_lj32,      \
                     c->d_start, c->d_spos32, c->d_smeta, c->d_sidx, c->d_ex_start, c->d_ex,  \
                     c->d_cblo, c->d_cbhi, c->d_facc, c->n, c->d_err, c->d_partial, slots,   \
                     c->d_spos_lo)
  if (energy) PMB_TILES_LAUNCH(true);
  else PMB_TILES_LAUNCH(false);
#undef PMB_TILES_LAUNCH
}

// (over the i-cells [cell0, cell0 + ncells), all by default)
template <int F>
void launch_pair_fp64(pmb200_ctx *c, unsigned flags, double *d_forces, int accumulate,
                      int blocks, cudaStream_t st, int cell0 = 0, int ncells = 1 << 30) {
  const GridParams &g = c->g;
  const bool energy = (flags & PMB200_ENERGY) != 0;
  const bool virial = (flags & (PMB200_VIRIAL | PMB200_MOLVIRIAL)) != 0;
  const bool molvir = (flags & PMB200_MOLVIRIAL) != 0;
#define PMB_FP64_LAUNCH(E, V, M)                                                           \
  k_pair_fp64<F, E, V, M><<<blocks, 128, 0, st>>>(g, c->fc, c->stencil, c->ntypes,          \
                                                  c->d_lj64, c->d_start, c->d_spos64,       \
                                                  c->d_smeta, c->d_sidx, c->d_ex_start,     \
                                                  c->d_ex, d_forces, accumulate,            \
                                                  c->d_partial, c->pb, c->d_com, cell0,     \
                                                  ncells)
  if (molvir) PMB_FP64_LAUNCH(true, true, true);
  else if (energy && virial) PMB_FP64_LAUNCH(true, true, false);
  else if (energy) PMB_FP64_LAUNCH(true, false, false);
  else if (virial) PMB_FP64_LAUNCH(false, true, false);
  else PMB_FP64_LAUNCH(false, false, false);
#undef PMB_FP64_LAUNCH
}

// The FP64 evaluation kernel (half shell, kFp64Slots warps per i-cell) into
// the sorted-order accumulator d_facc (two-word fixed point, cleared by the
// cell build).
constexpr int kFp64Slots = kEnergyCellSlots;
template <int F>
void launch_pair_fp64_half(pmb200_ctx *c, unsigned flags, cudaStream_t st) {
  const GridParams &g = c->g;
  const bool energy = (flags & PMB200_ENERGY) != 0;
  const bool virial = (flags & (PMB200_VIRIAL | PMB200_MOLVIRIAL)) != 0;
  const bool molvir = (flags & PMB200_MOLVIRIAL) != 0;
  const unsigned blocks = (unsigned)g.ncell * kFp64Slots;
  if (blocks == 0) return;
#define PMB_FP64H_LAUNCH(E, V, M)                                                          \
  k_pair_fp64_half<F, E, V, M><<<blocks, 32, 0, st>>>(                                    \
      g, c->fc, c->half, kFp64Slots, c->ntypes, c->d_lj64, c->d_start, c->d_spos64,         \
      c->d_smeta, c->d_sidx, c->d_ex_start, c->d_ex, c->d_facc, c->n, c->d_partial, c->pb,  \
      c->d_com, c->d_err)
  if (molvir) PMB_FP64H_LAUNCH(true, true, true);
  else if (energy && virial) PMB_FP64H_LAUNCH(true, true, false);
  else if (energy) PMB_FP64H_LAUNCH(true, false, false);
  else if (virial) PMB_FP64H_LAUNCH(false, true, false);
  else PMB_FP64H_LAUNCH(false, false, false);
#undef PMB_FP64H_LAUNCH
}

// Zeroes d_count when a launch sequence broke off after using it; a captured
// graph relies on its previous run having left it cleared.
int ensure_clear(pmb200_ctx *c, cudaStream_t st) {
  if (!c->count_zero && c->d_count && c->g.ncell > 0) {
    CK(cudaMemsetAsync(c->d_count, 0, sizeof(int) * (size_t)c->g.ncell, st));
    c->count_zero = true;
  }
  return PMB200_OK;
}

// Neighbour-cell stencils of the current grid for the cutoff rc: rows (dy,
// dz) with their dx span (full shell) and the half shell by cell (offsets
// with dz > 0, or dz == 0 and dy > 0, or dz == dy == 0 and dx >= 0; dx == 0
// is the home cell, pairs i < j) in a fixed pseudo-random order --
// consecutive cells of a warp's share then lie in different directions, so
// each staged batch holds a similar number of partners for every i atom.
// Orthogonal grid: every cell whose nearest point can lie within rc of the
// home cell.  General cell: every offset up to ceil(rc n_k / width_k) cells
// along each basis vector (the fractional extent of the cutoff sphere).
int build_stencils(pmb200_ctx *c, double rc, std::vector<Row> &rows, HalfStencil &half) {
  const GridParams &g = c->g;
  rows.clear();
  if (g.tric) {
    int R[3];
    for (int k = 0; k < 3; k++) R[k] = (int)std::ceil(rc / g.edge[k] - 1e-12);
    for (int dz = -R[2]; dz <= R[2]; dz++)
      for (int dy = -R[1]; dy <= R[1]; dy++) rows.push_back(Row{dy, dz, -R[0], R[0]});
  } else {
    int R[3];
    for (int a = 0; a < 3; a++) R[a] = (int)std::ceil(rc / g.edge[a] - 1e-12);
    const double rc2 = rc * rc * (1.0 + 1e-12);
    for (int dz = -R[2]; dz <= R[2]; dz++)
      for (int dy = -R[1]; dy <= R[1]; dy++) {
        const double yz = std::pow(std::max(std::abs(dy) - 1, 0) * g.edge[1], 2) +
                          std::pow(std::max(std::abs(dz) - 1, 0) * g.edge[2], 2);
        if (yz > rc2) continue;
        int hi = 0;
        for (int dx = 0; dx <= R[0]; dx++)
          if (yz + std::pow(std::max(dx - 1, 0) * g.edge[0], 2) <= rc2) hi = dx;
        rows.push_back(Row{dy, dz, -hi, hi});
      }
  }
  if ((int)rows.size() > kMaxRows)
    return fail(c, PMB200_EUNSUPPORTED, "stencil of %d rows (cell size too small)",
                (int)rows.size());
  half = HalfStencil{};
  for (const Row &rw : rows)
    for (int dx = rw.dxlo; dx <= rw.dxhi; dx++) {
      const bool keep = rw.dz > 0 || (rw.dz == 0 && rw.dy > 0) ||
                        (rw.dz == 0 && rw.dy == 0 && dx >= 0);
      if (!keep) continue;
      if (half.ncells >= kMaxHalfCells || std::abs(dx) > 8 || std::abs(rw.dy) > 8 ||
          std::abs(rw.dz) > 8)
        return fail(c, PMB200_EUNSUPPORTED, "neighbour stencil too large (cell size too small)");
      half.off[half.ncells++] =
          (unsigned short)((dx + 8) | ((rw.dy + 8) << 5) | ((rw.dz + 8) << 10));
    }
  unsigned long long x = 0x9E3779B97F4A7C15ull;
  for (int k = half.ncells - 1; k > 0; k--) {
    x = x * 6364136223846793005ull + 1442695040888963407ull;
    const int j = (int)((x >> 33) % (unsigned long long)(k + 1));
    std::swap(half.off[k], half.off[j]);
  }
  return PMB200_OK;
}

// Launch one evaluation on `st`.  accumulate: add into d_forces (1) or
// overwrite it (0).
// Counting sort of the atoms into the grid cells (cell index, scan,
// scatter, in-cell rank order), producing the cell-unit FP32 copies (mixed)
// or the Angstrom FP64 copies of the sorted positions; lo: also the FP32
// coordinates' rounding residuals (energy evaluations of the cutoff form).
// clear: an accumulator of nclear x n entries the build zeroes on the way
// (or null).
// After the first kernel each one is launched as a programmatic dependent of
// the one before it.
void launch_cell_build(pmb200_ctx *c, const double *d_pos, bool mixed, bool lo,
                       cudaStream_t st, unsigned long long *clear = nullptr, int nclear = 3) {
  const int n = c->n;
  const GridParams &g = c->g;
  if (!c->count_zero) cudaMemsetAsync(c->d_count, 0, sizeof(int) * g.ncell, st);
  c->count_zero = false;
  const unsigned nb = (unsigned)((n + 255) / 256);
  if (n > 0)
    launch_k(k_cell_index, nb, 256, 0, st, false, n, d_pos, g, c->d_cell_of, c->d_count,
             c->d_slot, mixed ? c->d_rel32 : nullptr, mixed ? nullptr : c->d_rel64, c->d_q,
             (float)(1.0 / std::sqrt(g.unit)), c->d_err, lo ? c->d_rel_lo : nullptr, clear,
             nclear);
  launch_k(k_scan, 1, 1024, 1024 * sizeof(int), st, n > 0, g.ncell, c->d_count, c->d_start);
  c->count_zero = cudaPeekAtLastError() == cudaSuccess;
  if (n > 0)
    launch_k(k_scatter, nb, 256, 0, st, true, n, c->d_cell_of, c->d_slot, c->d_start,
             c->d_tmp);
  launch_k(k_rank_gather, (unsigned)((g.ncell + 3) / 4), 128, 0, st, true, g.ncell,
           c->d_start, c->d_tmp, mixed ? c->d_rel32 : nullptr, mixed ? nullptr : c->d_rel64,
           c->d_type, c->d_mol, c->d_sidx, mixed ? c->d_spos32 : nullptr,
           mixed ? nullptr : c->d_spos64, c->d_smeta, lo ? c->d_rel_lo : nullptr,
           lo ? c->d_spos_lo : nullptr, (mixed && (c->tiles_e || c->tiles_f)) ? 1 : 0);
}

// One word copied on the device (the error flag into the results' copy).
__global__ void k_copy_word(const int *__restrict__ src, int *__restrict__ dst) { *dst = *src; }

// Host-buffer calls of mixed contexts read the forces back in FP32 (the
// mixed kernels' forces are good to ~1e-6; FP32 keeps 6e-8 of each, and the
// copy is half as long), then the result words.  (Sending the positions as
// 32-bit box fractions was measured too: the host's encoding pass cost what
// the shorter copy saved.)
__global__ void k_pack_out(size_t n3, const double *__restrict__ frc,
                           const double *__restrict__ res, const int *__restrict__ err,
                           float *__restrict__ out) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n3) out[k] = (float)frc[k];
  // the 20 result words and the device error flag behind them, after the
  // forces at a double boundary
  double *tail = reinterpret_cast<double *>(out + ((n3 + 1) & ~(size_t)1));
  if (k < 20) tail[k] = res[k];
  else if (k == 20) *reinterpret_cast<int *>(tail + 20) = *err;
}

// The supercluster kernel's grid, stencil, constants and buffers for the
// current box and topology (sc_ok = false where it does not apply: the
// other kernels then run).  Called when the box, the topology or the pair
// kernel choice changes.
int sc_prepare(pmb200_ctx *c) {
  c->sc_ok = false;
  if (!(c->clu_e || c->clu_f) || !c->have_box || !c->have_topo) return PMB200_OK;
  if (c->p.precision != PMB200_MIXED || c->form != FORM_CUTOFF || c->g.tric || c->vacuum ||
      c->ntypes > kMaxTypes || c->has_modified || c->n <= 0 || c->n >= (1 << 24))
    return PMB200_OK;
  const GridParams &gp = c->g;
  const double rc = ctx_rc(c);
  const double rlist = rc * (1.0 + 1e-5) + 1e-3;  // box tests with a margin
  ScGrid g{};
  double vol = 1.0;
  for (int a = 0; a < 3; a++) {
    g.boxmin[a] = gp.boxmin[a];
    g.boxlen[a] = gp.boxlen[a];
    g.L[a] = (float)gp.boxlen[a];
    vol *= gp.boxlen[a];
    // a lattice of about 3 A whose step divides the edge
    g.m[a] = std::max(1, (int)std::lround(gp.boxlen[a] / 3.0));
    g.h[a] = gp.boxlen[a] / g.m[a];
    g.hf[a] = (float)g.h[a];
  }
  // columns about the edge of a cube holding 32 atoms; slabs of about 1 A
  const double side = c->sc_side * std::cbrt(kScAtoms * vol / c->n);
  int ns[2];
  for (int a = 0; a < 2; a++) {
    ns[a] = std::max(1, (int)std::lround(gp.boxlen[a] / side));
    g.colw[a] = gp.boxlen[a] / ns[a];
    const int R = (int)std::ceil(rlist / g.colw[a]);
    if (ns[a] < 2 * R + 1) return PMB200_OK;  // columns must be distinct images
  }
  g.nsx = ns[0];
  g.nsy = ns[1];
  g.ncol = ns[0] * ns[1];
  g.nsz = std::max(1, (int)std::lround(gp.boxlen[2] / 1.0));
  g.slabw = gp.boxlen[2] / g.nsz;
  g.zmax_ext = (float)(0.5 * (gp.boxlen[2] - 2.0 * rlist) - 0.01);
  if (g.zmax_ext < 2.0f) return PMB200_OK;
  const long long ncell = (long long)g.ncol * g.nsz;
  if (ncell > (1 << 24)) return PMB200_OK;
  g.nsup_max = (c->n + kScAtoms - 1) / kScAtoms + g.ncol;
  g.nslot_max = g.nsup_max * kScAtoms;
  g.rlist2 = (float)(rlist * rlist);
  ScStencil st{};
  const int R0 = (int)std::ceil(rlist / g.colw[0]), R1 = (int)std::ceil(rlist / g.colw[1]);
  for (int dx = -R0; dx <= R0; dx++)
    for (int dy = -R1; dy <= R1; dy++) {
      const double gx = std::max(std::abs(dx) - 1, 0) * g.colw[0];
      const double gy = std::max(std::abs(dy) - 1, 0) * g.colw[1];
      if (gx * gx + gy * gy >= rlist * rlist) continue;
      if (st.n >= kScMaxCols) return PMB200_OK;
      st.off[st.n++] = make_short2((short)dx, (short)dy);
    }
  // buffers
  if (c->sc_ncell_alloc < (int)ncell) {
    CK(dalloc(c->d_sc_count, (size_t)ncell));
    CK(dalloc(c->d_sc_start, (size_t)ncell + 1));
    c->sc_ncell_alloc = (int)ncell;
  }
  CK(cudaMemset(c->d_sc_count, 0, sizeof(int) * (size_t)ncell));
  c->sc_count_zero = true;
  if (c->sc_ncol_alloc < g.ncol) {
    CK(dalloc(c->d_sc_supbase, (size_t)g.ncol + 1));
    c->sc_ncol_alloc = g.ncol;
  }
  if (!c->d_sc_ctl) CK(dalloc(c->d_sc_ctl, 4));
  if (c->sc_nsup_alloc < g.nsup_max) {
    const size_t ns_ = (size_t)g.nsup_max, nsl = ns_ * kScAtoms, ncl = ns_ * 8;
    const size_t ntask = ns_ * ((kScCap + kScChunk - 1) / kScChunk);
    CK(dalloc(c->d_sc_atom, nsl));
    CK(dalloc(c->d_sc_type, nsl));
    CK(dalloc(c->d_sc_mol, nsl));
    CK(dalloc(c->d_sc_xi, nsl));
    CK(dalloc(c->d_sc_xj, nsl));
    CK(dalloc(c->d_sc_xilo, nsl));
    CK(dalloc(c->d_sc_xjlo, nsl));
    CK(dalloc(c->d_sc_facc, 3 * nsl));
    CK(dalloc(c->d_sc_clo, ncl));
    CK(dalloc(c->d_sc_chi, ncl));
    CK(dalloc(c->d_sc_corg, ncl));
    CK(dalloc(c->d_sc_cmol, ncl));
    CK(dalloc(c->d_sc_sorg, ns_));
    CK(dalloc(c->d_sc_sbox, 2 * ns_));
    CK(dalloc(c->d_sc_cnt, ns_));
    CK(dalloc(c->d_sc_ent, ns_ * kScCap));
    CK(dalloc(c->d_sc_tasks, ntask));
    CK(dalloc(c->d_sc_part, ntask * kNacc));
    c->sc_nsup_alloc = g.nsup_max;
  }
  // the pair constants in A (the search kernel's, with unit 1)
  const pmb200_params &p = c->p;
  MixedConsts m = c->mc;
  {
    const double rl = p.cutoff_lj, ro = p.switchon, rq = p.cutoff_coul;
    const double t = rl * rl - ro * ro;
    m.cut2 = (float)(rc * rc);
    m.rclj2 = (float)(rl * rl);
    m.ron2 = (float)(ro * ro);
    m.rcc2 = (float)(rq * rq);
    m.s1 = (float)(1.0 / (t * t * t));
    m.s2 = (float)(rl * rl - 3.0 * ro * ro);
    m.s3 = (float)(4.0 / (t * t * t));
    m.c15_1 = (float)(1.5 / rq);
    m.c05_3 = (float)(0.5 / (rq * rq * rq));
    m.c15_3 = (float)(1.5 / (rq * rq * rq));
    m.e15 = 1.5 / rq;
    m.e05 = 0.5 / (rq * rq * rq);
  }
  int dev = 0, sms = 0, be = 0, bf = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const bool full = m.rclj2 >= m.cut2 && m.rcc2 >= m.cut2;
  if (full) {
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&be, k_sc_pair<true, true>, 32, 0));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bf, k_sc_pair<false, true>, 32, 0));
  } else {
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&be, k_sc_pair<true, false>, 32, 0));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bf, k_sc_pair<false, false>, 32, 0));
  }
  c->sc_full = full;
  c->sc_grid_e = sms * std::max(be, 1);
  c->sc_grid_f = sms * std::max(bf, 1);
  c->sg = g;
  c->sst = st;
  c->mca = m;
  c->sc_ok = true;
  release_graph(c);
  return PMB200_OK;
}

bool clusters_apply(const pmb200_ctx *c, unsigned flags) {
  return c->sc_ok && ((flags & PMB200_ENERGY) ? c->clu_e : c->clu_f) &&
         !(flags & (PMB200_VIRIAL | PMB200_MOLVIRIAL));
}

// One evaluation on the supercluster kernel: column sort, superclusters,
// lists, tasks, pair kernel, forces back to the original order, energies.
// Every kernel after the first is a programmatic dependent of the one before
// (except a timed pair kernel, whose events bracket it alone).
int launch_eval_clusters(pmb200_ctx *c, const double *d_pos, double *d_forces, double *d_out,
                         unsigned flags, int accumulate, cudaStream_t st, bool timed) {
  const int n = c->n;
  const ScGrid &g = c->sg;
  const bool energy = (flags & PMB200_ENERGY) != 0;
  const int ncell = g.ncol * g.nsz;
  // every kernel after the first as a programmatic dependent of the one
  // before it (the kernels read the counts their predecessors write through
  // volatile loads after their wait: sc_ctl)
  constexpr bool kChain = true;
  if (!c->sc_count_zero) cudaMemsetAsync(c->d_sc_count, 0, sizeof(int) * (size_t)ncell, st);
  c->sc_count_zero = false;
  const unsigned nb = (unsigned)((n + 255) / 256);
  launch_k(k_sc_index, nb, 256, 0, st, false, n, d_pos, g, c->d_cell_of, c->d_sc_count,
           c->d_slot, c->d_err);
  launch_k(k_scan, 1, 1024, 1024 * sizeof(int), st, kChain, ncell, c->d_sc_count, c->d_sc_start);
  c->sc_count_zero = cudaPeekAtLastError() == cudaSuccess;
  launch_k(k_scatter, nb, 256, 0, st, kChain, n, c->d_cell_of, c->d_slot, c->d_sc_start,
           c->d_tmp);
  launch_k(k_rank_gather, (unsigned)((ncell + 3) / 4), 128, 0, st, kChain, ncell, c->d_sc_start,
           c->d_tmp, (const float4 *)nullptr, (const double4 *)nullptr, c->d_type, c->d_mol,
           c->d_sidx, (float4 *)nullptr, (double4 *)nullptr, c->d_smeta,
           (const float4 *)nullptr, (float4 *)nullptr, 0);
  launch_k(k_sc_columns, 1, 1024, 0, st, kChain, g.ncol, g.nsz, c->d_sc_start, c->d_sc_supbase,
           c->d_sc_ctl);
  launch_k(k_sc_build, (unsigned)((g.nsup_max + kScBuildWarps - 1) / kScBuildWarps),
           32 * kScBuildWarps, 0, st, kChain, g, d_pos, c->d_sc_start, c->d_sidx, c->d_smeta,
           c->d_sc_supbase, c->d_sc_ctl, c->d_q, c->d_sc_atom, c->d_sc_type, c->d_sc_mol,
           c->d_sc_xi, c->d_sc_xj, energy ? c->d_sc_xilo : nullptr,
           energy ? c->d_sc_xjlo : nullptr, c->d_sc_clo, c->d_sc_chi, c->d_sc_corg,
           c->d_sc_cmol, c->d_sc_sorg, c->d_sc_sbox, c->d_sc_facc, c->d_err);
  launch_k(k_sc_list, (unsigned)g.nsup_max, 32 * kScListWarps, kScListSmem, st, kChain, g,
           c->sst, c->d_sc_supbase,
           c->d_sc_ctl, c->d_sc_clo, c->d_sc_chi, c->d_sc_corg, c->d_sc_cmol, c->d_sc_sorg,
           c->d_sc_sbox, c->d_sc_atom, c->d_sc_mol, c->d_ex_start, c->d_ex, c->d_sc_ent,
           c->d_sc_cnt, c->d_err);
  launch_k(k_sc_tasks, 1, 1024, 0, st, kChain, c->d_sc_cnt, c->d_sc_ctl, c->d_sc_tasks);
  CK(cudaGetLastError());
  if (timed) CK(cudaEventRecord(c->ev0, st));
  const bool pdl = !timed && kChain;
#define PMB_SC_PAIR(E, F)                                                                   \
  launch_k(k_sc_pair<E, F>, (unsigned)(E ? c->sc_grid_e : c->sc_grid_f), 32, 0, st, pdl,     \
           c->mca, c->ntypes, c->d_lj64, c->d_sc_tasks, c->d_sc_ctl, c->d_sc_xi, c->d_sc_xj, \
           c->d_sc_type, c->d_sc_ent, c->d_sc_xilo, c->d_sc_xjlo, g, c->d_sc_facc,           \
           c->d_sc_part, c->d_err)
  if (energy && c->sc_full) PMB_SC_PAIR(true, true);
  else if (energy) PMB_SC_PAIR(true, false);
  else if (c->sc_full) PMB_SC_PAIR(false, true);
  else PMB_SC_PAIR(false, false);
#undef PMB_SC_PAIR
  CK(cudaGetLastError());
  if (timed) CK(cudaEventRecord(c->ev1, st));
  launch_k(k_sc_finalize, (unsigned)((g.nslot_max + 255) / 256), 256, 0, st, pdl,
           (const int *)c->d_sc_ctl, g.nslot_max, (const int *)c->d_sc_atom,
           (const unsigned long long *)c->d_sc_facc, accumulate, d_forces);
  if (energy) {
    k_sc_reduce1<<<kRedBlocks, 256, 0, st>>>(c->d_sc_ctl + 1, c->d_sc_part, c->d_red, ACC_E);
    k_reduce2<<<1, 256, 0, st>>>(kRedBlocks, c->d_red, 1.0, d_out ? d_out : c->d_out,
                                c->d_pairs, ACC_E);
  }
  CK(cudaGetLastError());
  return PMB200_OK;
}

// f32 / tail (host-buffer calls of mixed contexts, or null): where the
// evaluation may put its forces in FP32 and the results with the error flag
// (k_finalize_reduce); *packed tells whether it did.
int launch_eval(pmb200_ctx *c, const double *d_pos, double *d_forces, double *d_out,
                unsigned flags, int accumulate, cudaStream_t st, float *f32 = nullptr,
                double *tail = nullptr, bool *packed = nullptr) {
  if (packed) *packed = false;
  const int n = c->n;
  const bool mixed = c->p.precision == PMB200_MIXED;
  const bool energy = (flags & PMB200_ENERGY) != 0;
  const bool virial = (flags & (PMB200_VIRIAL | PMB200_MOLVIRIAL)) != 0;
  const bool molvir = (flags & PMB200_MOLVIRIAL) != 0;
  const GridParams &g = c->g;
  if (mixed && clusters_apply(c, flags)) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(st, &cs));
    return launch_eval_clusters(c, d_pos, d_forces, d_out, flags, accumulate, st,
                                c->timing && cs == cudaStreamCaptureStatusNone);
  }
  // the cell build clears the accumulator on the way (still in L2 when the
  // pair kernel adds to it), so that the pair kernel follows the build's last
  // kernel directly
  launch_cell_build(c, d_pos, mixed, mixed && energy && c->form == FORM_CUTOFF, st, c->d_facc,
                    mixed ? 3 : 6);
  CK(cudaGetLastError());
  if (molvir && c->nmol > 0)
    k_com<<<(c->nmol + 127) / 128, 128, 0, st>>>(c->nmol, c->d_mstart, c->d_matoms, c->d_mass,
                                                  d_pos, c->d_com);
  // pair-kernel timing events are recorded on direct launches only (not
  // inside a stream capture)
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(st, &cap));
  const bool timed = c->timing && cap == cudaStreamCaptureStatusNone;
  if (timed) CK(cudaEventRecord(c->ev0, st));
  if (mixed) {
    const double fscale = 1.0 / g.unit;
    // (a programmatic dependent of the cell build's last kernel, except in
    // timed launches, whose events bracket the pair kernel alone)
    const bool pdl = !timed;
    if (tiles_apply(c, flags)) {
      if (c->form == FORM_EWALD_POLY5) launch_pair_tiles<FORM_EWALD_POLY5>(c, flags, st, pdl);
      else if (c->form == FORM_EWALD_EXACT) launch_pair_tiles<FORM_EWALD_EXACT>(c, flags, st, pdl);
      else launch_pair_tiles<FORM_CUTOFF>(c, flags, st, pdl);
    } else if (c->form == FORM_GENERIC)
      launch_pair_mixed<FORM_GENERIC>(c, flags, st, 0, -1, nullptr, pdl);
    else if (c->form == FORM_EWALD_POLY5)
      launch_pair_mixed<FORM_EWALD_POLY5>(c, flags, st, 0, -1, nullptr, pdl);
    else if (c->form == FORM_EWALD_EXACT)
      launch_pair_mixed<FORM_EWALD_EXACT>(c, flags, st, 0, -1, nullptr, pdl);
    else launch_pair_mixed<FORM_CUTOFF>(c, flags, st, 0, -1, nullptr, pdl);
    if (n > 0 && (energy || virial) && !timed) {
      // forces and the reduction of the partial rows in one launch
      const int ns = virial ? ACC_MV : ACC_E;  // the slots the launch filled
      launch_k(k_finalize_reduce, (unsigned)std::max((n + 255) / 256, kRedBlocks), 256, 0, st,
               pdl, n, (const unsigned long long *)c->d_facc, (const int *)c->d_sidx,
               fscale * kFixInv, accumulate, d_forces, g.ncell * ctx_slots(c, true),
               (const double *)c->d_partial, c->d_red, c->d_redctr, 1.0,
               d_out ? d_out : c->d_out, c->d_pairs, ns, f32, f32 ? tail : nullptr,
               (const int *)c->d_err);
      CK(cudaGetLastError());
      if (packed) *packed = f32 != nullptr;
      return PMB200_OK;
    }
    if (n > 0)
      launch_k(k_finalize, (unsigned)((n + 255) / 256), 256, 0, st, pdl, n,
               (const unsigned long long *)c->d_facc, (const int *)c->d_sidx, fscale * kFixInv,
               accumulate, d_forces);
  } else {
    if (c->form == FORM_GENERIC) launch_pair_fp64_half<FORM_GENERIC>(c, flags, st);
    else if (c->form == FORM_EWALD_POLY5) launch_pair_fp64_half<FORM_EWALD_POLY5>(c, flags, st);
    else if (c->form == FORM_EWALD_EXACT) launch_pair_fp64_half<FORM_EWALD_EXACT>(c, flags, st);
    else launch_pair_fp64_half<FORM_CUTOFF>(c, flags, st);
    if (n > 0)
      k_finalize64<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, c->d_facc, c->d_sidx,
                                                                 accumulate, d_forces);
  }
  CK(cudaGetLastError());
  if (timed) CK(cudaEventRecord(c->ev1, st));
  if (energy || virial) {
    // partial rows: one per (cell, slot) warp; both kernels visit each pair
    // once
    const int ns = virial ? ACC_MV : ACC_E;  // the slots the launch filled
    k_reduce1<<<kRedBlocks, 256, 0, st>>>(g.ncell * (mixed ? ctx_slots(c, true) : kFp64Slots),
                                          c->d_partial, c->d_red, ns);
    k_reduce2<<<1, 256, 0, st>>>(kRedBlocks, c->d_red, 1.0, d_out ? d_out : c->d_out,
                                c->d_pairs, ns);
    CK(cudaGetLastError());
  }
  return PMB200_OK;
}

// The integrator's kick + drift: plain, or with SETTLE on the rigid waters.
void launch_kick_drift(pmb200_ctx *c, double *d_pos, double *d_vel, const double *d_forces,
                       double kick, double h, cudaStream_t st) {
  const int n = c->n;
  if (n <= 0) return;
  if (c->nwater > 0) {
    const int units = c->nwater + c->nfree;
    k_kick_drift_settle<<<(units + 127) / 128, 128, 0, st>>>(
        c->nwater, c->d_widx, c->nfree, c->d_fidx, d_pos, d_vel, d_forces, c->d_mass, kick, h,
        c->sp);
  } else {
    k_kick_drift<<<(3 * n + 255) / 256, 256, 0, st>>>(n, d_pos, d_vel, d_forces, c->d_mass,
                                                      kick, h, 1);
  }
}

int check_ready(pmb200_ctx *c) {
  if (!c) return PMB200_EINVAL;
  if (!c->have_topo) return fail(c, PMB200_ESTATE, "pmb200_set_topology has not been called");
  if (!c->have_box) return fail(c, PMB200_ESTATE, "pmb200_set_box has not been called");
  return PMB200_OK;
}

}  // namespace

extern "C" {

int pmb200_create(const pmb200_params *params, pmb200_ctx **out) {
  pmb200_ctx *c = nullptr;
  if (!params || !out) return PMB200_EINVAL;
  *out = nullptr;
  const pmb200_params &p = *params;
  if (p.precision != PMB200_MIXED && p.precision != PMB200_FP64)
    return PMB200_EINVAL;
  // C2SwitchingFunction::make validation (C2SwitchingFunction.cpp:30-41)
  if (!(p.switchon >= 0.0) || !(p.cutoff_lj > 0.0) || !(p.switchon < p.cutoff_lj))
    return PMB200_EINVAL;
  if (!(p.cutoff_coul > 0.0) || !(p.cutoff_alg > 0.0)) return PMB200_EINVAL;
  if (p.cutoff_alg < rc_max(p)) return PMB200_EUNSUPPORTED;
  if (p.cellsize < 0.0) return PMB200_EINVAL;
  c = new pmb200_ctx();
  c->p = p;
  cudaError_t e = cudaSetDevice(p.device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(c->d_err, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_out, sizeof(double) * 20);
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_pairs, sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_red, sizeof(double) * kRedBlocks * ACC_MV);
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_redctr, sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(c->d_redctr, 0, sizeof(unsigned));
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
  if (e != cudaSuccess) {
    pmb200_destroy(c);
    return PMB200_ECUDA;
  }
  *out = c;
  return PMB200_OK;
}

int pmb200_create_ewald_real(const pmb200_ewald_params *params, pmb200_ctx **out) {
  if (!params || !out) return PMB200_EINVAL;
  *out = nullptr;
  const pmb200_ewald_params &e = *params;
  if (e.erfc != PMB200_ERFC_POLY5 && e.erfc != PMB200_ERFC_EXACT) return PMB200_EINVAL;
  if (!(e.accuracy > 0.0) || !(e.accuracy < 1.0) || !std::isfinite(e.alpha))
    return PMB200_EINVAL;
  if (e.cellsize < 0.0) return PMB200_EINVAL;
  // the shared construction path, with placeholder switch cutoffs
  pmb200_params p{};
  p.precision = e.precision;
  p.device = e.device;
  p.switchon = 0.0;
  p.cutoff_lj = p.cutoff_coul = p.cutoff_alg = 1.0;
  p.cellsize = e.cellsize;
  pmb200_ctx *c = nullptr;
  const int rc = pmb200_create(&p, &c);
  if (rc) return rc;
  c->form = e.erfc == PMB200_ERFC_EXACT ? FORM_EWALD_EXACT : FORM_EWALD_POLY5;
  c->ew_alpha_in = e.alpha;
  c->ew_accuracy = e.accuracy;
  *out = c;
  return PMB200_OK;
}

int pmb200_create_pair(const pmb200_pair_params *params, pmb200_ctx **out) {
  if (!params || !out) return PMB200_EINVAL;
  *out = nullptr;
  const pmb200_pair_params &q = *params;
  // LennardJonesTableForce<S, 7, Real> under UniversalSwitchingFunction: the
  // reference registers it for S = C2, Cn, ComplimentCnCn and alone
  // (NonbondedCutoffForceModule.cpp:67-72, 121-126)
  const bool table = (q.lj_switch & PMB200_SW_TABLE) != 0;
  if (table) {
    const int s = q.lj_switch & ~PMB200_SW_TABLE;
    if (q.coulomb_switch != PMB200_SW_NONE ||
        (s != PMB200_SW_C2 && s != PMB200_SW_CN && s != PMB200_SW_CMPCNCN))
      return PMB200_EUNSUPPORTED;
  }
  const int kinds[2] = {q.lj_switch & ~PMB200_SW_TABLE, q.coulomb_switch};
  const double *pars[2] = {q.lj, q.coulomb};
  double rcmax = 0.0;
  if (kinds[0] == PMB200_SW_NONE && kinds[1] == PMB200_SW_NONE) return PMB200_EINVAL;
  for (int k = 0; k < 2; k++) {
    const int kd = kinds[k];
    const double *pr = pars[k];
    if (kd == PMB200_SW_NONE) continue;
    if (kd != PMB200_SW_C1 && kd != PMB200_SW_C2 && kd != PMB200_SW_CN &&
        kd != PMB200_SW_CMPCNCN)
      return PMB200_EINVAL;
    const double ron = pr[0], rc = pr[1], order = pr[2], roff = pr[3];
    if (!(rc > 0.0) || !std::isfinite(rc)) return PMB200_EINVAL;
    if (kd == PMB200_SW_C2 && !(ron >= 0.0 && ron < rc)) return PMB200_EINVAL;
    if (kd == PMB200_SW_CN) {
      // CnSwitchingFunction::make (CnSwitchingFunction.cpp:84-112)
      if (!(ron >= 0.0 && ron < rc) || (roff > 0.0 && roff != rc) || order < 2.0 || order > 6.0)
        return PMB200_EINVAL;
      // the reference's order 5 has an all-zero coefficient row
      if ((int)order == 5 || order != std::floor(order)) return PMB200_EUNSUPPORTED;
      static const bool agree = cn_tables_agree();
      if (!agree) return PMB200_EUNSUPPORTED;
    }
    if (kd == PMB200_SW_CMPCNCN) {
      // CmpCnCnSwitchingFunction::make (CmpCnCnSwitchingFunction.cpp:53-68):
      // 0 <= switchon < switchoff <= cutoff, 2 <= order <= 6
      if (!(ron >= 0.0 && roff > 0.0 && ron < roff && roff <= rc) || order < 2.0 ||
          order > 6.0)
        return PMB200_EINVAL;
      // orders 2, 3, 4, 6 and 5 (read as 2); the reference truncates other
      // orders and its order-5 row is all zero: refused
      if (order != std::floor(order)) return PMB200_EUNSUPPORTED;
      static const bool agree = cn_tables_agree();
      if (!agree) return PMB200_EUNSUPPORTED;
    }
    rcmax = std::max(rcmax, rc);
  }
  if (!(q.cutoff_alg > 0.0) || q.cellsize < 0.0) return PMB200_EINVAL;
  if (q.cutoff_alg < rcmax) return PMB200_EUNSUPPORTED;
  pmb200_params p{};
  p.precision = q.precision;
  p.device = q.device;
  p.switchon = 0.0;
  p.cutoff_lj = p.cutoff_coul = rcmax;
  p.cutoff_alg = q.cutoff_alg;
  p.cellsize = q.cellsize;
  pmb200_ctx *c = nullptr;
  const int rc = pmb200_create(&p, &c);
  if (rc) return rc;
  c->form = FORM_GENERIC;
  for (int k = 0; k < 2; k++) {
    c->sw_kind[k] = kinds[k] == PMB200_SW_C1   ? SW_C1
                    : kinds[k] == PMB200_SW_C2 ? SW_C2
                    : kinds[k] == PMB200_SW_CN ? SW_CN
                    : kinds[k] == PMB200_SW_CMPCNCN ? SW_CMPCNCN
                                               : SW_OFF;
    for (int j = 0; j < 4; j++) c->sw_par[k][j] = pars[k][j];
  }
  if (table) {
    std::vector<double4> tab;
    build_lj_table(make_switch<double>(c->sw_kind[0], c->sw_par[0], 1.0), tab, c->tab_first,
                   c->tab_last);
    const bool ok = cudaSetDevice(c->p.device) == cudaSuccess &&
                    dalloc(c->d_ljtab, tab.size()) == cudaSuccess &&
                    cudaMemcpy(c->d_ljtab, tab.data(), sizeof(double4) * tab.size(),
                               cudaMemcpyHostToDevice) == cudaSuccess;
    if (!ok) {
      pmb200_destroy(c);
      return PMB200_ECUDA;
    }
  }
  *out = c;
  return PMB200_OK;
}

int pmb200_set_vacuum_domain(pmb200_ctx *c, const double lo[3], const double hi[3]) {
  if (!c) return PMB200_EINVAL;
  if (!lo || !hi) return fail(c, PMB200_EINVAL, "null domain corner");
  if (c->form == FORM_EWALD_POLY5 || c->form == FORM_EWALD_EXACT)
    return fail(c, PMB200_EUNSUPPORTED, "the Ewald term needs periodic boundaries");
  double e1[3] = {hi[0] - lo[0], 0, 0}, e2[3] = {0, hi[1] - lo[1], 0},
         e3[3] = {0, 0, hi[2] - lo[2]}, org[3];
  for (int a = 0; a < 3; a++) {
    if (!(hi[a] > lo[a]) || !std::isfinite(lo[a]) || !std::isfinite(hi[a]))
      return fail(c, PMB200_EINVAL, "domain axis %d: [%g, %g]", a, lo[a], hi[a]);
    org[a] = 0.5 * (lo[a] + hi[a]);
  }
  c->vacuum_pending = true;
  return pmb200_set_box(c, e1, e2, e3, org);
}

int pmb200_ewald_info(const pmb200_ctx *c, double *alpha, double *rc) {
  if (!c || !alpha || !rc) return PMB200_EINVAL;
  if (c->form == FORM_CUTOFF || !c->have_box || !c->have_topo) return PMB200_ESTATE;
  *alpha = c->ew_alpha;
  *rc = c->ew_rc;
  return PMB200_OK;
}

int pmb200_destroy(pmb200_ctx *c) {
  if (!c) return PMB200_OK;
  cudaSetDevice(c->p.device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  release_graph(c);
  dfree(c->d_type); dfree(c->d_mol); dfree(c->d_q); dfree(c->d_mass);
  dfree(c->d_ex_start); dfree(c->d_ex); dfree(c->d_mstart); dfree(c->d_matoms);
  dfree(c->d_lj32); dfree(c->d_lj64); dfree(c->d_ljtab); dfree(c->d_cblo); dfree(c->d_cbhi);
  dfree(c->d_count); dfree(c->d_start); dfree(c->d_err); dfree(c->d_partial);
  dfree(c->d_cell_of); dfree(c->d_slot); dfree(c->d_tmp); dfree(c->d_sidx);
  dfree(c->d_rel32); dfree(c->d_spos32); dfree(c->d_rel_lo); dfree(c->d_spos_lo); dfree(c->d_rel64); dfree(c->d_spos64);
  dfree(c->d_smeta); dfree(c->d_com); dfree(c->d_facc);
  dfree(c->d_tpart); dfree(c->d_gq); dfree(c->d_glj); dfree(c->d_wsorted);
  dfree(c->d_pairs); dfree(c->d_out); dfree(c->d_red); dfree(c->d_redctr); dfree(c->d_widx); dfree(c->d_fidx);
  dfree(c->d_sc_count); dfree(c->d_sc_start); dfree(c->d_sc_supbase); dfree(c->d_sc_ctl);
  dfree(c->d_sc_atom); dfree(c->d_sc_type); dfree(c->d_sc_mol); dfree(c->d_sc_cnt);
  dfree(c->d_sc_xi); dfree(c->d_sc_xj); dfree(c->d_sc_xilo); dfree(c->d_sc_xjlo);
  dfree(c->d_sc_clo); dfree(c->d_sc_chi); dfree(c->d_sc_sbox); dfree(c->d_sc_corg);
  dfree(c->d_sc_sorg); dfree(c->d_sc_tasks); dfree(c->d_sc_cmol); dfree(c->d_sc_ent);
  dfree(c->d_sc_facc); dfree(c->d_sc_part);
  if (c->h_pin_pos) cudaFreeHost(c->h_pin_pos);
  if (c->h_pin_frc) cudaFreeHost(c->h_pin_frc);
  if (c->h_pin_out) cudaFreeHost(c->h_pin_out); dfree(c->d_hpos); dfree(c->d_hfrc);
  dfree(c->d_hf32);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->ev_lj) cudaEventDestroy(c->ev_lj);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return PMB200_OK;
}

const char *pmb200_last_error(const pmb200_ctx *c) {
  return c ? c->err.c_str() : "null context";
}

int pmb200_set_topology(pmb200_ctx *c, int n, const int *type, const double *q_scaled,
                        const int *molecule, const double *mass, int ntypes,
                        const double *lj, int nexcl, const int *excl,
                        double coulomb_scaling) {
  if (!c) return PMB200_EINVAL;
  if (n < 0 || ntypes <= 0 || nexcl < 0) return fail(c, PMB200_EINVAL, "negative size");
  if (n > 0 && (!type || !q_scaled || !molecule)) return fail(c, PMB200_EINVAL, "null array");
  if (!lj) return fail(c, PMB200_EINVAL, "null LJ table");
  if (nexcl > 0 && !excl) return fail(c, PMB200_EINVAL, "null exclusion array");
  if (ntypes > kMaxTypesTable)
    return fail(c, PMB200_EUNSUPPORTED, "%d LJ types; at most %d supported", ntypes,
                kMaxTypesTable);
  CK(cudaSetDevice(c->p.device));
  int nmol = 0;
  for (int i = 0; i < n; i++) {
    if (type[i] < 0 || type[i] >= ntypes)
      return fail(c, PMB200_EINVAL, "atom %d: type %d outside [0, %d)", i, type[i], ntypes);
    if (molecule[i] < 0) return fail(c, PMB200_EINVAL, "atom %d: negative molecule id", i);
    if (!std::isfinite(q_scaled[i])) return fail(c, PMB200_EINVAL, "atom %d: charge", i);
    nmol = std::max(nmol, molecule[i] + 1);
  }
  for (int k = 0; k < 4 * ntypes * ntypes; k++)
    if (!std::isfinite(lj[k])) return fail(c, PMB200_EINVAL, "LJ table entry %d", k);
  // ExclusionTable::add semantics: keyed by (min, max), later entries win,
  // EXCLUSION_NONE removes (ExclusionTable.cpp:103-120).
  std::map<std::pair<int, int>, int> kinds;
  for (int e = 0; e < nexcl; e++) {
    int a = excl[3 * e], b = excl[3 * e + 1], k = excl[3 * e + 2];
    if (a < 0 || b < 0 || a >= n || b >= n)
      return fail(c, PMB200_EINVAL, "exclusion %d: atom index out of range", e);
    if (k < 0 || k > 2) return fail(c, PMB200_EINVAL, "exclusion %d: kind %d", e, k);
    if (a == b) continue;
    kinds[std::make_pair(std::min(a, b), std::max(a, b))] = k;
  }
  std::vector<std::vector<int2>> per(n);
  bool modified = false;
  for (const auto &kv : kinds) {
    if (kv.second == 0) continue;
    modified = modified || kv.second == 1;
    per[kv.first.first].push_back(make_int2(kv.first.second, kv.second));
    per[kv.first.second].push_back(make_int2(kv.first.first, kv.second));
  }
  std::vector<int> ex_start(n + 1, 0);
  std::vector<int2> ex;
  for (int i = 0; i < n; i++) {
    std::sort(per[i].begin(), per[i].end(), [](int2 x, int2 y) { return x.x < y.x; });
    ex_start[i] = (int)ex.size();
    ex.insert(ex.end(), per[i].begin(), per[i].end());
  }
  ex_start[n] = (int)ex.size();
  std::vector<int> mstart(nmol + 1, 0), matoms(n);
  for (int i = 0; i < n; i++) mstart[molecule[i] + 1]++;
  for (int m = 0; m < nmol; m++) mstart[m + 1] += mstart[m];
  {
    std::vector<int> fill(mstart.begin(), mstart.end() - 1);
    for (int i = 0; i < n; i++) matoms[fill[molecule[i]]++] = i;
  }
  release_graph(c);
  c->nwater = c->nfree = 0;  // rigid waters refer to the old atom list
  c->n = n;
  c->ntypes = ntypes;
  c->nmol = nmol;
  c->csf = coulomb_scaling;
  c->has_modified = modified;
  c->have_mass = mass != nullptr;
  c->h_lj.assign(lj, lj + 4 * ntypes * ntypes);
  c->lj_dev_newer = false;
  const size_t nn = (size_t)std::max(n, 1);
  CK(dalloc(c->d_type, nn));
  CK(dalloc(c->d_mol, nn));
  CK(dalloc(c->d_q, nn));
  CK(dalloc(c->d_mass, nn));
  CK(dalloc(c->d_ex_start, nn + 1));
  CK(dalloc(c->d_ex, std::max<size_t>(ex.size(), 1)));
  CK(dalloc(c->d_mstart, (size_t)nmol + 1));
  CK(dalloc(c->d_matoms, nn));
  CK(dalloc(c->d_com, 3 * (size_t)std::max(nmol, 1)));
  CK(dalloc(c->d_lj32, (size_t)ntypes * ntypes));
  CK(dalloc(c->d_lj64, (size_t)ntypes * ntypes));
  if (n > 0) {
    CK(cudaMemcpy(c->d_type, type, sizeof(int) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_mol, molecule, sizeof(int) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_q, q_scaled, sizeof(double) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_matoms, matoms.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    if (mass) CK(cudaMemcpy(c->d_mass, mass, sizeof(double) * n, cudaMemcpyHostToDevice));
  }
  CK(cudaMemcpy(c->d_ex_start, ex_start.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
  if (!ex.empty())
    CK(cudaMemcpy(c->d_ex, ex.data(), sizeof(int2) * ex.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_mstart, mstart.data(), sizeof(int) * (nmol + 1), cudaMemcpyHostToDevice));
  int rc = ensure_atom_buffers(c);
  if (rc) return rc;
  c->have_topo = true;
  // an Ewald context's cutoff may depend on N (default alpha): rebuild the grid
  if (c->form != FORM_CUTOFF && c->box_given)
    return pmb200_set_box(c, c->box_e[0], c->box_e[1], c->box_e[2], c->box_origin);
  if (c->have_box) {
    const int r = upload_lj(c);
    return r ? r : sc_prepare(c);
  }
  return PMB200_OK;
}

int pmb200_set_box(pmb200_ctx *c, const double e1[3], const double e2[3], const double e3[3],
                   const double origin[3]) {
  if (!c) return PMB200_EINVAL;
  // a box is periodic unless it comes from pmb200_set_vacuum_domain
  const bool vacuum = c->vacuum_pending;
  c->vacuum_pending = false;
  if (!e1 || !e2 || !e3 || !origin) return fail(c, PMB200_EINVAL, "null box vector");
  c->vacuum = vacuum;
  // PeriodicBoundaryConditions::set (PeriodicBoundaryConditions.cpp:38-66):
  // orthogonal when every off-diagonal component is zero; the reciprocal
  // vectors e_k^r = (e_{k+1} x e_{k+2}) / (e_k . (e_{k+1} x e_{k+2}))
  const bool ortho = !(e1[1] != 0.0 || e1[2] != 0.0 || e2[0] != 0.0 || e2[2] != 0.0 ||
                       e3[0] != 0.0 || e3[1] != 0.0);
  const double *ev[3] = {e1, e2, e3};
  for (int k = 0; k < 3; k++)
    for (int a = 0; a < 3; a++)
      if (!std::isfinite(ev[k][a])) return fail(c, PMB200_EINVAL, "box vector %d", k + 1);
  if (!ortho && vacuum)
    return fail(c, PMB200_EINVAL, "a vacuum domain is an axis-aligned box");
  auto cross = [](const double *a, const double *b, double *o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
  };
  auto dot = [](const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
  double er[3][3], width[3];
  for (int k = 0; k < 3; k++) {
    double x[3];
    cross(ev[(k + 1) % 3], ev[(k + 2) % 3], x);
    const double den = dot(ev[k], x);
    for (int a = 0; a < 3; a++) er[k][a] = x[a] / den;
    width[k] = 1.0 / std::sqrt(dot(er[k], er[k]));  // distance between the faces
  }
  double cr[3];
  cross(e1, e2, cr);
  const double volume = std::fabs(dot(cr, e3));
  if (!(volume > 0.0) || !std::isfinite(volume)) return fail(c, PMB200_EINVAL, "box has no volume");
  const double L[3] = {std::fabs(e1[0]), std::fabs(e2[1]), std::fabs(e3[2])};
  for (int a = 0; a < 3; a++) {
    if (ortho && (!(L[a] > 0.0) || !std::isfinite(L[a])))
      return fail(c, PMB200_EINVAL, "box edge %d is %g", a, L[a]);
    if (!std::isfinite(origin[a])) return fail(c, PMB200_EINVAL, "origin");
  }
  for (int k = 0; k < 3; k++) {
    c->box_e[0][k] = e1[k]; c->box_e[1][k] = e2[k]; c->box_e[2][k] = e3[k];
    c->box_origin[k] = origin[k];
  }
  c->box_given = true;
  if (c->form != FORM_CUTOFF) {
    if (!c->have_topo) {  // alpha may need N: finish when the topology arrives
      c->have_box = false;
      return PMB200_OK;
    }
    ewald_derive(c, volume);
  }
  const double rc = ctx_rc(c);
  for (int a = 0; a < 3; a++) {
    if (width[a] < 2.0 * rc && !c->vacuum)
      return fail(c, PMB200_EUNSUPPORTED,
                  "box width %g is below twice the cutoff %g (minimum image would need more "
                  "than one image per pair)", width[a], rc);
  }
  CK(cudaSetDevice(c->p.device));
  release_graph(c);
  GridParams &g = c->g;
  g.tric = ortho ? 0 : 1;
  int nd[3];
  if (ortho) {
    const double target = c->p.cellsize > 0.0 ? std::max(c->p.cellsize, rc / 3.0) : rc / 2.0;
    for (int a = 0; a < 3; a++) {
      nd[a] = std::max(1, (int)std::floor(L[a] / target));
      g.edge[a] = L[a] / nd[a];
      g.boxlen[a] = L[a];
      g.boxmin[a] = origin[a] - 0.5 * L[a];
    }
    g.unit = g.edge[0];
  } else {
    // cells along each basis vector, a third of the cutoff wide by default;
    // every neighbour-cell offset must be distinct modulo the grid, which
    // also makes the image a cell offset gives a pair within the cutoff the
    // reference's (fractional rounding) image
    const double target = c->p.cellsize > 0.0 ? std::max(c->p.cellsize, rc / 4.0) : rc / 3.0;
    double unit = 1e300;
    for (int k = 0; k < 3; k++) {
      nd[k] = std::max(1, (int)std::floor(width[k] / target));
      const int R = (int)std::ceil(rc * nd[k] / width[k] - 1e-12);
      if (2 * R + 1 > nd[k])
        return fail(c, PMB200_EUNSUPPORTED,
                    "general periodic cell: width %g along basis vector %d holds %d cells of "
                    "%g A, but the cutoff %g needs %d on each side of a cell (widths of about "
                    "3 cutoffs or more are supported)", width[k], k + 1, nd[k],
                    width[k] / nd[k], rc, R);
      g.edge[k] = width[k] / nd[k];
      unit = std::min(unit, g.edge[k]);
      for (int a = 0; a < 3; a++) {
        g.lat[3 * k + a] = nd[k] * er[k][a];
        g.ec[3 * a + k] = ev[k][a] / nd[k];
      }
    }
    g.unit = unit;
    for (int q = 0; q < 9; q++) g.m[q] = g.ec[q] / unit;
    for (int a = 0; a < 3; a++) {
      g.org[a] = origin[a];
      g.boxmin[a] = origin[a] - 0.5 * (e1[a] + e2[a] + e3[a]);
      g.boxlen[a] = 0.0;  // (not used by the lattice cell build)
    }
  }
  g.nx = nd[0]; g.ny = nd[1]; g.nz = nd[2];
  g.periodic = c->vacuum ? 0 : 1;
  const long long ncell = (long long)nd[0] * nd[1] * nd[2];
  if (ncell > (1 << 24)) return fail(c, PMB200_EUNSUPPORTED, "%lld cells", ncell);
  g.ncell = (int)ncell;
  // stencils for the cutoff: the FP64 kernel's full shell and the mixed
  // kernel's half shell
  int src = build_stencils(c, rc, c->rows, c->half);
  if (src) return src;
  g.nrows = (int)c->rows.size();
  c->stencil = Stencil{};
  for (size_t r = 0; r < c->rows.size(); r++) c->stencil.rows[r] = c->rows[r];
  if (c->ncell_alloc < g.ncell) {
    CK(dalloc(c->d_count, (size_t)g.ncell));
    CK(cudaMemset(c->d_count, 0, sizeof(int) * (size_t)g.ncell));
    c->count_zero = true;
    CK(dalloc(c->d_start, (size_t)g.ncell + 1));
    CK(dalloc(c->d_partial, (size_t)g.ncell * kMaxCellSlots * kNacc));
    c->ncell_alloc = g.ncell;
  }
  // constants
  const pmb200_params &p = c->p;
  const double u = g.unit;
  const double rl = p.cutoff_lj / u, ro = p.switchon / u, rq = p.cutoff_coul / u;
  const double t = rl * rl - ro * ro;
  MixedConsts &m = c->mc;
  m.cut2 = (float)((rc / u) * (rc / u));
  m.rclj2 = (float)(rl * rl);
  m.ron2 = (float)(ro * ro);
  m.rcc2 = (float)(rq * rq);
  m.s1 = (float)(1.0 / (t * t * t));
  m.s2 = (float)(rl * rl - 3.0 * ro * ro);
  m.s3 = (float)(4.0 / (t * t * t));
  m.c15_1 = (float)(1.5 / rq);
  m.c05_3 = (float)(0.5 / (rq * rq * rq));
  m.c15_3 = (float)(1.5 / (rq * rq * rq));
  m.e15 = 1.5 / rq;
  m.e05 = 0.5 / (rq * rq * rq);
  m.csf = (float)c->csf;
  m.ey = (float)(g.edge[1] / u);
  m.ez = (float)(g.edge[2] / u);
  m.swl = make_switch<float>(c->sw_kind[0], c->sw_par[0], u);
  m.swc = make_switch<float>(c->sw_kind[1], c->sw_par[1], u);
  m.ea = (float)(c->ew_alpha * u);
  m.ea2pi = (float)(2.0 * c->ew_alpha * u / std::sqrt(M_PI));
  Fp64Consts &f = c->fc;
  const double tl = p.cutoff_lj * p.cutoff_lj - p.switchon * p.switchon;
  f.cut2 = rc * rc;
  f.rclj2 = p.cutoff_lj * p.cutoff_lj;
  f.ron2 = p.switchon * p.switchon;
  f.rcc2 = p.cutoff_coul * p.cutoff_coul;
  f.s1 = 1.0 / ((tl * tl) * tl);
  f.s2 = p.cutoff_lj * p.cutoff_lj - 3.0 * p.switchon * p.switchon;
  f.s3 = 4.0 / ((tl * tl) * tl);
  f.c15_1 = 1.5 / p.cutoff_coul;
  f.c05_3 = 0.5 / (p.cutoff_coul * p.cutoff_coul * p.cutoff_coul);
  f.c15_3 = 1.5 / (p.cutoff_coul * p.cutoff_coul * p.cutoff_coul);
  f.csf = c->csf;
  f.swl = make_switch<double>(c->sw_kind[0], c->sw_par[0], 1.0);
  f.swc = make_switch<double>(c->sw_kind[1], c->sw_par[1], 1.0);
  f.ljtab = c->d_ljtab;
  f.tfirst = c->tab_first;
  f.tlast = c->tab_last;
  f.ea = c->ew_alpha;
  f.ea2 = c->ew_alpha * c->ew_alpha;
  f.ea2pi = 2.0 * c->ew_alpha / std::sqrt(M_PI);
  // PeriodicBoundaryConditions::set, orthogonal case (min/max corners,
  // myH, myH2, reciprocal basis, myD), for the molecule-centre image
  PbcRef &b = c->pb;
  b = PbcRef{};
  for (int a = 0; a < 3; a++) {
    const double lo = origin[a] - L[a] * 0.5, hi = origin[a] + L[a] * 0.5;
    b.e[a] = L[a];
    b.h[a] = std::max(lo, hi) - std::min(lo, hi);
    b.h2[a] = b.h[a] * 0.5;
  }
  b.er[0] = (L[1] * L[2]) / (L[0] * (L[1] * L[2]));
  b.er[1] = (L[2] * L[0]) / (L[1] * (L[2] * L[0]));
  b.er[2] = (L[0] * L[1]) / (L[2] * (L[0] * L[1]));
  b.d = std::min((L[0] * 0.5) * (L[0] * 0.5),
                 std::min((L[1] * 0.5) * (L[1] * 0.5), (L[2] * 0.5) * (L[2] * 0.5)));
  if (!ortho) {  // the general branch of minimalDifference
    b.tric = 1;
    for (int k = 0; k < 3; k++)
      for (int a = 0; a < 3; a++) {
        b.ev[3 * k + a] = ev[k][a];
        b.erv[3 * k + a] = er[k][a];
      }
  }
  if (c->vacuum) b.d = std::numeric_limits<double>::infinity();  // no images
  c->have_box = true;
  if (c->have_topo) {
    const int r = upload_lj(c);
    return r ? r : sc_prepare(c);
  }
  return PMB200_OK;
}

int pmb200_eval_device(pmb200_ctx *c, const double *d_pos, double *d_forces, double *d_out,
                       unsigned flags, void *stream) {
  int rc = check_ready(c);
  if (rc) return rc;
  if ((flags & PMB200_MOLVIRIAL) && !c->have_mass)
    return fail(c, PMB200_EINVAL, "molecular virial needs masses");
  if (c->n > 0 && (!d_pos || !d_forces)) return fail(c, PMB200_EINVAL, "null device buffer");
  CK(cudaSetDevice(c->p.device));
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  return launch_eval(c, d_pos, d_forces, d_out, flags, 1, st);
}

}  // extern "C"

namespace {

// ---- single-context autotuner ----
// Choices found for a workload, kept for the process: contexts with the same
// key take them without timing again.
struct TuneChoice {
  double cellsize;         // the cell-size hint applied (0: the default)
  int slots_e, slots_f;    // mixed warps per i-cell (0 for FP64 contexts)
  bool tiles_e, tiles_f;   // the cluster-pair kernel with / without energies
  bool clu_e, clu_f;       // the supercluster kernel with / without energies
  double sc_side;          // its column width factor (sc_prepare)
  double ms_e, ms_f;       // median evaluation times with and without energies
  int tried;               // configurations timed
};
std::mutex g_tune_mutex;
std::map<std::string, TuneChoice> g_tune_cache;

std::string tune_key(const pmb200_ctx *c) {
  cudaDeviceProp prop{};
  cudaGetDeviceProperties(&prop, c->p.device);
  char buf[512];
  std::snprintf(buf, sizeof buf,
                "%s|%d|form%d|prec%d|n%d|t%d|vac%d|rc%.6g|%.6g %.6g %.6g|%.6g %.6g %.6g|"
                "%.6g %.6g %.6g|sw%d,%d|%.6g %.6g %.6g %.6g|tab%d",
                prop.name, prop.multiProcessorCount, c->form, c->p.precision, c->n, c->ntypes,
                c->vacuum ? 1 : 0, ctx_rc(c), c->box_e[0][0], c->box_e[0][1], c->box_e[0][2],
                c->box_e[1][0], c->box_e[1][1], c->box_e[1][2], c->box_e[2][0], c->box_e[2][1],
                c->box_e[2][2], c->sw_kind[0], c->sw_kind[1], c->sw_par[0][0], c->sw_par[0][1],
                c->sw_par[1][0], c->sw_par[1][1], c->d_ljtab ? 1 : 0);
  return buf;
}

// Re-applies the context's box (or vacuum domain) under its current hint.
int reapply_box(pmb200_ctx *c) {
  if (c->vacuum) c->vacuum_pending = true;
  return pmb200_set_box(c, c->box_e[0], c->box_e[1], c->box_e[2], c->box_origin);
}

}  // namespace

extern "C" {

int pmb200_set_pair_kernel(pmb200_ctx *c, int kernel) {
  if (!c) return PMB200_EINVAL;
  if (kernel != PMB200_KERNEL_SEARCH && kernel != PMB200_KERNEL_TILES &&
      kernel != PMB200_KERNEL_CLUSTERS)
    return fail(c, PMB200_EINVAL, "pair kernel %d", kernel);
  CK(cudaSetDevice(c->p.device));
  c->tiles_e = c->tiles_f = kernel == PMB200_KERNEL_TILES;
  c->clu_e = c->clu_f = kernel == PMB200_KERNEL_CLUSTERS;
  release_graph(c);  // graphs hold the previous kernel
  return sc_prepare(c);
}

int pmb200_autotune(pmb200_ctx *c, const double *d_pos, void *stream, int reps,
                    double result[8]) {
  int rc = check_ready(c);
  if (rc) return rc;
  if (c->n > 0 && !d_pos) return fail(c, PMB200_EINVAL, "null device buffer");
  if (reps < 1 || reps > 1000) return fail(c, PMB200_EINVAL, "reps %d (1..1000)", reps);
  CK(cudaSetDevice(c->p.device));
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  const bool mixed = c->p.precision == PMB200_MIXED;
  const std::string key = tune_key(c);
  TuneChoice best{};
  bool cached = false;
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      best = it->second;
      cached = true;
    }
  }
  const double hint0 = c->p.cellsize;
  if (!cached) {
    // candidate cell sizes (as hints; the grid takes the largest cell of at
    // most the hint that divides each box edge, so some give the same grid)
    const double rc_cut = ctx_rc(c);
    // the library's defaults first (rc/2 cells, rc/3 for general cells; 4
    // warps per i-cell; the search kernel): another configuration replaces
    // the incumbent only when it is kTuneMargin faster, so that timing noise
    // between near-equal configurations does not move the choice
    constexpr double kTuneMargin = 0.02;
    const double divs_o[] = {2.0, 1.5, 2.5, 3.0, 3.5, 4.0};
    const double divs_t[] = {3.0, 1.5, 2.0, 2.5, 3.5, 4.0};
    const bool tric0 = c->g.tric != 0;
    const int slot_opts[] = {4, 8, 2};
    auto faster = [&](double t, double incumbent) { return t < incumbent * (1.0 - kTuneMargin); };
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    // one evaluation as the library runs it in a step or a host-buffer call:
    // captured once as a graph and replayed (launching its kernels one by one
    // from the host would time the host's launch rate for the paths with
    // more kernels)
    auto timed = [&](unsigned flags, double &ms) -> int {
      std::vector<float> t((size_t)reps);
      int r = ensure_clear(c, st);
      if (r) return r;
      cudaGraph_t gr = nullptr;
      cudaGraphExec_t ge = nullptr;
      if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        // a stream that cannot be captured (the legacy default stream):
        // direct launches, timed the same way
        cudaGetLastError();
        r = launch_eval(c, d_pos, c->d_hfrc, c->d_out, flags, 0, st);  // warm-up
        for (int k = 0; k < reps && !r; k++) {
          if (cudaEventRecord(e0, st) != cudaSuccess) return PMB200_ECUDA;
          r = launch_eval(c, d_pos, c->d_hfrc, c->d_out, flags, 0, st);
          if (!r && (cudaEventRecord(e1, st) != cudaSuccess ||
                     cudaEventSynchronize(e1) != cudaSuccess ||
                     cudaEventElapsedTime(&t[k], e0, e1) != cudaSuccess))
            r = PMB200_ECUDA;
        }
        if (r) return r;
        std::nth_element(t.begin(), t.begin() + reps / 2, t.end());
        ms = t[reps / 2];
        return PMB200_OK;
      }
      r = launch_eval(c, d_pos, c->d_hfrc, c->d_out, flags, 0, st);
      const cudaError_t ce = cudaStreamEndCapture(st, &gr);
      if (r || ce != cudaSuccess || cudaGraphInstantiate(&ge, gr, 0) != cudaSuccess) {
        if (gr) cudaGraphDestroy(gr);
        return r ? r : fail(c, PMB200_ECUDA, "autotune: capture failed");
      }
      if (cudaGraphLaunch(ge, st) != cudaSuccess) r = PMB200_ECUDA;  // warm-up
      for (int k = 0; k < reps && !r; k++) {
        if (cudaEventRecord(e0, st) != cudaSuccess || cudaGraphLaunch(ge, st) != cudaSuccess ||
            cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&t[k], e0, e1) != cudaSuccess)
          r = PMB200_ECUDA;
      }
      cudaGraphExecDestroy(ge);
      cudaGraphDestroy(gr);
      if (r) return fail(c, r, "autotune: timed replay failed");
      std::nth_element(t.begin(), t.begin() + reps / 2, t.end());
      ms = t[reps / 2];
      return PMB200_OK;
    };
    int last_dims[3] = {-1, -1, -1};
    best.ms_e = 1e300;
    int status = PMB200_OK;
    const double *divs = tric0 ? divs_t : divs_o;
    for (int di = 0; di < 6; di++) {
      c->p.cellsize = rc_cut / divs[di];
      c->tiles_e = c->tiles_f = false;
      if (reapply_box(c) != PMB200_OK) continue;  // a grid the stencil limits refuse
      const int dims[3] = {c->g.nx, c->g.ny, c->g.nz};
      if (dims[0] == last_dims[0] && dims[1] == last_dims[1] && dims[2] == last_dims[2])
        continue;  // the same grid as the previous hint
      for (int a = 0; a < 3; a++) last_dims[a] = dims[a];
      TuneChoice cand{};
      cand.cellsize = c->p.cellsize;
      cand.ms_e = cand.ms_f = 1e300;
      // the search kernel, and the cluster-pair kernel where it applies
      for (int kern = 0; kern < 2 && !status; kern++) {
        c->tiles_e = c->tiles_f = kern == 1;
        if (kern == 1 && !tiles_apply(c, PMB200_ENERGY) && !tiles_apply(c, 0u)) break;
        for (int so : slot_opts) {
          if (!mixed && so != slot_opts[0]) break;  // the FP64 kernel's split is fixed
          double me = 0.0, mf = 0.0;
          c->slots_e = c->slots_f = mixed ? so : 0;
          status = timed(PMB200_ENERGY, me);
          if (!status) status = timed(0u, mf);
          if (status) break;
          best.tried++;
          if (faster(me, cand.ms_e)) {
            cand.ms_e = me;
            cand.slots_e = mixed ? so : 0;
            cand.tiles_e = kern == 1;
          }
          if (faster(mf, cand.ms_f)) {
            cand.ms_f = mf;
            cand.slots_f = mixed ? so : 0;
            cand.tiles_f = kern == 1;
          }
        }
      }
      c->tiles_e = c->tiles_f = false;
      if (status) break;
      if (faster(cand.ms_e, best.ms_e)) {
        const int tried = best.tried;
        best = cand;
        best.tried = tried;
      }
    }
    if (!status && best.ms_e < 1e300 && mixed) {
      // the supercluster kernel where it applies (its own grid: the cell size
      // and the warps per i-cell do not concern it), on the best cell grid
      // column widths of 0.8 to 1.15 times the edge of a cube of 32 atoms (how
      // many superclusters a column's atoms fill, and so the padding, varies
      // with it)
      c->p.cellsize = best.cellsize;
      c->clu_e = c->clu_f = true;
      double bme = 1e300, bmf = 1e300, bside = 1.0;
      int last_cols = -1;
      for (double side : {1.0, 0.9, 0.8, 1.15}) {
        c->sc_side = side;
        if (reapply_box(c) != PMB200_OK || !c->sc_ok) continue;
        if (c->sg.ncol == last_cols) continue;  // the same columns as the previous width
        last_cols = c->sg.ncol;
        double me = 0.0, mf = 0.0;
        int r = timed(PMB200_ENERGY, me);
        if (!r) r = timed(0u, mf);
        int e = 0;
        if (!r && (cudaStreamSynchronize(st) != cudaSuccess ||
                   cudaMemcpy(&e, c->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess))
          r = PMB200_ECUDA;
        if (e) cudaMemset(c->d_err, 0, sizeof(int));  // (lists too long: not a candidate)
        if (r) {
          status = r;
          break;
        }
        if (e) continue;
        best.tried += 2;
        if (me < bme) {
          bme = me;
          bmf = mf;
          bside = side;
        }
      }
      if (!status && bme < 1e300) {
        if (faster(bme, best.ms_e)) {
          best.ms_e = bme;
          best.clu_e = true;
          best.tiles_e = false;
        }
        if (faster(bmf, best.ms_f)) {
          best.ms_f = bmf;
          best.clu_f = true;
          best.tiles_f = false;
        }
        best.sc_side = bside;
      }
      c->clu_e = c->clu_f = false;
      c->sc_side = 1.0;
      c->sc_ok = false;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (status || best.ms_e >= 1e300) {
      c->p.cellsize = hint0;
      c->slots_e = c->slots_f = 0;
      c->tiles_e = c->tiles_f = false;
      c->clu_e = c->clu_f = false;
      const int r2 = reapply_box(c);
      return status ? status : (r2 ? r2 : fail(c, PMB200_EUNSUPPORTED, "no grid to tune"));
    }
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache[key] = best;
  }
  // apply the choice
  c->p.cellsize = best.cellsize;
  rc = reapply_box(c);
  if (rc) {
    c->p.cellsize = hint0;
    reapply_box(c);
    return rc;
  }
  c->slots_e = best.slots_e;
  c->slots_f = best.slots_f;
  c->tiles_e = best.tiles_e;
  c->tiles_f = best.tiles_f;
  c->clu_e = best.clu_e;
  c->clu_f = best.clu_f;
  c->sc_side = best.sc_side > 0.0 ? best.sc_side : 1.0;
  rc = sc_prepare(c);
  if (rc) return rc;
  release_graph(c);  // graphs hold the previous launch shapes
  if (result) {
    result[0] = best.cellsize;
    result[1] = best.slots_e;
    result[2] = best.slots_f;
    result[3] = best.ms_e;
    result[4] = best.ms_f;
    result[5] = cached ? 0.0 : best.tried;
    result[6] = best.clu_e ? PMB200_KERNEL_CLUSTERS
                           : (best.tiles_e ? PMB200_KERNEL_TILES : PMB200_KERNEL_SEARCH);
    result[7] = best.clu_f ? PMB200_KERNEL_CLUSTERS
                           : (best.tiles_f ? PMB200_KERNEL_TILES : PMB200_KERNEL_SEARCH);
  }
  return PMB200_OK;
}

// Force decomposition: shard s of nshards takes the i-cells
// [ncell * s / nshards, ncell * (s + 1) / nshards) of the half-shell walk.
int pmb200_shard_eval_device(pmb200_ctx *c, const double *d_pos, int shard, int nshards,
                             long long *d_facc, double *d_out, unsigned flags, void *stream) {
  int rc = check_ready(c);
  if (rc) return rc;
  if (c->p.precision != PMB200_MIXED)
    return fail(c, PMB200_EUNSUPPORTED, "sharded evaluation needs a mixed-precision context");
  if (nshards < 1 || shard < 0 || shard >= nshards)
    return fail(c, PMB200_EINVAL, "shard %d of %d", shard, nshards);
  if ((flags & PMB200_MOLVIRIAL) && !c->have_mass)
    return fail(c, PMB200_EINVAL, "molecular virial needs masses");
  if (c->n > 0 && (!d_pos || !d_facc)) return fail(c, PMB200_EINVAL, "null device buffer");
  if (flags && !d_out) return fail(c, PMB200_EINVAL, "null output buffer");
  CK(cudaSetDevice(c->p.device));
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  const GridParams &g = c->g;
  const int n = c->n;
  const bool energy = (flags & PMB200_ENERGY) != 0;
  const bool virial = (flags & (PMB200_VIRIAL | PMB200_MOLVIRIAL)) != 0;
  const int lo = (int)((long long)g.ncell * shard / nshards);
  const int hi = (int)((long long)g.ncell * (shard + 1) / nshards);
  unsigned long long *facc = reinterpret_cast<unsigned long long *>(d_facc);
  launch_cell_build(c, d_pos, true, energy && c->form == FORM_CUTOFF, st);
  if ((flags & PMB200_MOLVIRIAL) && c->nmol > 0)
    k_com<<<(c->nmol + 127) / 128, 128, 0, st>>>(c->nmol, c->d_mstart, c->d_matoms, c->d_mass,
                                                  d_pos, c->d_com);
  if (n > 0) CK(cudaMemsetAsync(facc, 0, sizeof(unsigned long long) * 3 * (size_t)n, st));
  if (hi > lo) {
    if (c->form == FORM_GENERIC) launch_pair_mixed<FORM_GENERIC>(c, flags, st, lo, hi - lo, facc);
    else if (c->form == FORM_EWALD_POLY5)
      launch_pair_mixed<FORM_EWALD_POLY5>(c, flags, st, lo, hi - lo, facc);
    else if (c->form == FORM_EWALD_EXACT)
      launch_pair_mixed<FORM_EWALD_EXACT>(c, flags, st, lo, hi - lo, facc);
    else launch_pair_mixed<FORM_CUTOFF>(c, flags, st, lo, hi - lo, facc);
  }
  CK(cudaGetLastError());
  if (energy || virial) {
    if (hi > lo) {
      // this shard's partial rows: one per (cell, slot) warp
      const int ns = (flags & (PMB200_VIRIAL | PMB200_MOLVIRIAL)) ? ACC_MV : ACC_E;
      k_reduce1<<<kRedBlocks, 256, 0, st>>>((hi - lo) * ctx_slots(c, true),
                                            c->d_partial, c->d_red, ns);
      k_reduce2<<<1, 256, 0, st>>>(kRedBlocks, c->d_red, 1.0, d_out, c->d_pairs, ns);
    } else {
      CK(cudaMemsetAsync(d_out, 0, sizeof(double) * 20, st));
      CK(cudaMemsetAsync(c->d_pairs, 0, sizeof(double), st));
    }
    CK(cudaGetLastError());
  }
  return PMB200_OK;
}

int pmb200_shard_finalize(pmb200_ctx *c, const long long *d_facc, double *d_forces,
                          void *stream) {
  int rc = check_ready(c);
  if (rc) return rc;
  if (c->p.precision != PMB200_MIXED)
    return fail(c, PMB200_EUNSUPPORTED, "sharded evaluation needs a mixed-precision context");
  if (c->n > 0 && (!d_facc || !d_forces)) return fail(c, PMB200_EINVAL, "null device buffer");
  CK(cudaSetDevice(c->p.device));
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  if (c->n > 0)
    k_finalize<<<(c->n + 255) / 256, 256, 0, st>>>(
        c->n, reinterpret_cast<const unsigned long long *>(d_facc), c->d_sidx,
        kFixInv / c->g.unit, 1, d_forces);
  CK(cudaGetLastError());
  return PMB200_OK;
}

// Derivative kernels (FP64 pair arithmetic whatever the context's
// precision; cutoff form only): the half-shell kernel for Hessian-vector
// products and, with at most kDerivRegTypes LJ types, for the parameter
// derivatives; the full-shell kernel for the parameter derivatives of larger
// tables.
#ifndef PMB200_HVP_SLOTS
#define PMB200_HVP_SLOTS 4
#endif
constexpr int kDerivSlots = PMB200_HVP_SLOTS;  // warps per i-cell of k_deriv_fp64_half
static int launch_deriv(pmb200_ctx *c, int mode, const double *d_pos, const double *d_w,
                        double *d_hv, double *d_dq, double *d_dlj, cudaStream_t st) {
  const GridParams &g = c->g;
  const size_t nt4 = (size_t)c->ntypes * c->ntypes * 4;
  const int n = c->n;
  // a Hessian-vector product asked for neither parameter derivative skips them
  const bool params = mode == DERIV_PARAMS || d_dq || d_dlj;
  const bool half = !params || c->ntypes <= kDerivRegTypes;
  const int blocks = half ? g.ncell * kDerivSlots : (g.ncell + 3) / 4;
  if (params) {
    if (c->tpart_alloc < (size_t)blocks * nt4) {
      CK(dalloc(c->d_tpart, (size_t)blocks * nt4));
      c->tpart_alloc = (size_t)blocks * nt4;
    }
    if (!d_dq) {
      if (c->gq_alloc < (size_t)std::max(n, 1)) {
        CK(dalloc(c->d_gq, (size_t)std::max(n, 1)));
        c->gq_alloc = (size_t)std::max(n, 1);
      }
      d_dq = c->d_gq;
    }
    if (!d_dlj) {
      if (c->glj_alloc < nt4) {
        CK(dalloc(c->d_glj, nt4));
        c->glj_alloc = nt4;
      }
      d_dlj = c->d_glj;
    }
  }
  if (mode == DERIV_VJP && c->ws_alloc < (size_t)std::max(n, 1)) {
    CK(dalloc(c->d_wsorted, (size_t)std::max(n, 1)));
    c->ws_alloc = (size_t)std::max(n, 1);
  }
  // the half-shell kernel sums into the fixed-point accumulator, which the
  // cell build clears (hv words 0-5, dq words 6-7)
  launch_cell_build(c, d_pos, false, false, st, half ? c->d_facc : nullptr, params ? 8 : 6);
  if (mode == DERIV_VJP && n > 0)
    k_gather_sorted<<<(n + 255) / 256, 256, 0, st>>>(n, c->d_sidx, d_w, c->d_wsorted);
  if (half && n == 0) {
    if (params) CK(cudaMemsetAsync(d_dlj, 0, sizeof(double) * nt4, st));
  } else if (half) {
#define PMB_DERIV_HALF(M, P)                                                                 \
  k_deriv_fp64_half<M, P><<<(unsigned)blocks, 32, 0, st>>>(                                 \
      g, c->fc, c->half, kDerivSlots, c->ntypes, c->d_lj64, c->d_start, c->d_spos64,         \
      c->d_smeta, c->d_sidx, c->d_ex_start, c->d_ex, c->d_wsorted, c->d_facc, n, c->d_tpart, \
      c->d_err)
    if (mode == DERIV_PARAMS) PMB_DERIV_HALF(DERIV_PARAMS, true);
    else if (params) PMB_DERIV_HALF(DERIV_VJP, true);
    else PMB_DERIV_HALF(DERIV_VJP, false);
#undef PMB_DERIV_HALF
    if (mode == DERIV_VJP)
      k_finalize64<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, c->d_facc, c->d_sidx, 0,
                                                                 d_hv);
    if (params)
      k_finalize_q<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, c->d_facc, c->d_sidx, d_dq);
  } else {
    const size_t smem = sizeof(double) * nt4;
    if (mode == DERIV_PARAMS)
      k_deriv_fp64<DERIV_PARAMS><<<blocks, 128, smem, st>>>(
          g, c->fc, c->stencil, c->ntypes, c->d_lj64, c->d_start, c->d_spos64, c->d_smeta,
          c->d_sidx, c->d_ex_start, c->d_ex, nullptr, nullptr, d_dq, c->d_tpart);
    else
      k_deriv_fp64<DERIV_VJP, true><<<blocks, 128, smem, st>>>(
          g, c->fc, c->stencil, c->ntypes, c->d_lj64, c->d_start, c->d_spos64, c->d_smeta,
          c->d_sidx, c->d_ex_start, c->d_ex, c->d_wsorted, d_hv, d_dq, c->d_tpart);
  }
  if (params && !(half && n == 0))
    k_reduce_columns<<<(unsigned)nt4, 256, 0, st>>>(blocks, (int)nt4, c->d_tpart, d_dlj);
  CK(cudaGetLastError());
  return PMB200_OK;
}

static int deriv_ready(pmb200_ctx *c) {
  int rc = check_ready(c);
  if (rc) return rc;
  if (c->form != FORM_CUTOFF)
    return fail(c, PMB200_EUNSUPPORTED, "derivative kernels cover the cutoff LJ + Coulomb force");
  // the table derivatives are summed per block in shared memory (48 KB)
  if (sizeof(double) * 4 * (size_t)c->ntypes * c->ntypes > 48 * 1024)
    return fail(c, PMB200_EUNSUPPORTED, "derivative kernels: at most 39 LJ types (%d given)",
                c->ntypes);
  return PMB200_OK;
}

int pmb200_param_grad_device(pmb200_ctx *c, const double *d_pos, double *d_dq, double *d_dlj,
                             void *stream) {
  int rc = deriv_ready(c);
  if (rc) return rc;
  if (c->n > 0 && (!d_pos || !d_dq)) return fail(c, PMB200_EINVAL, "null device buffer");
  if (!d_dlj) return fail(c, PMB200_EINVAL, "null device buffer");
  CK(cudaSetDevice(c->p.device));
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  return launch_deriv(c, DERIV_PARAMS, d_pos, nullptr, nullptr, d_dq, d_dlj, st);
}

int pmb200_hvp_device(pmb200_ctx *c, const double *d_pos, const double *d_w, double *d_hv,
                      double *d_dq, double *d_dlj, void *stream) {
  int rc = deriv_ready(c);
  if (rc) return rc;
  if (c->n > 0 && (!d_pos || !d_w || !d_hv)) return fail(c, PMB200_EINVAL, "null device buffer");
  CK(cudaSetDevice(c->p.device));
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  return launch_deriv(c, DERIV_VJP, d_pos, d_w, d_hv, d_dq, d_dlj, st);
}

int pmb200_update_params(pmb200_ctx *c, const double *q_scaled, const double *lj) {
  if (!c) return PMB200_EINVAL;
  if (!c->have_topo) return fail(c, PMB200_ESTATE, "pmb200_set_topology has not been called");
  CK(cudaSetDevice(c->p.device));
  if (q_scaled) {
    for (int i = 0; i < c->n; i++)
      if (!std::isfinite(q_scaled[i])) return fail(c, PMB200_EINVAL, "atom %d: charge", i);
    if (c->n > 0)
      CK(cudaMemcpy(c->d_q, q_scaled, sizeof(double) * c->n, cudaMemcpyHostToDevice));
  }
  if (lj) {
    const int t4 = 4 * c->ntypes * c->ntypes;
    for (int k = 0; k < t4; k++)
      if (!std::isfinite(lj[k])) return fail(c, PMB200_EINVAL, "LJ table entry %d", k);
    c->h_lj.assign(lj, lj + t4);
    c->lj_dev_newer = false;
    if (c->have_box) return upload_lj(c);
  }
  return PMB200_OK;
}

// Parameters from device buffers: charges copied, the table copied to the
// FP64 table and scaled into the FP32 one (the quotients upload_lj takes);
// a non-finite value sets error bit 4.
__global__ void k_update_q(int n, const double *__restrict__ src, double *__restrict__ dst,
                           int *__restrict__ err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double v = src[i];
  if (!isfinite(v)) atomicOr(err, 4);
  dst[i] = v;
}

__global__ void k_update_lj(int t2, const double *__restrict__ src, double u6, double u12,
                            double4 *__restrict__ lj64, float4 *__restrict__ lj32,
                            int *__restrict__ err) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= t2) return;
  const double a = src[4 * k], b = src[4 * k + 1], a14 = src[4 * k + 2], b14 = src[4 * k + 3];
  if (!(isfinite(a) && isfinite(b) && isfinite(a14) && isfinite(b14))) atomicOr(err, 4);
  lj64[k] = make_double4(a, b, a14, b14);
  lj32[k] = make_float4((float)(a / u12), (float)(b / u6), (float)(a14 / u12), (float)(b14 / u6));
}

int pmb200_update_params_device(pmb200_ctx *c, const double *d_q_scaled, const double *d_lj,
                                void *stream) {
  if (!c) return PMB200_EINVAL;
  if (!c->have_topo) return fail(c, PMB200_ESTATE, "pmb200_set_topology has not been called");
  if (d_lj && !c->have_box)
    return fail(c, PMB200_ESTATE, "a device LJ table needs the box (pmb200_set_box)");
  CK(cudaSetDevice(c->p.device));
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  if (d_q_scaled && c->n > 0)
    k_update_q<<<(c->n + 255) / 256, 256, 0, st>>>(c->n, d_q_scaled, c->d_q, c->d_err);
  if (d_lj) {
    const int t2 = c->ntypes * c->ntypes;
    const double u6 = std::pow(c->g.unit, 6.0), u12 = u6 * u6;
    k_update_lj<<<(t2 + 127) / 128, 128, 0, st>>>(t2, d_lj, u6, u12, c->d_lj64, c->d_lj32,
                                                  c->d_err);
    if (!c->ev_lj) CK(cudaEventCreateWithFlags(&c->ev_lj, cudaEventDisableTiming));
    CK(cudaEventRecord(c->ev_lj, st));
    c->lj_dev_newer = true;
  }
  CK(cudaGetLastError());
  return PMB200_OK;
}

// The device error flag's value e (read after the work that set it has
// finished): clears the flag and reports.
static int device_error(pmb200_ctx *c, int e) {
  if (!e) return PMB200_OK;
  CK(cudaMemset(c->d_err, 0, sizeof(int)));
  if (e & 1) return fail(c, PMB200_EDEVICE, "non-finite atom position in an evaluation");
  if (e & 4) return fail(c, PMB200_EDEVICE, "non-finite charge or LJ table entry (device update)");
  if (e & 8)
    return fail(c, PMB200_EDEVICE, "supercluster kernel: a cluster list exceeded %d entries "
                "(atoms packed denser than the kernel supports; use PMB200_KERNEL_SEARCH)",
                kScCap);
  if (e & (16 | 32))
    return fail(c, PMB200_EDEVICE, "supercluster kernel: a supercluster is taller than the box "
                "allows for a unique periodic image (sparse system; use PMB200_KERNEL_SEARCH)");
  return fail(c, PMB200_EDEVICE,
              "a pair term exceeded the fixed-point accumulator's range (atoms overlap)");
}

int pmb200_sync(pmb200_ctx *c) {
  if (!c) return PMB200_EINVAL;
  CK(cudaSetDevice(c->p.device));
  CK(cudaStreamSynchronize(c->stream));
  int e = 0;
  CK(cudaMemcpy(&e, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  return device_error(c, e);
}

int pmb200_eval(pmb200_ctx *c, const double *pos, double *forces, double *energies,
                double *virial, double *molvirial, unsigned flags) {
  int rc = check_ready(c);
  if (rc) return rc;
  if (c->n > 0 && (!pos || !forces)) return fail(c, PMB200_EINVAL, "null host buffer");
  if ((flags & PMB200_ENERGY) && !energies) return fail(c, PMB200_EINVAL, "null energies");
  if ((flags & PMB200_VIRIAL) && !virial) return fail(c, PMB200_EINVAL, "null virial");
  if ((flags & PMB200_MOLVIRIAL) && !molvirial) return fail(c, PMB200_EINVAL, "null molvirial");
  if ((flags & PMB200_MOLVIRIAL) && !c->have_mass)
    return fail(c, PMB200_EINVAL, "molecular virial needs masses");
  CK(cudaSetDevice(c->p.device));
  const size_t cnt = 3 * (size_t)c->n;
  const size_t bytes = sizeof(double) * cnt;
  cudaStream_t st = c->stream;
  if (c->n_pin < c->n || !c->h_pin_out) {
    release_graph(c);  // the evaluation graph copies through these buffers
    if (c->h_pin_pos) cudaFreeHost(c->h_pin_pos);
    if (c->h_pin_frc) cudaFreeHost(c->h_pin_frc);
    if (c->h_pin_out) cudaFreeHost(c->h_pin_out);
    c->h_pin_pos = c->h_pin_frc = c->h_pin_out = nullptr;
    CK(cudaMallocHost((void **)&c->h_pin_pos, std::max<size_t>(bytes, 8)));
    CK(cudaMallocHost((void **)&c->h_pin_frc, bytes + sizeof(double) * (kPinOut + 3)));
    CK(cudaMallocHost((void **)&c->h_pin_out, sizeof(double) * kPinOut));
    c->n_pin = c->n;
  }
  // the results travel behind the forces in one copy: d_hfrc holds the 3n
  // forces, then the 20 result words, then the device error flag
  double *d_hout = c->d_hfrc + cnt;
  const size_t res_bytes = bytes + sizeof(double) * kPinOut;
  bool f32out = false;  // FP32 forces back this call (set below)
  // positions through pinned staging; this evaluation's forces are computed
  // on the device (overwrite), read back, and added to the caller's array
  if (c->n > 0) {
    // page-locked caller arrays are transferred directly; pageable ones go
    // through the pinned staging copy, made on the host's cores
    // FP32 forces back for mixed contexts (see k_pack_out)
    f32out = c->p.precision == PMB200_MIXED;
    cudaPointerAttributes attr{};
    const bool pinned = cudaPointerGetAttributes(&attr, pos) == cudaSuccess &&
                        attr.type == cudaMemoryTypeHost;
    cudaGetLastError();  // a pageable pointer may leave an error behind
    const double *src = pos;
    if (!pinned) {
      const long long chunks = (long long)((cnt + 8191) / 8192);
#pragma omp parallel for schedule(static) if (chunks > 8)
      for (long long b = 0; b < chunks; b++) {
        const size_t lo = (size_t)b * 8192, m = std::min<size_t>(8192, cnt - lo);
        std::memcpy(c->h_pin_pos + lo, pos + lo, sizeof(double) * m);
      }
      src = c->h_pin_pos;
    }
    // copy in, evaluate, copy out: one graph per (source array, flags),
    // replayed while the context's box and topology stay the same (the
    // pair-kernel timing mode launches directly).  The results and the
    // error flag follow the forces in d_hfrc, so one copy brings all back.
    const size_t f32_slots = (cnt + 1) & ~(size_t)1;  // FP32 forces, to a double boundary
    const size_t res32_bytes = sizeof(float) * f32_slots + sizeof(double) * kPinOut;
    auto sequence = [&]() -> int {
      const unsigned eb = (unsigned)((cnt + 255) / 256);
      cudaError_t e = cudaMemcpyAsync(c->d_hpos, src, bytes, cudaMemcpyHostToDevice, st);
      if (e != cudaSuccess) return fail(c, PMB200_ECUDA, "copy in: %s", cudaGetErrorString(e));
      // (a mixed energy evaluation packs the FP32 forces, results and error
      // flag itself)
      double *tail = reinterpret_cast<double *>(c->d_hf32 + f32_slots);
      bool packed = false;
      int r = launch_eval(c, c->d_hpos, c->d_hfrc, d_hout, flags, 0, st,
                          f32out ? c->d_hf32 : nullptr, tail, &packed);
      if (r) return r;
      if (packed) {
        e = cudaMemcpyAsync(c->h_pin_frc, c->d_hf32, res32_bytes, cudaMemcpyDeviceToHost, st);
      } else if (f32out) {
        // (the error flag goes into the packed copy's tail)
        k_pack_out<<<eb, 256, 0, st>>>(cnt, c->d_hfrc, d_hout, c->d_err, c->d_hf32);
        e = cudaGetLastError();
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(c->h_pin_frc, c->d_hf32, res32_bytes, cudaMemcpyDeviceToHost, st);
      } else {
        k_copy_word<<<1, 1, 0, st>>>(c->d_err, reinterpret_cast<int *>(d_hout + 20));
        e = cudaGetLastError();
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(c->h_pin_frc, c->d_hfrc, res_bytes, cudaMemcpyDeviceToHost, st);
      }
      if (e != cudaSuccess) return fail(c, PMB200_ECUDA, "copy out: %s", cudaGetErrorString(e));
      return PMB200_OK;
    };
    if (c->timing) {
      rc = sequence();
      if (rc) return rc;
    } else {
      const unsigned gkey = flags | (f32out ? 0x80000000u : 0u);
      if (!c->hgraph_exec || c->hgraph_src != src || c->hgraph_flags != gkey) {
        if (c->hgraph_exec) cudaGraphExecDestroy(c->hgraph_exec);
        if (c->hgraph) cudaGraphDestroy(c->hgraph);
        c->hgraph_exec = nullptr;
        c->hgraph = nullptr;
        c->hgraph_src = nullptr;
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        rc = sequence();
        cudaGraph_t gr = nullptr;
        const cudaError_t e = cudaStreamEndCapture(st, &gr);
        if (rc) {
          if (gr) cudaGraphDestroy(gr);
          return rc;
        }
        if (e != cudaSuccess) return fail(c, PMB200_ECUDA, "capture: %s", cudaGetErrorString(e));
        c->hgraph = gr;
        CK(cudaGraphInstantiate(&c->hgraph_exec, gr, 0));
        c->hgraph_src = src;
        c->hgraph_flags = gkey;
      }
      rc = ensure_clear(c, st);
      if (rc) return rc;
      CK(cudaGraphLaunch(c->hgraph_exec, st));
    }
  } else {
    rc = launch_eval(c, c->d_hpos, c->d_hfrc, d_hout, flags, 0, st);
    if (rc) return rc;
    k_copy_word<<<1, 1, 0, st>>>(c->d_err, reinterpret_cast<int *>(d_hout + 20));
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->h_pin_frc, d_hout, sizeof(double) * kPinOut, cudaMemcpyDeviceToHost,
                       st));
  }
  // the error flag came back with the results: one synchronisation
  CK(cudaStreamSynchronize(st));
  const size_t res_at = f32out ? ((cnt + 1) & ~(size_t)1) / 2 : cnt;  // (in doubles)
  const double *out = c->h_pin_frc + res_at;
  rc = device_error(c, *reinterpret_cast<const int *>(out + 20));
  if (rc) return rc;
  {
    const long long m = (long long)cnt;
    if (f32out) {
      const float *src = reinterpret_cast<const float *>(c->h_pin_frc);
#pragma omp parallel for schedule(static) if (m > 65536)
      for (long long k = 0; k < m; k++) forces[k] += (double)src[k];
    } else {
      const double *src = c->h_pin_frc;
#pragma omp parallel for schedule(static) if (m > 65536)
      for (long long k = 0; k < m; k++) forces[k] += src[k];
    }
  }
  if (flags & PMB200_ENERGY) {
    energies[0] += out[0];
    energies[1] += out[1];
  }
  if (flags & PMB200_VIRIAL)
    for (int k = 0; k < 9; k++) virial[k] += out[2 + k];
  if (flags & PMB200_MOLVIRIAL)
    for (int k = 0; k < 9; k++) molvirial[k] += out[11 + k];
  return PMB200_OK;
}

// Host-buffer evaluation of the pairs whose i-cell lies in [cell_lo,
// cell_hi): the share of one block range of the reference's
// parallelEvaluate.  Direct launches (no graph); forces, energies and
// virials are accumulated into the caller's arrays.
int pmb200_eval_cells(pmb200_ctx *c, const double *pos, double *forces, double *energies,
                      double *virial, double *molvirial, unsigned flags, int cell_lo,
                      int cell_hi) {
  int rc = check_ready(c);
  if (rc) return rc;
  if (cell_lo < 0 || cell_hi < cell_lo || cell_hi > c->g.ncell)
    return fail(c, PMB200_EINVAL, "cell range [%d, %d) of %d cells", cell_lo, cell_hi,
                c->g.ncell);
  if (c->n > 0 && (!pos || !forces)) return fail(c, PMB200_EINVAL, "null host buffer");
  if ((flags & PMB200_ENERGY) && !energies) return fail(c, PMB200_EINVAL, "null energies");
  if ((flags & PMB200_VIRIAL) && !virial) return fail(c, PMB200_EINVAL, "null virial");
  if ((flags & PMB200_MOLVIRIAL) && !molvirial) return fail(c, PMB200_EINVAL, "null molvirial");
  if ((flags & PMB200_MOLVIRIAL) && !c->have_mass)
    return fail(c, PMB200_EINVAL, "molecular virial needs masses");
  if (cell_hi == cell_lo || c->n == 0) return PMB200_OK;  // nothing in this share
  CK(cudaSetDevice(c->p.device));
  const size_t cnt = 3 * (size_t)c->n;
  const size_t bytes = sizeof(double) * cnt;
  cudaStream_t st = c->stream;
  if (c->n_pin < c->n || !c->h_pin_out) {
    release_graph(c);  // the host-buffer graph copies through these buffers
    if (c->h_pin_pos) cudaFreeHost(c->h_pin_pos);
    if (c->h_pin_frc) cudaFreeHost(c->h_pin_frc);
    if (c->h_pin_out) cudaFreeHost(c->h_pin_out);
    c->h_pin_pos = c->h_pin_frc = c->h_pin_out = nullptr;
    CK(cudaMallocHost((void **)&c->h_pin_pos, std::max<size_t>(bytes, 8)));
    CK(cudaMallocHost((void **)&c->h_pin_frc, std::max<size_t>(bytes, 8)));
    CK(cudaMallocHost((void **)&c->h_pin_out, sizeof(double) * kPinOut));
    c->n_pin = c->n;
  }
  int *h_err = reinterpret_cast<int *>(c->h_pin_out + 20);
  std::memcpy(c->h_pin_pos, pos, bytes);
  CK(cudaMemcpyAsync(c->d_hpos, c->h_pin_pos, bytes, cudaMemcpyHostToDevice, st));
  const bool mixed = c->p.precision == PMB200_MIXED;
  const bool energy = (flags & PMB200_ENERGY) != 0;
  const bool anyvir = (flags & (PMB200_VIRIAL | PMB200_MOLVIRIAL)) != 0;
  const GridParams &g = c->g;
  const int nc = cell_hi - cell_lo;
  launch_cell_build(c, c->d_hpos, mixed, mixed && energy && c->form == FORM_CUTOFF, st,
                    mixed ? c->d_facc : nullptr);
  if ((flags & PMB200_MOLVIRIAL) && c->nmol > 0)
    k_com<<<(c->nmol + 127) / 128, 128, 0, st>>>(c->nmol, c->d_mstart, c->d_matoms, c->d_mass,
                                                  c->d_hpos, c->d_com);
  int rows = nc;
  double *prow = c->d_partial;
  if (mixed) {
    if (c->form == FORM_GENERIC) launch_pair_mixed<FORM_GENERIC>(c, flags, st, cell_lo, nc);
    else if (c->form == FORM_EWALD_POLY5)
      launch_pair_mixed<FORM_EWALD_POLY5>(c, flags, st, cell_lo, nc);
    else if (c->form == FORM_EWALD_EXACT)
      launch_pair_mixed<FORM_EWALD_EXACT>(c, flags, st, cell_lo, nc);
    else launch_pair_mixed<FORM_CUTOFF>(c, flags, st, cell_lo, nc);
    k_finalize<<<(c->n + 255) / 256, 256, 0, st>>>(c->n, c->d_facc, c->d_sidx,
                                                  kFixInv / g.unit, 0, c->d_hfrc);
    rows = nc * ctx_slots(c, true);
  } else {
    CK(cudaMemsetAsync(c->d_hfrc, 0, bytes, st));
    const int blocks = (nc + 3) / 4;
    if (c->form == FORM_GENERIC)
      launch_pair_fp64<FORM_GENERIC>(c, flags, c->d_hfrc, 1, blocks, st, cell_lo, nc);
    else if (c->form == FORM_EWALD_POLY5)
      launch_pair_fp64<FORM_EWALD_POLY5>(c, flags, c->d_hfrc, 1, blocks, st, cell_lo, nc);
    else if (c->form == FORM_EWALD_EXACT)
      launch_pair_fp64<FORM_EWALD_EXACT>(c, flags, c->d_hfrc, 1, blocks, st, cell_lo, nc);
    else launch_pair_fp64<FORM_CUTOFF>(c, flags, c->d_hfrc, 1, blocks, st, cell_lo, nc);
    prow = c->d_partial + (size_t)cell_lo * kNacc;  // the FP64 kernel's rows are by cell
  }
  CK(cudaGetLastError());
  if (energy || anyvir) {
    const int ns = anyvir ? ACC_MV : ACC_E;
    k_reduce1<<<kRedBlocks, 256, 0, st>>>(rows, prow, c->d_red, ns);
    k_reduce2<<<1, 256, 0, st>>>(kRedBlocks, c->d_red, mixed ? 1.0 : 0.5, c->d_out,
                                c->d_pairs, ns);
    CK(cudaMemcpyAsync(c->h_pin_out, c->d_out, sizeof(double) * 20, cudaMemcpyDeviceToHost,
                       st));
  }
  CK(cudaMemcpyAsync(c->h_pin_frc, c->d_hfrc, bytes, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(h_err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  rc = device_error(c, *h_err);
  if (rc) return rc;
  for (size_t k = 0; k < cnt; k++) forces[k] += c->h_pin_frc[k];
  const double *out = c->h_pin_out;
  if (flags & PMB200_ENERGY) {
    energies[0] += out[0];
    energies[1] += out[1];
  }
  if (flags & PMB200_VIRIAL)
    for (int k = 0; k < 9; k++) virial[k] += out[2 + k];
  if (flags & PMB200_MOLVIRIAL)
    for (int k = 0; k < 9; k++) molvirial[k] += out[11 + k];
  return PMB200_OK;
}

int pmb200_leapfrog_device(pmb200_ctx *c, double *d_pos, double *d_vel, double *d_forces,
                           double *d_out, double dt_fs, int nsteps, unsigned flags,
                           void *stream) {
  int rc = check_ready(c);
  if (rc) return rc;
  if (!c->have_mass) return fail(c, PMB200_EINVAL, "leapfrog needs masses");
  if (nsteps < 1) return PMB200_OK;
  if (!(dt_fs > 0.0)) return fail(c, PMB200_EINVAL, "time step %g", dt_fs);
  if (c->n > 0 && (!d_pos || !d_vel || !d_forces))
    return fail(c, PMB200_EINVAL, "null device buffer");
  CK(cudaSetDevice(c->p.device));
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  const double h = dt_fs * 0.02045482828087295;  // Constant::INV_TIMEFACTOR
  const int n = c->n;
  const int tb = 256, nb = (3 * n + tb - 1) / tb;
  // initial forces, then the first (half-kick) step
  rc = launch_eval(c, d_pos, d_forces, nullptr, 0, 0, st);
  if (rc) return rc;
  auto step = [&](double kick, unsigned fl) -> int {
    launch_kick_drift(c, d_pos, d_vel, d_forces, kick * h, h, st);
    return launch_eval(c, d_pos, d_forces, d_out, fl, 0, st);
  };
  rc = step(0.5, nsteps == 1 ? flags : 0);
  if (rc) return rc;
  const int middle = nsteps - 2;  // steps 2..nsteps-1 replay one captured graph
  if (middle > 0) {
    const void *key[4] = {d_pos, d_vel, d_forces, (const void *)st};
    bool same = c->graph_exec && c->graph_dt == dt_fs;
    for (int k = 0; k < 4 && same; k++) same = c->graph_key[k] == key[k];
    if (!same) {
      release_graph(c);
      CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      rc = step(1.0, 0);
      cudaGraph_t gr = nullptr;
      cudaError_t e = cudaStreamEndCapture(st, &gr);
      if (rc) {
        if (gr) cudaGraphDestroy(gr);
        return rc;
      }
      if (e != cudaSuccess) return fail(c, PMB200_ECUDA, "capture: %s", cudaGetErrorString(e));
      c->graph = gr;
      CK(cudaGraphInstantiate(&c->graph_exec, gr, 0));
      for (int k = 0; k < 4; k++) c->graph_key[k] = key[k];
      c->graph_dt = dt_fs;
    }
    rc = ensure_clear(c, st);
    if (rc) return rc;
    for (int s = 0; s < middle; s++) CK(cudaGraphLaunch(c->graph_exec, st));
  }
  if (nsteps >= 2) {
    rc = step(1.0, flags);
    if (rc) return rc;
  }
  if (n > 0)
    k_kick_drift<<<nb, tb, 0, st>>>(n, d_pos, d_vel, d_forces, c->d_mass, 0.5 * h, h, 0);
  CK(cudaGetLastError());
  return PMB200_OK;
}

int pmb200_step_device(pmb200_ctx *c, double *d_pos, double *d_vel, double *d_forces,
                       double *d_out, double dt_fs, unsigned flags, void *stream) {
  int rc = check_ready(c);
  if (rc) return rc;
  if (!c->have_mass) return fail(c, PMB200_EINVAL, "leapfrog needs masses");
  if (!(dt_fs > 0.0)) return fail(c, PMB200_EINVAL, "time step %g", dt_fs);
  if (c->n > 0 && (!d_pos || !d_vel || !d_forces))
    return fail(c, PMB200_EINVAL, "null device buffer");
  if (!stream) return fail(c, PMB200_EINVAL, "pmb200_step_device needs an explicit stream");
  if ((flags & PMB200_MOLVIRIAL)) return fail(c, PMB200_EINVAL, "molecular virial in a step");
  CK(cudaSetDevice(c->p.device));
  cudaStream_t st = (cudaStream_t)stream;
  const void *key[5] = {d_pos, d_vel, d_forces, d_out, stream};
  bool same = c->sgraph_exec && c->sgraph_dt == dt_fs && c->sgraph_flags == flags;
  for (int k = 0; k < 5 && same; k++) same = c->sgraph_key[k] == key[k];
  if (!same) {
    if (c->sgraph_exec) cudaGraphExecDestroy(c->sgraph_exec);
    if (c->sgraph) cudaGraphDestroy(c->sgraph);
    c->sgraph_exec = nullptr;
    c->sgraph = nullptr;
    const double h = dt_fs * 0.02045482828087295;  // Constant::INV_TIMEFACTOR
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    launch_kick_drift(c, d_pos, d_vel, d_forces, h, h, st);
    rc = launch_eval(c, d_pos, d_forces, d_out, flags, 0, st);
    cudaGraph_t gr = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &gr);
    if (rc) {
      if (gr) cudaGraphDestroy(gr);
      return rc;
    }
    if (e != cudaSuccess) return fail(c, PMB200_ECUDA, "capture: %s", cudaGetErrorString(e));
    c->sgraph = gr;
    CK(cudaGraphInstantiate(&c->sgraph_exec, gr, 0));
    for (int k = 0; k < 5; k++) c->sgraph_key[k] = key[k];
    c->sgraph_dt = dt_fs;
    c->sgraph_flags = flags;
  }
  rc = ensure_clear(c, st);
  if (rc) return rc;
  CK(cudaGraphLaunch(c->sgraph_exec, st));
  return PMB200_OK;
}

int pmb200_set_rigid_waters(pmb200_ctx *c, int nwater, const int *widx, double d_oh,
                            double d_hh) {
  if (!c) return PMB200_EINVAL;
  if (!c->have_topo) return fail(c, PMB200_ESTATE, "pmb200_set_topology has not been called");
  if (nwater < 0 || (nwater > 0 && !widx)) return fail(c, PMB200_EINVAL, "water list");
  if (nwater > 0 && !c->have_mass) return fail(c, PMB200_EINVAL, "rigid waters need masses");
  if (nwater > 0 && !(d_oh > 0.0 && d_hh > 0.0 && d_hh < 2.0 * d_oh))
    return fail(c, PMB200_EINVAL, "constraint lengths O-H %g, H-H %g", d_oh, d_hh);
  CK(cudaSetDevice(c->p.device));
  release_graph(c);
  std::vector<char> used(c->n, 0);
  std::vector<double> mass(c->n);
  if (c->n > 0 && nwater > 0)
    CK(cudaMemcpy(mass.data(), c->d_mass, sizeof(double) * c->n, cudaMemcpyDeviceToHost));
  for (int w = 0; w < 3 * nwater; w++) {
    const int a = widx[w];
    if (a < 0 || a >= c->n) return fail(c, PMB200_EINVAL, "water atom index %d", a);
    if (used[a]) return fail(c, PMB200_EINVAL, "atom %d in two waters", a);
    used[a] = 1;
  }
  for (int w = 0; w < nwater; w++) {  // every water shares the first one's masses
    if (mass[widx[3 * w]] != mass[widx[0]] || mass[widx[3 * w + 1]] != mass[widx[1]] ||
        mass[widx[3 * w + 2]] != mass[widx[1]])
      return fail(c, PMB200_EINVAL, "water %d: masses differ from the first water's", w);
  }
  std::vector<int> fidx;
  for (int i = 0; i < c->n; i++)
    if (!used[i]) fidx.push_back(i);
  c->nwater = nwater;
  c->nfree = (int)fidx.size();
  if (nwater > 0) {
    CK(dalloc(c->d_widx, 3 * (size_t)nwater));
    CK(cudaMemcpy(c->d_widx, widx, sizeof(int) * 3 * nwater, cudaMemcpyHostToDevice));
    CK(dalloc(c->d_fidx, std::max<size_t>(fidx.size(), 1)));
    if (!fidx.empty())
      CK(cudaMemcpy(c->d_fidx, fidx.data(), sizeof(int) * fidx.size(), cudaMemcpyHostToDevice));
    const double mo = mass[widx[0]], mh = mass[widx[1]];
    const double rcv = 0.5 * d_hh, t = std::sqrt(d_oh * d_oh - rcv * rcv);
    c->sp.mo = mo;
    c->sp.mh = mh;
    c->sp.rc = rcv;
    c->sp.ra = 2.0 * mh * t / (mo + 2.0 * mh);
    c->sp.rb = t - c->sp.ra;
  }
  return PMB200_OK;
}

int pmb200_set_kernel_timing(pmb200_ctx *c, int on) {
  if (!c) return PMB200_EINVAL;
  c->timing = on ? 1 : 0;
  return PMB200_OK;
}

int pmb200_last_kernel_ms(pmb200_ctx *c, float *ms) {
  if (!c || !ms) return PMB200_EINVAL;
  CK(cudaSetDevice(c->p.device));
  CK(cudaEventElapsedTime(ms, c->ev0, c->ev1));
  return PMB200_OK;
}

int pmb200_last_pair_count(pmb200_ctx *c, long long *pairs) {
  if (!c || !pairs) return PMB200_EINVAL;
  double v = 0.0;
  CK(cudaSetDevice(c->p.device));
  CK(cudaMemcpy(&v, c->d_pairs, sizeof(double), cudaMemcpyDeviceToHost));
  *pairs = (long long)llround(v);
  return PMB200_OK;
}

// SETTLE on the host (the algorithm of settle_water on the device) for kW
// waters at once, structure of arrays: X0 the pre-step positions, X1 the
// unconstrained new ones (in) and the constrained ones (out), rows
// {O, H1, H2} x {x, y, z}.  Every loop runs over the lanes with no
// dependence between them, so it vectorises; the waters' dependency chains
// (seven square roots and divisions each) overlap.  Built for AVX-512 and
// AVX2 as well, picked at load time where the host has them (eight or four
// lanes per instruction instead of two); floating-point contraction is off
// in this build, so every host rounds alike.
constexpr int kW = 8;
__attribute__((target_clones("avx512f", "avx2", "default")))
static void host_settle_w(const SettleParams &sp, double inv_m, double inv_ra,
                          const double (&X0)[9][kW], double (&X1)[9][kW]) {
#define PMB_LANES _Pragma("omp simd") for (int l = 0; l < kW; l++)
  double com[3][kW], a1[3][kW], b1[3][kW], c1[3][kW], b0[3][kW], c0[3][kW];
  double ex[3][kW], ey[3][kW], ez[3][kW];
  for (int k = 0; k < 3; k++)
    PMB_LANES {
      com[k][l] = (sp.mo * X1[k][l] + sp.mh * X1[3 + k][l] + sp.mh * X1[6 + k][l]) * inv_m;
      a1[k][l] = X1[k][l] - com[k][l];
      b1[k][l] = X1[3 + k][l] - com[k][l];
      c1[k][l] = X1[6 + k][l] - com[k][l];
      b0[k][l] = X0[3 + k][l] - X0[k][l];
      c0[k][l] = X0[6 + k][l] - X0[k][l];
    }
  auto cross = [](const double a[3][kW], const double b[3][kW], double o[3][kW]) {
    PMB_LANES {
      o[0][l] = a[1][l] * b[2][l] - a[2][l] * b[1][l];
      o[1][l] = a[2][l] * b[0][l] - a[0][l] * b[2][l];
      o[2][l] = a[0][l] * b[1][l] - a[1][l] * b[0][l];
    }
  };
  auto unit = [](double a[3][kW]) {
    PMB_LANES {
      const double s = 1.0 / std::sqrt(a[0][l] * a[0][l] + a[1][l] * a[1][l] + a[2][l] * a[2][l]);
      a[0][l] *= s; a[1][l] *= s; a[2][l] *= s;
    }
  };
  auto dot = [](const double a[3][kW], const double b[3][kW], double o[kW]) {
    PMB_LANES o[l] = a[0][l] * b[0][l] + a[1][l] * b[1][l] + a[2][l] * b[2][l];
  };
  cross(b0, c0, ez);
  cross(a1, ez, ex);
  cross(ez, ex, ey);
  unit(ex); unit(ey); unit(ez);
  double xb0[kW], yb0[kW], xc0[kW], yc0[kW], za1[kW], xb1[kW], yb1[kW], zb1[kW], xc1[kW],
      yc1[kW], zc1[kW];
  dot(ex, b0, xb0); dot(ey, b0, yb0); dot(ex, c0, xc0); dot(ey, c0, yc0); dot(ez, a1, za1);
  dot(ex, b1, xb1); dot(ey, b1, yb1); dot(ez, b1, zb1);
  dot(ex, c1, xc1); dot(ey, c1, yc1); dot(ez, c1, zc1);
  double ya2[kW], xb2[kW], yb2[kW], yc2[kW], sth[kW], cth[kW];
  PMB_LANES {
    const double sphi = za1[l] * inv_ra, cphi = std::sqrt(1.0 - sphi * sphi);
    const double spsi = (zb1[l] - zc1[l]) / (2.0 * sp.rc * cphi);
    const double cpsi = std::sqrt(1.0 - spsi * spsi);
    ya2[l] = sp.ra * cphi;
    xb2[l] = -sp.rc * cpsi;
    const double t1 = -sp.rb * cphi, t2 = sp.rc * spsi * sphi;
    yb2[l] = t1 - t2;
    yc2[l] = t1 + t2;
    const double al = xb2[l] * (xb0[l] - xc0[l]) + yb0[l] * yb2[l] + yc0[l] * yc2[l];
    const double be = xb2[l] * (yc0[l] - yb0[l]) + xb0[l] * yb2[l] + xc0[l] * yc2[l];
    const double ga = xb0[l] * yb1[l] - xb1[l] * yb0[l] + xc0[l] * yc1[l] - xc1[l] * yc0[l];
    const double ab = al * al + be * be;
    sth[l] = (al * ga - be * std::sqrt(ab - ga * ga)) / ab;
    cth[l] = std::sqrt(1.0 - sth[l] * sth[l]);
  }
  for (int k = 0; k < 3; k++)
    PMB_LANES {
      const double xa3 = -ya2[l] * sth[l], ya3 = ya2[l] * cth[l];
      const double xb3 = xb2[l] * cth[l] - yb2[l] * sth[l];
      const double yb3 = xb2[l] * sth[l] + yb2[l] * cth[l];
      const double xc3 = -xb2[l] * cth[l] - yc2[l] * sth[l];
      const double yc3 = -xb2[l] * sth[l] + yc2[l] * cth[l];
      X1[k][l] = com[k][l] + xa3 * ex[k][l] + ya3 * ey[k][l] + za1[l] * ez[k][l];
      X1[3 + k][l] = com[k][l] + xb3 * ex[k][l] + yb3 * ey[k][l] + zb1[l] * ez[k][l];
      X1[6 + k][l] = com[k][l] + xc3 * ex[k][l] + yc3 * ey[k][l] + zc1[l] * ez[k][l];
    }
#undef PMB_LANES
}

int pmb200_host_kick_drift(int n, double *pos, double *vel, double *forces,
                           const double *mass, double dt_fs, double kick, int nwater,
                           const int *widx, double d_oh, double d_hh, int clear_forces) {
  if (n < 0 || (n > 0 && (!pos || !vel || !forces || !mass)) || !(dt_fs > 0.0))
    return PMB200_EINVAL;
  if (nwater < 0 || (nwater > 0 && !widx) || 3LL * nwater > n) return PMB200_EINVAL;
  const double h = dt_fs * 0.02045482828087295;  // Constant::INV_TIMEFACTOR
  // which atoms the rigid waters hold: each index in range and at most once,
  // checked before anything is written.  Strictly increasing indices (the
  // usual listing) are checked on all cores with no shared writes; when the
  // waters hold every atom nothing else is needed, otherwise the atoms they
  // hold are marked.  Any other order: the marks, one index at a time.
  static thread_local std::vector<unsigned char> in_water;
  bool mark = false;
  if (nwater > 0) {
    const int nw3 = 3 * nwater;
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad) if (nwater > 1024)
    for (int w = 0; w < nw3; w++) {
      const int a = widx[w];
      bad |= (a < 0 || a >= n || (w + 1 < nw3 && widx[w + 1] <= a)) ? 1 : 0;
    }
    mark = nw3 < n;
    if (bad) {
      in_water.assign((size_t)n, 0);
      for (int w = 0; w < nw3; w++) {
        const int a = widx[w];
        if (a < 0 || a >= n || in_water[a]) return PMB200_EINVAL;
        in_water[a] = 1;
      }
      mark = false;  // already marked
    } else if (mark) {
      in_water.assign((size_t)n, 0);
    }
  }
  const double kh = kick * h, inv_h = 1.0 / h;
  SettleParams sp{};
  double inv_m = 0.0, inv_ra = 0.0;
  if (nwater > 0) {
    const double mo = mass[widx[0]], mh = mass[widx[1]];
    const double rcv = 0.5 * d_hh, t = std::sqrt(d_oh * d_oh - rcv * rcv);
    sp.mo = mo; sp.mh = mh; sp.rc = rcv;
    sp.ra = 2.0 * mh * t / (mo + 2.0 * mh);
    sp.rb = t - sp.ra;
    inv_m = 1.0 / (mo + 2.0 * mh);
    inv_ra = 1.0 / sp.ra;
  }
  const int ngroups = (nwater + kW - 1) / kW;  // kW waters per group
  const int nchunk = 3 * nwater < n ? (n + 4095) / 4096 : 0;  // atoms outside the waters
  unsigned char *inw = nchunk > 0 && nwater > 0 ? in_water.data() : nullptr;
#pragma omp parallel if (n > 4096)
  {
    if (mark) {  // distinct indices: no two threads write the same byte
#pragma omp for schedule(static)
      for (int w = 0; w < 3 * nwater; w++) inw[widx[w]] = 1;
    }
    // atoms outside the waters: kick and drift (independent per atom)
#pragma omp for schedule(static) nowait
    for (int cidx = 0; cidx < nchunk; cidx++) {
      const int i1 = std::min(n, (cidx + 1) * 4096);
      for (int i = cidx * 4096; i < i1; i++) {
        if (inw && inw[i]) continue;
        const double s = kh / mass[i];
        for (int k = 0; k < 3; k++) {
          const size_t q = 3 * (size_t)i + k;
          vel[q] += forces[q] * s;
          pos[q] += vel[q] * h;
          if (clear_forces) forces[q] = 0.0;
        }
      }
    }
    // one pass per group of waters: kick and drift into the group's arrays,
    // constrain, write the positions and take the velocities from the
    // constrained displacement; a short last group repeats its first water
    // in the spare lanes and writes only its own
#pragma omp for schedule(static)
    for (int gidx = 0; gidx < ngroups; gidx++) {
      const int w0 = gidx * kW, wn = std::min(kW, nwater - w0);
      double X0[9][kW], X1[9][kW];
      for (int l = 0; l < kW; l++)
        for (int m = 0; m < 3; m++) {
          const int a = widx[3 * (w0 + (l < wn ? l : 0)) + m];
          const double s = kh / mass[a];
          for (int k = 0; k < 3; k++) {
            const size_t q = 3 * (size_t)a + k;
            const double v = vel[q] + forces[q] * s;
            X0[3 * m + k][l] = pos[q];
            X1[3 * m + k][l] = pos[q] + v * h;
          }
        }
      if (clear_forces)  // after the gather: a short group reads its first water twice
        for (int l = 0; l < wn; l++)
          for (int m = 0; m < 3; m++)
            for (int k = 0; k < 3; k++) forces[3 * (size_t)widx[3 * (w0 + l) + m] + k] = 0.0;
      host_settle_w(sp, inv_m, inv_ra, X0, X1);
      for (int l = 0; l < wn; l++)
        for (int m = 0; m < 3; m++) {
          const int a = widx[3 * (w0 + l) + m];
          for (int k = 0; k < 3; k++) {
            const size_t q = 3 * (size_t)a + k;
            pos[q] = X1[3 * m + k][l];
            vel[q] = (X1[3 * m + k][l] - X0[3 * m + k][l]) * inv_h;
          }
        }
    }
  }
  return PMB200_OK;
}

int pmb200_measure_fp32_peak(int device, double *tflops) {
  pmb200_ctx *c = nullptr;
  if (!tflops) return PMB200_EINVAL;
  CK(cudaSetDevice(device));
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  float *sink = nullptr;
  CK(cudaMalloc((void **)&sink, sizeof(float) * 1024));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const int threads = 512, blocks = sms * 4, iters = 4096;
  k_fma_peak<<<blocks, threads>>>(64, 1.0f, sink);  // warm-up
  CK(cudaEventRecord(e0));
  k_fma_peak<<<blocks, threads>>>(iters, 1.0f, sink);
  CK(cudaEventRecord(e1));
  CK(cudaEventSynchronize(e1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  const double flops = 2.0 * 8.0 * 16.0 * (double)iters * threads * blocks;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return PMB200_OK;
}

// ---------------------------------------------------------------------------
// pmb200_eval_noalloc: the mixed-precision evaluation with every piece of
// scratch memory in one file-scope device array instead of cudaMalloc'd
// context buffers.  It exists for callers that must not allocate device
// memory: hosts that hand all device memory to their own pool allocator and
// forbid libraries to take more, or that cannot afford cudaFree's implicit
// device synchronisation inside their time step.  The array is sized for at
// most kNoAllocAtoms atoms and kNoAllocCells cells and stays resident on
// every device that loads this library until the process exits.
// ---------------------------------------------------------------------------
namespace {

constexpr int kNoAllocAtoms = 32768;
constexpr int kNoAllocCells = 8192;

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

struct NoAllocLayout {  // byte offsets inside the scratch array
  static constexpr size_t count = 0;
  static constexpr size_t start = align256(count + sizeof(int) * kNoAllocCells);
  static constexpr size_t partial = align256(start + sizeof(int) * (kNoAllocCells + 1));
  static constexpr size_t cell_of =
      align256(partial + sizeof(double) * kNoAllocCells * kEnergyCellSlots * kNacc);
  static constexpr size_t slot = align256(cell_of + sizeof(int) * kNoAllocAtoms);
  static constexpr size_t tmp = align256(slot + sizeof(int) * kNoAllocAtoms);
  static constexpr size_t sidx = align256(tmp + sizeof(int) * kNoAllocAtoms);
  static constexpr size_t rel32 = align256(sidx + sizeof(int) * kNoAllocAtoms);
  static constexpr size_t spos32 = align256(rel32 + sizeof(float4) * kNoAllocAtoms);
  static constexpr size_t smeta = align256(spos32 + sizeof(float4) * kNoAllocAtoms);
  static constexpr size_t facc = align256(smeta + sizeof(int2) * kNoAllocAtoms);
  static constexpr size_t red = align256(facc + sizeof(unsigned long long) * 3 * kNoAllocAtoms);
  static constexpr size_t rel_lo = align256(red + sizeof(double) * kRedBlocks * ACC_MV);
  static constexpr size_t spos_lo = align256(rel_lo + sizeof(float4) * kNoAllocAtoms);
  static constexpr size_t lj32 = align256(spos_lo + sizeof(float4) * kNoAllocAtoms);
  static constexpr size_t pairs = align256(lj32 + sizeof(float4) * kMaxTypes * kMaxTypes);
  static constexpr size_t err = align256(pairs + sizeof(double));
  // the final reduction's 20 doubles (energies, virial, molecular virial);
  // only the two energies are copied to the caller
  static constexpr size_t out = align256(err + sizeof(int));
  static constexpr size_t total = align256(out + sizeof(double) * 20);
};

// The LJ table travels as a kernel parameter (4 KB), so no host buffer is
// copied and nothing waits for the stream.
struct NoAllocLj {
  float4 v[kMaxTypes * kMaxTypes];
};

// Writes the call's LJ table into the scratch array and clears the device
// error word (one block).
__global__ void k_noalloc_setup(const NoAllocLj tbl, int nlj, float4 *__restrict__ dlj,
                                int *__restrict__ err) {
  for (int k = threadIdx.x; k < nlj; k += blockDim.x) dlj[k] = tbl.v[k];
  if (threadIdx.x == 0) *err = 0;
}

// The caller's status word: PMB200_OK, or PMB200_EDEVICE when a device-side
// check failed (non-finite coordinate, or a pair force beyond the
// fixed-point range).
__global__ void k_noalloc_status(const int *__restrict__ err, int *__restrict__ status) {
  *status = *err ? PMB200_EDEVICE : PMB200_OK;
}

// The scratch array itself.  Host code must not pass its name to a kernel
// (on the host it names a stand-in, not device memory); the device address
// comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NoAllocLayout::total];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
void *g_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once
// per device.
cudaError_t noalloc_scratch(unsigned char **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_addr[dev] = p;
  }
  *out = (unsigned char *)g_noalloc_addr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" int pmb200_eval_noalloc(const pmb200_params *p, int n, const double *d_pos,
                                   const int *d_type, const double *d_q, const int *d_mol,
                                   const int *d_ex_start, const int *d_ex_pairs, int ntypes,
                                   const double *lj, double coulomb_scaling, const double box[3],
                                   const double origin[3], double *d_forces, double *d_energy,
                                   int *d_status, void *stream) {
  // argument checks first: nothing reaches the device for a rejected call
  if (!p || !box || !origin || !lj) return PMB200_EINVAL;
  if (!std::isfinite(coulomb_scaling)) return PMB200_EINVAL;
  if (p->precision != PMB200_MIXED) return PMB200_EUNSUPPORTED;
  if (!(p->switchon >= 0.0) || !(p->cutoff_lj > 0.0) || !(p->switchon < p->cutoff_lj) ||
      !(p->cutoff_coul > 0.0) || !(p->cutoff_alg > 0.0))
    return PMB200_EINVAL;
  if (p->cutoff_alg < rc_max(*p)) return PMB200_EUNSUPPORTED;
  if (n < 0 || n > kNoAllocAtoms) return PMB200_ENOMEM;  // beyond the fixed scratch
  if (ntypes <= 0 || ntypes > kMaxTypes) return PMB200_EUNSUPPORTED;
  for (int k = 0; k < 4 * ntypes * ntypes; k++)
    if (!std::isfinite(lj[k])) return PMB200_EINVAL;
  if (n > 0 && (!d_pos || !d_type || !d_q || !d_mol || !d_ex_start || !d_ex_pairs || !d_forces))
    return PMB200_EINVAL;
  if (((uintptr_t)d_ex_pairs & 7u) != 0) return PMB200_EINVAL;  // read as int2
  const int2 *d_ex = (const int2 *)d_ex_pairs;
  const double rc = rc_max(*p);
  double L[3], edge[3];
  int nd[3];
  const double target = p->cellsize > 0.0 ? std::max(p->cellsize, rc / 3.0) : rc / 2.0;
  for (int a = 0; a < 3; a++) {
    L[a] = box[a];
    if (!(L[a] > 0.0) || !std::isfinite(L[a]) || !std::isfinite(origin[a])) return PMB200_EINVAL;
    if (L[a] < 2.0 * rc) return PMB200_EUNSUPPORTED;
    nd[a] = std::max(1, (int)std::floor(L[a] / target));
    edge[a] = L[a] / nd[a];
  }
  const long long ncell = (long long)nd[0] * nd[1] * nd[2];
  if (ncell > kNoAllocCells) return PMB200_ENOMEM;  // beyond the fixed scratch
  GridParams g{};
  g.periodic = 1;
  g.nx = nd[0]; g.ny = nd[1]; g.nz = nd[2];
  g.ncell = (int)ncell;
  for (int a = 0; a < 3; a++) {
    g.edge[a] = edge[a];
    g.boxlen[a] = L[a];
    g.boxmin[a] = origin[a] - 0.5 * L[a];
  }
  g.unit = edge[0];
  // half-shell neighbour cells (same rule as pmb200_set_box)
  HalfStencil half{};
  {
    int R[3];
    for (int a = 0; a < 3; a++) R[a] = (int)std::ceil(rc / edge[a] - 1e-12);
    const double rc2 = rc * rc * (1.0 + 1e-12);
    for (int dz = 0; dz <= R[2]; dz++)
      for (int dy = (dz == 0 ? 0 : -R[1]); dy <= R[1]; dy++) {
        const double yz = std::pow(std::max(std::abs(dy) - 1, 0) * edge[1], 2) +
                          std::pow(std::max(std::abs(dz) - 1, 0) * edge[2], 2);
        if (yz > rc2) continue;
        int hi = 0;
        for (int dx = 0; dx <= R[0]; dx++)
          if (yz + std::pow(std::max(dx - 1, 0) * edge[0], 2) <= rc2) hi = dx;
        for (int dx = (dz == 0 && dy == 0) ? 0 : -hi; dx <= hi; dx++) {
          if (half.ncells >= kMaxHalfCells || hi > 8 || std::abs(dy) > 8 || dz > 8)
            return PMB200_EUNSUPPORTED;
          half.off[half.ncells++] = (unsigned short)((dx + 8) | ((dy + 8) << 5) | ((dz + 8) << 10));
        }
      }
  }
  const double u = g.unit;
  const double rl = p->cutoff_lj / u, ro = p->switchon / u, rq = p->cutoff_coul / u;
  const double t = rl * rl - ro * ro;
  MixedConsts mc{};
  mc.cut2 = (float)((rc / u) * (rc / u));
  mc.rclj2 = (float)(rl * rl);
  mc.ron2 = (float)(ro * ro);
  mc.rcc2 = (float)(rq * rq);
  mc.s1 = (float)(1.0 / (t * t * t));
  mc.s2 = (float)(rl * rl - 3.0 * ro * ro);
  mc.s3 = (float)(4.0 / (t * t * t));
  mc.c15_1 = (float)(1.5 / rq);
  mc.c05_3 = (float)(0.5 / (rq * rq * rq));
  mc.c15_3 = (float)(1.5 / (rq * rq * rq));
  mc.e15 = 1.5 / rq;
  mc.e05 = 0.5 / (rq * rq * rq);
  mc.csf = (float)coulomb_scaling;
  mc.ey = (float)(edge[1] / u);
  mc.ez = (float)(edge[2] / u);
  NoAllocLj lj32{};
  const double u6 = std::pow(u, 6.0), u12 = u6 * u6;
  for (int k = 0; k < ntypes * ntypes; k++)
    lj32.v[k] = make_float4((float)(lj[4 * k] / u12), (float)(lj[4 * k + 1] / u6),
                          (float)(lj[4 * k + 2] / u12), (float)(lj[4 * k + 3] / u6));

  cudaError_t e = cudaSuccess;
  unsigned char *base = nullptr;
  if ((e = noalloc_scratch(&base)) != cudaSuccess) return PMB200_ECUDA;
  using Lo = NoAllocLayout;
  int *count = (int *)(base + Lo::count);
  int *start = (int *)(base + Lo::start);
  double *partial = (double *)(base + Lo::partial);
  int *cell_of = (int *)(base + Lo::cell_of);
  int *slot = (int *)(base + Lo::slot);
  int *tmp = (int *)(base + Lo::tmp);
  int *sidx = (int *)(base + Lo::sidx);
  float4 *rel32 = (float4 *)(base + Lo::rel32);
  float4 *spos32 = (float4 *)(base + Lo::spos32);
  float4 *rel_lo = (float4 *)(base + Lo::rel_lo);
  float4 *spos_lo = (float4 *)(base + Lo::spos_lo);
  int2 *smeta = (int2 *)(base + Lo::smeta);
  unsigned long long *facc = (unsigned long long *)(base + Lo::facc);
  double *red = (double *)(base + Lo::red);
  float4 *dlj = (float4 *)(base + Lo::lj32);
  double *pairs = (double *)(base + Lo::pairs);
  int *err = (int *)(base + Lo::err);
  double *out = (double *)(base + Lo::out);
  cudaStream_t st = (cudaStream_t)stream;
  // the array keeps the previous call's contents: zero what accumulates
  k_noalloc_setup<<<1, 256, 0, st>>>(lj32, ntypes * ntypes, dlj, err);
  e = cudaMemsetAsync(count, 0, sizeof(int) * g.ncell, st);
  if (e == cudaSuccess && n > 0)
    e = cudaMemsetAsync(facc, 0, sizeof(unsigned long long) * 3 * (size_t)n, st);
  if (e != cudaSuccess) return PMB200_ECUDA;
  const PbcRef pb{};
  if (n > 0)
    k_cell_index<<<(n + 255) / 256, 256, 0, st>>>(n, d_pos, g, cell_of, count, slot, rel32,
                                                   nullptr, d_q, (float)(1.0 / std::sqrt(u)),
                                                   err, d_energy ? rel_lo : nullptr);
  k_scan<<<1, 1024, 1024 * sizeof(int), st>>>(g.ncell, count, start);
  if (n > 0) k_scatter<<<(n + 255) / 256, 256, 0, st>>>(n, cell_of, slot, start, tmp);
  k_rank_gather<<<(g.ncell + 3) / 4, 128, 0, st>>>(g.ncell, start, tmp, rel32, nullptr, d_type,
                                                    d_mol, sidx, spos32, nullptr, smeta,
                                                    d_energy ? rel_lo : nullptr,
                                                    d_energy ? spos_lo : nullptr);
  const size_t smem = mixed_smem_bytes(FORM_CUTOFF, ntypes, half.ncells);
  const int slots = mixed_cell_slots(d_energy != nullptr, n, g.ncell);
  if (d_energy)
    k_pair_mixed<FORM_CUTOFF, true, false, false><<<g.ncell * slots, 32, smem, st>>>(
        g, mc, half, ntypes, dlj, start, spos32, smeta, sidx, d_ex_start, d_ex, facc, n, err,
        partial, pb, nullptr, slots, spos_lo, 0);
  else
    k_pair_mixed<FORM_CUTOFF, false, false, false><<<g.ncell * slots, 32, smem, st>>>(
        g, mc, half, ntypes, dlj, start, spos32, smeta, sidx, d_ex_start, d_ex, facc, n, err,
        partial, pb, nullptr, slots, spos_lo, 0);
  if (n > 0)
    k_finalize<<<(n + 255) / 256, 256, 0, st>>>(n, facc, sidx, kFixInv / u, 0, d_forces);
  if (d_energy) {
    k_reduce1<<<kRedBlocks, 256, 0, st>>>(g.ncell * slots, partial, red, ACC_E);
    // the reduction writes 20 doubles (energies, virial, molecular
    // virial) into the scratch; the caller's buffer receives the two energies
    k_reduce2<<<1, 256, 0, st>>>(kRedBlocks, red, 1.0, out, pairs, ACC_E);
    e = cudaMemcpyAsync(d_energy, out, 2 * sizeof(double), cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return PMB200_ECUDA;
  }
  if (d_status) k_noalloc_status<<<1, 1, 0, st>>>(err, d_status);
  if (cudaGetLastError() != cudaSuccess) return PMB200_ECUDA;
  return PMB200_OK;
}

int pmb200_grid(const pmb200_ctx *c, int dims[3], double edge[3]) {
  if (!c || !dims || !edge) return PMB200_EINVAL;
  if (!c->have_box) return PMB200_ESTATE;
  dims[0] = c->g.nx; dims[1] = c->g.ny; dims[2] = c->g.nz;
  for (int a = 0; a < 3; a++) edge[a] = c->g.edge[a];
  return PMB200_OK;
}

}  // extern "C"

// ===========================================================================
// Batches of independent systems (pmb200_batch_*): see pmb200_batch.cuh for
// the device layout.
// ===========================================================================
#include "pmb200_batch.cuh"

struct pmb200_batch {
  std::string err;
  int device = 0;
  int form = FORM_CUTOFF;
  int nsys = 0, N = 0, C = 0, ntasks = 0;
  std::vector<BatchSys> h_sys;
  std::vector<double> cost;  // per system: estimated work of one cell task
  BatchSys *d_sys = nullptr;
  int *d_atom_sys = nullptr, *d_type = nullptr, *d_mol = nullptr;
  double *d_q = nullptr;
  int *d_ex_start = nullptr;
  int2 *d_ex = nullptr;
  unsigned short *d_st = nullptr;
  float4 *d_lj32 = nullptr;
  int *d_cell_of = nullptr, *d_count = nullptr, *d_start = nullptr, *d_slot = nullptr;
  int *d_tmp = nullptr, *d_sidx = nullptr, *d_err = nullptr, *d_counter = nullptr;
  float4 *d_rel32 = nullptr, *d_spos32 = nullptr;
  float4 *d_rel_lo = nullptr, *d_spos_lo = nullptr;
  int2 *d_smeta = nullptr;
  unsigned long long *d_facc = nullptr;
  double *d_partial = nullptr, *d_pairs = nullptr, *d_scratch_f = nullptr;
  int4 *d_tasks = nullptr;
  int *d_rows_start = nullptr, *d_rows = nullptr;
  // schedule: stencil parts per cell, task order (0 as built, 1 by cost,
  // largest first), persistent blocks per SM
  int parts = 1, order = 1, bpsm = 0, max_bpsm = 1, nsm = 1;
  int occ[4] = {1, 1, 1, 1};  // resident blocks per SM per variant (energy | virial << 1)
  int lj_max = 0;             // largest LJ table (records) of any system
  size_t smem = 0;            // dynamic shared memory of the pair kernel
  // graph of one evaluation (pmb200_batch_eval_device with a stream)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  const void *gkey[4] = {nullptr, nullptr, nullptr, nullptr};
  unsigned gflags = 0;
  int timing = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace {

int bfail(pmb200_batch *b, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (b) b->err = buf;
  return code;
}

#define BCK(call)                                                                 \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess)                                                        \
      return bfail(b, PMB200_ECUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

void batch_release_graph(pmb200_batch *b) {
  if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->graph_exec = nullptr;
  b->graph = nullptr;
  for (auto &k : b->gkey) k = nullptr;
}

// The task list for the current schedule: every (system, cell, part), in
// system order or by estimated cost (largest first, stable), and each
// system's rows in list order.
int batch_build_tasks(pmb200_batch *b) {
  std::vector<int4> tasks;
  tasks.reserve((size_t)b->C * b->parts);
  for (int s = 0; s < b->nsys; s++)
    for (int c = 0; c < b->h_sys[s].g.ncell; c++)
      for (int p = 0; p < b->parts; p++) tasks.push_back(make_int4(s, c, p, b->parts));
  if (b->order == 1)
    std::stable_sort(tasks.begin(), tasks.end(), [&](const int4 &x, const int4 &y) {
      return b->cost[x.x] > b->cost[y.x];
    });
  const int T = (int)tasks.size();
  std::vector<int> rs(b->nsys + 1, 0), rows(std::max(T, 1));
  for (const int4 &t : tasks) rs[t.x + 1]++;
  for (int s = 0; s < b->nsys; s++) rs[s + 1] += rs[s];
  {
    std::vector<int> fill(rs.begin(), rs.end() - 1);
    for (int t = 0; t < T; t++) rows[fill[tasks[t].x]++] = t;
  }
  if (b->ntasks < T || !b->d_tasks) {
    BCK(dalloc(b->d_tasks, (size_t)std::max(T, 1)));
    BCK(dalloc(b->d_rows, (size_t)std::max(T, 1)));
    BCK(dalloc(b->d_partial, (size_t)std::max(T, 1) * kNacc));
  }
  b->ntasks = T;
  if (T > 0) {
    BCK(cudaMemcpy(b->d_tasks, tasks.data(), sizeof(int4) * T, cudaMemcpyHostToDevice));
    BCK(cudaMemcpy(b->d_rows, rows.data(), sizeof(int) * T, cudaMemcpyHostToDevice));
  }
  BCK(cudaMemcpy(b->d_rows_start, rs.data(), sizeof(int) * (b->nsys + 1),
                 cudaMemcpyHostToDevice));
  batch_release_graph(b);
  return PMB200_OK;
}

template <int F>
void batch_launch_pair(pmb200_batch *b, bool energy, bool virial, int grid, cudaStream_t st) {
#define PMB_BATCH_LAUNCH(E, V)                                                           \
  k_pair_mixed_batch<F, E, V><<<grid, 32, b->smem, st>>>(                                   \
      b->d_sys, b->d_tasks, b->ntasks, b->d_counter, b->d_st, b->d_lj32, b->d_start,       \
      b->d_spos32, b->d_smeta, b->d_sidx, b->d_ex_start, b->d_ex, b->d_facc, b->N,         \
      b->d_partial, b->d_err, b->d_spos_lo, b->lj_max)
  if (energy && virial) PMB_BATCH_LAUNCH(true, true);
  else if (energy) PMB_BATCH_LAUNCH(true, false);
  else if (virial) PMB_BATCH_LAUNCH(false, true);
  else PMB_BATCH_LAUNCH(false, false);
#undef PMB_BATCH_LAUNCH
}

// One evaluation of every system on `st` (forces accumulated into d_forces,
// or overwritten when accumulate is 0).
int batch_launch_eval(pmb200_batch *b, const double *d_pos, double *d_forces, double *d_out,
                      unsigned flags, int accumulate, cudaStream_t st, bool timed) {
  const int N = b->N;
  const bool energy = (flags & PMB200_ENERGY) != 0;
  const bool virial = (flags & PMB200_VIRIAL) != 0;
  // the FP32 coordinates' residuals feed the cutoff form's energy sums
  const bool lo = energy && b->form == FORM_CUTOFF;
  BCK(cudaMemsetAsync(b->d_count, 0, sizeof(int) * b->C, st));
  if (N > 0)
    k_cell_index_batch<<<(N + 255) / 256, 256, 0, st>>>(N, d_pos, b->d_sys, b->d_atom_sys,
                                                        b->d_cell_of, b->d_count, b->d_slot,
                                                        b->d_rel32, b->d_q, b->d_err,
                                                        lo ? b->d_rel_lo : nullptr);
  k_scan<<<1, 1024, 1024 * sizeof(int), st>>>(b->C, b->d_count, b->d_start);
  if (N > 0)
    k_scatter<<<(N + 255) / 256, 256, 0, st>>>(N, b->d_cell_of, b->d_slot, b->d_start,
                                                 b->d_tmp);
  k_rank_gather<<<(b->C + 3) / 4, 128, 0, st>>>(b->C, b->d_start, b->d_tmp, b->d_rel32,
                                                  nullptr, b->d_type, b->d_mol, b->d_sidx,
                                                  b->d_spos32, nullptr, b->d_smeta,
                                                  lo ? b->d_rel_lo : nullptr,
                                                  lo ? b->d_spos_lo : nullptr);
  if (N > 0)
    BCK(cudaMemsetAsync(b->d_facc, 0, sizeof(unsigned long long) * 3 * (size_t)N, st));
  BCK(cudaMemsetAsync(b->d_counter, 0, sizeof(int), st));
  // resident blocks per SM of the variant launched (registers differ)
  const int fit = b->occ[(energy ? 1 : 0) | (virial ? 2 : 0)];
  const int bpsm = b->bpsm > 0 ? std::min(b->bpsm, fit) : fit;
  const int grid = std::max(1, std::min(b->ntasks, bpsm * b->nsm));
  if (timed) BCK(cudaEventRecord(b->ev0, st));
  if (b->form == FORM_GENERIC) batch_launch_pair<FORM_GENERIC>(b, energy, virial, grid, st);
  else if (b->form == FORM_EWALD_POLY5) batch_launch_pair<FORM_EWALD_POLY5>(b, energy, virial, grid, st);
  else if (b->form == FORM_EWALD_EXACT) batch_launch_pair<FORM_EWALD_EXACT>(b, energy, virial, grid, st);
  else batch_launch_pair<FORM_CUTOFF>(b, energy, virial, grid, st);
  if (timed) BCK(cudaEventRecord(b->ev1, st));
  if (N > 0)
    k_finalize_batch<<<(N + 255) / 256, 256, 0, st>>>(N, b->d_facc, b->d_sidx, b->d_atom_sys,
                                                      b->d_sys, accumulate, d_forces);
  if ((energy || virial) && d_out)
    k_reduce_batch<<<(b->nsys + 3) / 4, 128, 0, st>>>(b->nsys, b->d_rows_start, b->d_rows,
                                                       b->d_partial, b->d_sys, d_out, b->d_pairs,
                                                       virial ? ACC_MV : ACC_E);
  BCK(cudaGetLastError());
  return PMB200_OK;
}

}  // namespace

extern "C" {

int pmb200_batch_destroy(pmb200_batch *b) {
  if (!b) return PMB200_OK;
  cudaSetDevice(b->device);
  batch_release_graph(b);
  dfree(b->d_sys); dfree(b->d_atom_sys); dfree(b->d_type); dfree(b->d_mol); dfree(b->d_q);
  dfree(b->d_ex_start); dfree(b->d_ex); dfree(b->d_st); dfree(b->d_lj32);
  dfree(b->d_cell_of); dfree(b->d_count); dfree(b->d_start); dfree(b->d_slot);
  dfree(b->d_tmp); dfree(b->d_sidx); dfree(b->d_err); dfree(b->d_counter);
  dfree(b->d_rel32); dfree(b->d_spos32); dfree(b->d_rel_lo); dfree(b->d_spos_lo); dfree(b->d_smeta); dfree(b->d_facc);
  dfree(b->d_partial); dfree(b->d_pairs); dfree(b->d_scratch_f); dfree(b->d_tasks);
  dfree(b->d_rows_start); dfree(b->d_rows);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  delete b;
  return PMB200_OK;
}

const char *pmb200_batch_last_error(const pmb200_batch *b) { return b ? b->err.c_str() : ""; }

int pmb200_batch_create(pmb200_ctx *const *systems, int nsys, pmb200_batch **out) {
  if (!out || nsys <= 0 || !systems) return PMB200_EINVAL;
  *out = nullptr;
  for (int s = 0; s < nsys; s++) {
    const pmb200_ctx *c = systems[s];
    if (!c) return PMB200_EINVAL;
    if (!c->have_topo || !c->have_box) return PMB200_ESTATE;
    if (c->p.precision != PMB200_MIXED) return PMB200_EUNSUPPORTED;
    if (c->ntypes > kMaxTypes) return PMB200_EUNSUPPORTED;  // tables staged in shared memory
    if (c->g.tric) return PMB200_EUNSUPPORTED;  // the batch bins orthogonal boxes only
    if (c->form != systems[0]->form || c->p.device != systems[0]->p.device)
      return PMB200_EINVAL;
  }
  pmb200_batch *b = new pmb200_batch();
  b->nsys = nsys;
  b->device = systems[0]->p.device;
  b->form = systems[0]->form;
  int rc = PMB200_OK;
  auto done = [&](int code) {
    if (code) pmb200_batch_destroy(b);
    else *out = b;
    return code;
  };
  if (cudaSetDevice(b->device) != cudaSuccess) return done(PMB200_ECUDA);
  // offsets and per-system parameters
  std::vector<unsigned short> st;
  std::vector<float4> lj;
  std::vector<int> atom_sys;
  long long N = 0, C = 0;
  for (int s = 0; s < nsys; s++) {
    pmb200_ctx *c = systems[s];
    if (pull_lj(c)) return done(PMB200_ECUDA);
    BatchSys y{};
    y.g = c->g;
    y.mc = c->mc;
    y.pb = c->pb;
    y.fscale = kFixInv / c->g.unit;
    y.qscale32 = (float)(1.0 / std::sqrt(c->g.unit));
    y.cell0 = (int)C;
    y.atom0 = (int)N;
    y.natoms = c->n;
    y.st0 = (int)st.size();
    y.st_n = c->half.ncells;
    st.insert(st.end(), c->half.off, c->half.off + c->half.ncells);
    y.lj0 = (int)lj.size();
    y.ntypes = c->ntypes;
    const double u = c->g.unit, u6 = std::pow(u, 6.0), u12 = u6 * u6;
    for (int k = 0; k < c->ntypes * c->ntypes; k++) {
      const double *p = &c->h_lj[4 * k];
      lj.push_back(make_float4((float)(p[0] / u12), (float)(p[1] / u6), (float)(p[2] / u12),
                               (float)(p[3] / u6)));
    }
    b->h_sys.push_back(y);
    const double per_cell = c->g.ncell > 0 ? (double)c->n / c->g.ncell : 0.0;
    b->cost.push_back(per_cell * per_cell * c->half.ncells);
    atom_sys.insert(atom_sys.end(), c->n, s);
    N += c->n;
    C += c->g.ncell;
  }
  if (N > (1LL << 30) || C > (1LL << 28)) return done(bfail(b, PMB200_EUNSUPPORTED, "batch too large"));
  b->N = (int)N;
  b->C = (int)C;
  const size_t n1 = (size_t)std::max<long long>(N, 1);
  // per-atom data gathered from the contexts (exclusions re-indexed)
  std::vector<int> ex_start(N + 1, 0);
  std::vector<int2> ex;
  auto cuda = [&](cudaError_t e) { if (e != cudaSuccess && !rc) rc = bfail(b, PMB200_ECUDA, "%s", cudaGetErrorString(e)); };
  cuda(dalloc(b->d_type, n1));
  cuda(dalloc(b->d_mol, n1));
  cuda(dalloc(b->d_q, n1));
  if (rc) return done(rc);
  for (int s = 0; s < nsys; s++) {
    const pmb200_ctx *c = systems[s];
    const int a0 = b->h_sys[s].atom0, n = c->n;
    if (n == 0) continue;
    cuda(cudaMemcpy(b->d_type + a0, c->d_type, sizeof(int) * n, cudaMemcpyDeviceToDevice));
    cuda(cudaMemcpy(b->d_mol + a0, c->d_mol, sizeof(int) * n, cudaMemcpyDeviceToDevice));
    cuda(cudaMemcpy(b->d_q + a0, c->d_q, sizeof(double) * n, cudaMemcpyDeviceToDevice));
    std::vector<int> es(n + 1);
    cuda(cudaMemcpy(es.data(), c->d_ex_start, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost));
    std::vector<int2> e(std::max(es[n], 1));
    if (es[n] > 0)
      cuda(cudaMemcpy(e.data(), c->d_ex, sizeof(int2) * es[n], cudaMemcpyDeviceToHost));
    const int base = (int)ex.size();
    for (int i = 0; i < n; i++) ex_start[a0 + i] = base + es[i];
    for (int k = 0; k < es[n]; k++) ex.push_back(make_int2(e[k].x + a0, e[k].y));
  }
  ex_start[N] = (int)ex.size();
  if (rc) return done(rc);
  cuda(dalloc(b->d_sys, (size_t)nsys));
  cuda(dalloc(b->d_atom_sys, n1));
  cuda(dalloc(b->d_ex_start, n1 + 1));
  cuda(dalloc(b->d_ex, std::max<size_t>(ex.size(), 1)));
  cuda(dalloc(b->d_st, std::max<size_t>(st.size(), 1)));
  cuda(dalloc(b->d_lj32, std::max<size_t>(lj.size(), 1)));
  cuda(dalloc(b->d_cell_of, n1));
  cuda(dalloc(b->d_slot, n1));
  cuda(dalloc(b->d_tmp, n1));
  cuda(dalloc(b->d_sidx, n1));
  cuda(dalloc(b->d_rel32, n1));
  cuda(dalloc(b->d_spos32, n1));
  cuda(dalloc(b->d_rel_lo, n1));
  cuda(dalloc(b->d_spos_lo, n1));
  cuda(dalloc(b->d_smeta, n1));
  cuda(dalloc(b->d_facc, 3 * n1));
  cuda(dalloc(b->d_scratch_f, 3 * n1));
  cuda(dalloc(b->d_count, (size_t)std::max<long long>(C, 1)));
  cuda(dalloc(b->d_start, (size_t)C + 1));
  cuda(dalloc(b->d_err, 1));
  cuda(dalloc(b->d_counter, 1));
  cuda(dalloc(b->d_pairs, (size_t)nsys));
  cuda(dalloc(b->d_rows_start, (size_t)nsys + 1));
  cuda(cudaEventCreate(&b->ev0));
  cuda(cudaEventCreate(&b->ev1));
  if (rc) return done(rc);
  cuda(cudaMemcpy(b->d_sys, b->h_sys.data(), sizeof(BatchSys) * nsys, cudaMemcpyHostToDevice));
  if (N > 0)
    cuda(cudaMemcpy(b->d_atom_sys, atom_sys.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
  cuda(cudaMemcpy(b->d_ex_start, ex_start.data(), sizeof(int) * (N + 1), cudaMemcpyHostToDevice));
  if (!ex.empty())
    cuda(cudaMemcpy(b->d_ex, ex.data(), sizeof(int2) * ex.size(), cudaMemcpyHostToDevice));
  if (!st.empty())
    cuda(cudaMemcpy(b->d_st, st.data(), sizeof(unsigned short) * st.size(), cudaMemcpyHostToDevice));
  if (!lj.empty())
    cuda(cudaMemcpy(b->d_lj32, lj.data(), sizeof(float4) * lj.size(), cudaMemcpyHostToDevice));
  cuda(cudaMemset(b->d_err, 0, sizeof(int)));
  if (rc) return done(rc);
  // dynamic shared memory: the largest LJ table, then the largest stencil
  int st_max = 0;
  for (const BatchSys &y : b->h_sys) {
    b->lj_max = std::max(b->lj_max, y.ntypes * y.ntypes);
    st_max = std::max(st_max, y.st_n);
  }
  b->smem = sizeof(float4) * (size_t)b->lj_max +
            ((sizeof(unsigned short) * (size_t)st_max + 15) & ~(size_t)15);
  // persistent grid: resident blocks per SM of the pair kernel
  int dev_sm = 1;
  cuda(cudaDeviceGetAttribute(&dev_sm, cudaDevAttrMultiProcessorCount, b->device));
  auto fits = [&](auto kernel, int &out) {
    int o = 1;
    cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kernel, 32, b->smem));
    out = std::max(1, o);
  };
  // per (energy, virial) variant of the batch's form
  if (b->form == FORM_GENERIC) {
    fits(k_pair_mixed_batch<FORM_GENERIC, false, false>, b->occ[0]);
    fits(k_pair_mixed_batch<FORM_GENERIC, true, false>, b->occ[1]);
    fits(k_pair_mixed_batch<FORM_GENERIC, false, true>, b->occ[2]);
    fits(k_pair_mixed_batch<FORM_GENERIC, true, true>, b->occ[3]);
  } else if (b->form == FORM_EWALD_POLY5) {
    fits(k_pair_mixed_batch<FORM_EWALD_POLY5, false, false>, b->occ[0]);
    fits(k_pair_mixed_batch<FORM_EWALD_POLY5, true, false>, b->occ[1]);
    fits(k_pair_mixed_batch<FORM_EWALD_POLY5, false, true>, b->occ[2]);
    fits(k_pair_mixed_batch<FORM_EWALD_POLY5, true, true>, b->occ[3]);
  } else if (b->form == FORM_EWALD_EXACT) {
    fits(k_pair_mixed_batch<FORM_EWALD_EXACT, false, false>, b->occ[0]);
    fits(k_pair_mixed_batch<FORM_EWALD_EXACT, true, false>, b->occ[1]);
    fits(k_pair_mixed_batch<FORM_EWALD_EXACT, false, true>, b->occ[2]);
    fits(k_pair_mixed_batch<FORM_EWALD_EXACT, true, true>, b->occ[3]);
  } else {
    fits(k_pair_mixed_batch<FORM_CUTOFF, false, false>, b->occ[0]);
    fits(k_pair_mixed_batch<FORM_CUTOFF, true, false>, b->occ[1]);
    fits(k_pair_mixed_batch<FORM_CUTOFF, false, true>, b->occ[2]);
    fits(k_pair_mixed_batch<FORM_CUTOFF, true, true>, b->occ[3]);
  }
  if (rc) return done(rc);
  b->nsm = dev_sm;
  b->max_bpsm = std::max(std::max(b->occ[0], b->occ[1]), std::max(b->occ[2], b->occ[3]));
  return done(batch_build_tasks(b));
}

int pmb200_batch_set_schedule(pmb200_batch *b, int parts, int order, int blocks_per_sm) {
  if (!b) return PMB200_EINVAL;
  if (parts < 1 || parts > 8 || order < 0 || order > 1 || blocks_per_sm < 0)
    return bfail(b, PMB200_EINVAL, "schedule parts %d order %d blocks/SM %d", parts, order,
                 blocks_per_sm);
  BCK(cudaSetDevice(b->device));
  b->parts = parts;
  b->order = order;
  b->bpsm = blocks_per_sm;
  return batch_build_tasks(b);
}

int pmb200_batch_get_schedule(const pmb200_batch *b, int sched[4]) {
  if (!b || !sched) return PMB200_EINVAL;
  sched[0] = b->parts;
  sched[1] = b->order;
  sched[2] = b->bpsm > 0 ? std::min(b->bpsm, b->occ[0]) : b->occ[0];
  sched[3] = b->ntasks;
  return PMB200_OK;
}

int pmb200_batch_eval_device(pmb200_batch *b, const double *d_pos, double *d_forces,
                             double *d_out, unsigned flags, void *stream) {
  if (!b) return PMB200_EINVAL;
  if (flags & PMB200_MOLVIRIAL)
    return bfail(b, PMB200_EUNSUPPORTED, "molecular virial is not offered for batches");
  if (b->N > 0 && (!d_pos || !d_forces)) return bfail(b, PMB200_EINVAL, "null device buffer");
  if ((flags & (PMB200_ENERGY | PMB200_VIRIAL)) && !d_out)
    return bfail(b, PMB200_EINVAL, "null output buffer");
  BCK(cudaSetDevice(b->device));
  cudaStream_t st = (cudaStream_t)stream;
  if (!stream || b->timing) return batch_launch_eval(b, d_pos, d_forces, d_out, flags, 1, st, b->timing != 0);
  const void *key[4] = {d_pos, d_forces, d_out, stream};
  bool same = b->graph_exec && b->gflags == flags;
  for (int k = 0; k < 4 && same; k++) same = b->gkey[k] == key[k];
  if (!same) {
    batch_release_graph(b);
    BCK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = batch_launch_eval(b, d_pos, d_forces, d_out, flags, 1, st, false);
    cudaGraph_t gr = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &gr);
    if (rc) {
      if (gr) cudaGraphDestroy(gr);
      return rc;
    }
    if (e != cudaSuccess) return bfail(b, PMB200_ECUDA, "capture: %s", cudaGetErrorString(e));
    b->graph = gr;
    BCK(cudaGraphInstantiate(&b->graph_exec, gr, 0));
    for (int k = 0; k < 4; k++) b->gkey[k] = key[k];
    b->gflags = flags;
  }
  BCK(cudaGraphLaunch(b->graph_exec, st));
  return PMB200_OK;
}

int pmb200_batch_sync(pmb200_batch *b, void *stream) {
  if (!b) return PMB200_EINVAL;
  BCK(cudaSetDevice(b->device));
  if (stream) BCK(cudaStreamSynchronize((cudaStream_t)stream));
  else BCK(cudaDeviceSynchronize());
  int e = 0;
  BCK(cudaMemcpy(&e, b->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    BCK(cudaMemset(b->d_err, 0, sizeof(int)));
    if (e & 1) return bfail(b, PMB200_EDEVICE, "non-finite atom position in a batch evaluation");
    return bfail(b, PMB200_EDEVICE,
                 "a pair force exceeded the fixed-point range in a batch evaluation (atoms overlap)");
  }
  return PMB200_OK;
}

int pmb200_batch_set_kernel_timing(pmb200_batch *b, int on) {
  if (!b) return PMB200_EINVAL;
  b->timing = on ? 1 : 0;
  return PMB200_OK;
}

int pmb200_batch_last_kernel_ms(pmb200_batch *b, float *ms) {
  if (!b || !ms) return PMB200_EINVAL;
  BCK(cudaSetDevice(b->device));
  BCK(cudaEventSynchronize(b->ev1));
  BCK(cudaEventElapsedTime(ms, b->ev0, b->ev1));
  return PMB200_OK;
}

int pmb200_batch_pair_counts(pmb200_batch *b, long long *counts) {
  if (!b || !counts) return PMB200_EINVAL;
  BCK(cudaSetDevice(b->device));
  std::vector<double> v(b->nsys);
  BCK(cudaDeviceSynchronize());
  BCK(cudaMemcpy(v.data(), b->d_pairs, sizeof(double) * b->nsys, cudaMemcpyDeviceToHost));
  for (int s = 0; s < b->nsys; s++) counts[s] = (long long)llround(v[s]);
  return PMB200_OK;
}

int pmb200_batch_autotune(pmb200_batch *b, const double *d_pos, void *stream, int reps,
                          int sched[4], float *best_ms) {
  if (!b || !sched || !best_ms) return PMB200_EINVAL;
  if (b->N > 0 && !d_pos) return bfail(b, PMB200_EINVAL, "null device buffer");
  if (reps < 1) reps = 5;
  BCK(cudaSetDevice(b->device));
  cudaStream_t st = (cudaStream_t)stream;
  const int parts_c[4] = {1, 2, 4, 8};
  const int bpsm_c[2] = {b->occ[0], std::max(1, b->occ[0] / 2)};
  float best = -1.0f;
  int bp = 1, bo = 1, bb = 0;
  for (int pi = 0; pi < 4; pi++)
    for (int order = 0; order < 2; order++)
      for (int bi = 0; bi < (bpsm_c[1] != bpsm_c[0] ? 2 : 1); bi++) {
        int rc = pmb200_batch_set_schedule(b, parts_c[pi], order, bpsm_c[bi]);
        if (rc) return rc;
        float tot = 0.0f;
        for (int r = 0; r < reps + 2; r++) {
          rc = batch_launch_eval(b, d_pos, b->d_scratch_f, nullptr, 0, 0, st, true);
          if (rc) return rc;
          float ms = 0.0f;
          BCK(cudaEventSynchronize(b->ev1));
          BCK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
          if (r >= 2) tot += ms;
        }
        const float mean = tot / reps;
        if (best < 0.0f || mean < best) {
          best = mean;
          bp = parts_c[pi];
          bo = order;
          bb = bpsm_c[bi];
        }
      }
  int rc = pmb200_batch_set_schedule(b, bp, bo, bb);
  if (rc) return rc;
  *best_ms = best;
  return pmb200_batch_get_schedule(b, sched);
}

}  // extern "C"
