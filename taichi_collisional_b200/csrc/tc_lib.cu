// C ABI and host orchestration of the B200 FMM gravity evaluation (include/taichi_b200.h).
//
// One tc_evaluate call replaces get_force_and_potential(bodies, false)
// (integrator.h:459-562, taichi_with_jerks/integrator.h:308-432) on the theta-MAC path:
//   bounds -> Morton keys -> radix sort -> octree levels      (build_tree.h)
//   smallest enclosing balls + P2M / M2M, deepest level first  (traverse_eager.h:9-34)
//   dual traversal -> sorted M2L and P2P lists                 (traverse_eager.h:151-216)
//   M2L (rotation, FP64) and P2P                               (kernel_fast_lean.h)
//   L2L level by level, L2P                                    (traverse_eager.h:326-346)
// All arithmetic runs on the GPU; there is no CPU fallback.  The only host reads are the
// tree's level table and the list sizes (to size launches and buffers).
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "tc_common.cuh"
#include "tc_tree.cuh"
#include "tc_upward.cuh"
#include "tc_traverse.cuh"
#include "tc_m2l.cuh"
#include "tc_m2l_mixed.cuh"
#include "tc_m2l_tc.cuh"
#include "tc_emac.cuh"
#include "tc_down.cuh"
#include "tc_p2p.cuh"
#include "tc_select.cuh"
#include "tc_mlp.cuh"
#include "tc_train.cuh"
#include "tc_order.cuh"
#include "tc_diag.cuh"
#include "tdesign.h"

using namespace tc;

namespace {

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaError_t ensure(size_t want) {
    if (want <= n && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    size_t alloc = want + want / 8 + 16;
    cudaError_t e = cudaMalloc((void**)&p, alloc * sizeof(T));
    if (e == cudaSuccess) n = alloc;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

// Source chunks per target leaf of the FP64 near field: 1 at large n; at small n (few target
// leaves, ~48 bodies each) enough chunks for ~32 warps per SM, at most 16.  A function of n only,
// so the direct launches and a captured graph of the same call sum in the same order.
static inline int p2p_nsplit(int n) {
  long long k = (148LL * 32 * 48 + n - 1) / (n > 0 ? n : 1);
  return (int)(k < 1 ? 1 : k > 16 ? 16 : k);
}

// what a captured evaluation was recorded for (a call must match to replay it)
struct TcGraphKey {
  int n = -1, mem = -1;
  const void* ptr[15] = {};
  tc_params prm;
  double step_dt = 0.0;  // != 0: the whole leapfrog step (tc_step_leapfrog) around the evaluation
};

// read back after a replay (small device structs, copied by the graph into pinned memory)
struct TcGraphStatus {
  unsigned err;
  unsigned small[4];
  unsigned hist[32];  // pairs per order (order selection)
  TcLevels lv;
  TcTravCounters cnt;
};

struct EvalTimes {
  cudaEvent_t e[8];
};

}  // namespace

struct tc_ctx {
  tc_params prm;
  cudaStream_t stream = nullptr;
  std::string err;
  tc_stats stats;
  // staging (host-memory calls)
  DBuf<double> in_d;  // 7 * N
  DBuf<uint8_t> in_f;
  DBuf<double> out_d;  // 7 * N (caller order)
  // bodies
  DBuf<unsigned long long> keys, keys_alt;
  DBuf<int> vals, vals_alt;
  DBuf<uint32_t> hist;
  DBuf<double> bod;  // 7 * N sorted
  DBuf<uint8_t> bflags;
  DBuf<int> perm;
  DBuf<double> outs;  // 7 * N sorted
  // cells
  DBuf<int> cint;      // 6 * ccap
  DBuf<double> cdbl;   // 7 * ccap
  DBuf<uint8_t> csink;
  DBuf<int> split_off;
  DBuf<double> expn;   // (2 or 4) * expn_stride * NT
  size_t expn_stride = 0;  // cells per expansion array: ncell, or ccap in a captured graph
  size_t ccap = 0;
  // lists
  DBuf<int2> front[2];
  DBuf<unsigned long long> m2l, m2l_alt, p2p, p2p_alt;
  DBuf<int> m2l_start, m2l_src, p2p_start, p2p_src, m2l_tl, p2p_tl, leaves;
  DBuf<double> cell_pn;
  DBuf<int> cls_start, cls_tl;  // per order class: per-target offsets and target lists
  int n_classes = 0, class_order[16];
  long long class_pairs[16];
  double flop_frac = 1.0;
  // per-pair orders with a per-target budget: |a| of the last evaluation (caller order, valid for
  // amag_n bodies), per-body and per-cell budget scales, the regrouped source lists and orders
  DBuf<double> amag, body_scale, cell_scale;
  int amag_n = -1;
  DBuf<int> m2l_src2;
  DBuf<uint8_t> m2l_off;
  DBuf<int> cls_rng;  // per order class and cell: begin, then end, of the class's source range
  DBuf<float> cell_feat;  // per cell: the learned selector's per-cell features
  unsigned* d_hist = nullptr;  // 32 counters
  // learned selector
  bool mlp_ready = false;
  int mlp_nout = 0;
  DBuf<float> mlp_w;
  TcMlpNorm mlp_norm;
  std::vector<float> train_feat, train_lab;
  int train_n = 0;
  double judge_rms = 0.0;
  int judge_redo = 0;
  DBuf<int> judge_idx;
  DBuf<double> judge_out;
  // time-step pass (tc_evaluate_steps): per-body sum of 1/tau^4 in Morton order
  bool steps = false;
  double dt_param = 0.025;
  DBuf<double> tsum;
  // tc_direct_sums: bodies in caller order, targets, partial and final sums
  DBuf<double> ds_bod, ds_out;
  DBuf<double> diag;  // system diagnostics: block partials + the 9 results
  DBuf<double> p2p_part;  // near-field partial sums per source chunk (few target leaves)
  // block-time-step integrator: accelerations, potential, 1/tau^4 sums; split counters, pair
  // positions, kick flags
  DBuf<double> ev_d;
  DBuf<uint32_t> ev_u;
  DBuf<int> ev_i;
  DBuf<uint8_t> ev_f;
  DBuf<uint8_t> ds_flags;
  DBuf<int> ds_idx, ds_tgt;
  DBuf<double> kd_scratch;  // direct kicks of small systems: 14 arrays of kd_cap entries
  DBuf<int> kd_index;
  DBuf<uint8_t> kd_flags;
  size_t kd_cap = 0;
  size_t fcap = 0, mcap = 0, pcap = 0;
  // small device structs
  TcRootInfo* d_root = nullptr;
  TcLevels* d_lv = nullptr;
  TcTravCounters* d_cnt = nullptr;
  unsigned int* d_err = nullptr;
  unsigned int* d_small = nullptr;  // [0] m2l targets, [1] p2p targets, [2] leaves, [9] tensor M2L counter,
                                    // [10] target counter of the persistent FP64 M2L (graph)
  DBuf<float> tc_bins;  // tensor-core M2L bin matrices (hi, lo) of order tc_bins_q
  int tc_bins_q = -1;
  long long wait_limit = kTcWaitLimit;  // clock cycles a bounded device wait may take (tc_set_wait_limit)
  int nsm = 0;
  DBuf<double> bpart;
  // last evaluation
  TcLevels lv;
  int n = 0, ncell = 0, nleaf = 0, max_level = 0, direct = 0;
  unsigned long long n_m2l = 0, n_p2p = 0;
  int sbits = 1;
  long long launches = 0;
  unsigned tree_flags = 0;
  unsigned long long n_inter = 0;
  cudaEvent_t ev[8];
  bool events = false;
  // CUDA graph of the whole evaluation (tc_set_graph)
  bool graph_on = false, gvalid = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaStream_t gstream = nullptr;
  TcGraphKey gkey;
  TcGraphStatus* hstat = nullptr;  // pinned: written by the graph's last copies
  double* hjudge = nullptr;        // pinned: 7 x judge targets (FP64 direct sums and FMM values)
  size_t hjudge_cap = 0;
  int gjudge_nt = 0;
  long long glaunches = 0;
  int gsbits = 1;
  std::string gfail;  // why the last capture was abandoned (empty: captured)
  std::vector<const void*> gsig;  // buffers and capacities baked into the captured graph
  double gstep_dt = 0.0;          // the graph being planned holds a leapfrog step of this dt
  bool gselect = false;           // the captured graph selects per-pair orders
  int gcls_q[TC_MAX_CLASSES];     // ... with these class orders
  int gcls_n = 0;
  // error-controlled MAC of the top tree (tc_set_error_mac) and its low-order pre-pass
  bool emac = false;
  double emac_fa = 2.0e-7;
  DBuf<double> low_rgeo, low_m9, low_l9, acc_old, min_acc, pn_ref, low_f;
  DBuf<int> cell_of;
};

static bool g_const_init[64];

static tc_status cuda_fail(tc_ctx* c, cudaError_t e, const char* what) {
  if (c) c->err = std::string(what) + ": " + cudaGetErrorString(e);
  return TC_ERR_CUDA;
}

#define TC_CK(call)                                   \
  do {                                                \
    cudaError_t e_ = (call);                          \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
  } while (0)

static cudaError_t init_constants(int dev) {
  if (dev >= 0 && dev < 64 && g_const_init[dev]) return cudaSuccess;
  double fact[2 * TC_PMAX_DEV + 2];
  fact[0] = 1.0;
  for (int i = 1; i < 2 * TC_PMAX_DEV + 2; i++) fact[i] = fact[i - 1] * (double)i;
  double fc[TC_NTERM(TC_PMAX_DEV)], fci[TC_NTERM(TC_PMAX_DEV)];
  for (int n = 0; n <= TC_PMAX_DEV; n++)
    for (int m = -n; m <= n; m++) {
      int am = m < 0 ? -m : m;
      double f = fact[n + am] * fact[n - am];
      fc[n * n + n + m] = f;
      fci[n * n + n + m] = 1.0 / f;
    }
  cudaError_t e;
  if ((e = cudaMemcpyToSymbol(c_fact, fact, sizeof(fact))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_fc, fc, sizeof(fc))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_fcinv, fci, sizeof(fci))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_tdesign, tc_tdesign, sizeof(tc_tdesign))) != cudaSuccess) return e;
  // mixed-precision M2L scalings (tc_m2l_mixed.cuh)
  double mF[TC_NTERM(TC_PMAX_DEV)], mDoF[TC_NTERM(TC_PMAX_DEV)];
  static float mC[(TC_PMAX_DEV + 1) * (TC_PMAX_DEV + 1) * (TC_PMAX_DEV + 1)];
  for (int n = 0; n <= TC_PMAX_DEV; n++)
    for (int m = -n; m <= n; m++) {
      int am = m < 0 ? -m : m;
      double D = fact[n + am] * fact[n - am];
      double F = sqrt(D) * (am ? sqrt(2.0) : 1.0);
      mF[n * n + n + m] = F;
      mDoF[n * n + n + m] = D / F;
    }
  for (int n = 0; n <= TC_PMAX_DEV; n++)
    for (int k = 0; k <= TC_PMAX_DEV; k++)
      for (int m = 0; m <= TC_PMAX_DEV; m++) {
        double v = 0.0;
        if (m <= n && m <= k && n + k <= 2 * TC_PMAX_DEV)
          v = ((m & 1) ? -1.0 : 1.0) * fact[n + k] /
              sqrt(fact[n + m] * fact[n - m] * fact[k + m] * fact[k - m]);
        mC[(n * (TC_PMAX_DEV + 1) + k) * (TC_PMAX_DEV + 1) + m] = (float)v;
      }
  if ((e = cudaMemcpyToSymbol(c_mF, mF, sizeof(mF))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_mDoF, mDoF, sizeof(mDoF))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_mC, mC, sizeof(mC))) != cudaSuccess) return e;
  if (dev >= 0 && dev < 64) g_const_init[dev] = true;
  return cudaSuccess;
}

// bin matrices of the tensor-core M2L at order Q (tc_m2l_tc.cuh): the orthogonal swap
// T_n = E S_n E^-1 of every degree (S from the exact tables of swap_tables.h,
// E_k = c_m / sqrt((n+|m|)!(n-|m|)!)) and the translation C[n,k,m] = (-1)^m (n+k)! /
// sqrt((n+m)!(n-m)!(k+m)!(k-m)!) for n + k <= Q, each rounded to TF32 as hi + lo
static float tc_tf32_host(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
  float r;
  memcpy(&r, &u, 4);
  return r;
}

template <int Q>
static void tc_build_bins(std::vector<float>& img) {
  using PL = TcTcPlan<Q>;
  const int NB = PL::NH + PL::NTB;
  std::vector<double> full((size_t)NB * 256, 0.0);
  double fact[2 * TC_TC_QMAX + 2];
  fact[0] = 1.0;
  for (int i = 1; i < 2 * TC_TC_QMAX + 2; i++) fact[i] = fact[i - 1] * (double)i;
  auto deg = [](int i) { int n = 0; while ((n + 1) * (n + 1) <= i) n++; return n; };
  auto E = [&](int n, int m) {
    int a = m < 0 ? -m : m;
    return (a ? sqrt(2.0) : 1.0) / sqrt(fact[n + a] * fact[n - a]);
  };
  // swap halves: out position o, in position k of the same half (same degree only)
  for (int h = 0; h < PL::NH; h++)
    for (int o = 0; o < 16; o++)
      for (int k = 0; k < 16; k++) {
        int no = PL::half_nat[h][o], ni = PL::half_nat[h][k];
        if (no < 0 || ni < 0) continue;
        int n = deg(no);
        if (deg(ni) != n) continue;
        double sv = 0.0;
        for (int r = tc_swap_rowptr[no]; r < tc_swap_rowptr[no + 1]; r++)
          if (tc_swap_col[r] == ni) sv = tc_swap_val[r];
        full[(size_t)h * 256 + tc_tc_bin_index(o, k)] = sv * E(n, no - n * n - n) / E(n, ni - n * n - n);
      }
  // translation bins (real arrangement; the imaginary parts use the same matrix)
  for (int b = 0; b < PL::NTB; b++)
    for (int o = 0; o < 16; o++)
      for (int k = 0; k < 16; k++) {
        int no = PL::trans_nat[b][o], ni = PL::trans_nat[b][k];
        if (no < 0 || ni < 0) continue;
        int N = deg(no), K = deg(ni);
        int mo = no - N * N - N, mi = ni - K * K - K;
        if (mo != mi || N + K > Q) continue;
        int m = mo < 0 ? -mo : mo;
        double v = ((m & 1) ? -1.0 : 1.0) * fact[N + K] / sqrt(fact[N + m] * fact[N - m] * fact[K + m] * fact[K - m]);
        full[(size_t)(PL::NH + b) * 256 + tc_tc_bin_index(o, k)] = v;
      }
  img.assign((size_t)2 * NB * 256, 0.f);
  for (size_t i = 0; i < full.size(); i++) {
    float hi = tc_tf32_host((float)full[i]);
    img[i] = hi;
    img[full.size() + i] = tc_tf32_host((float)(full[i] - (double)hi));
  }
}

template <int Q>
static cudaError_t tc_ensure_bins(tc_ctx* ctx) {
  if (ctx->tc_bins_q == Q) return cudaSuccess;
  std::vector<float> img;
  tc_build_bins<Q>(img);
  cudaError_t e = ctx->tc_bins.ensure(img.size());
  if (e != cudaSuccess) return e;
  e = cudaMemcpy(ctx->tc_bins.p, img.data(), img.size() * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) ctx->tc_bins_q = Q;
  return e;
}

static inline int nblocks(long long n, int t) { return (int)((n + t - 1) / t); }

static TcCells cells_view(tc_ctx* c, int NT) {
  TcCells v;
  size_t cc = c->ccap;
  int* ci = c->cint.p;
  v.begin = ci; v.nbody = ci + cc; v.nchild = ci + 2 * cc; v.child = ci + 3 * cc; v.parent = ci + 4 * cc;
  v.level = ci + 5 * cc;
  double* cd = c->cdbl.p;
  v.gx = cd; v.gy = cd + cc; v.gz = cd + 2 * cc; v.X = cd + 3 * cc; v.Y = cd + 4 * cc; v.Z = cd + 5 * cc;
  v.R = cd + 6 * cc;
  v.has_sink = c->csink.p;
  size_t ne = c->expn_stride * NT;
  bool jerk = c->prm.variant == TC_VARIANT_JERKS;
  v.M = c->expn.p;
  v.L = c->expn.p ? c->expn.p + ne : nullptr;
  v.Md = (jerk && c->expn.p) ? c->expn.p + 2 * ne : nullptr;
  v.Ld = (jerk && c->expn.p) ? c->expn.p + 3 * ne : nullptr;
  return v;
}

static TcBodies bodies_view(tc_ctx* c, int n, bool jerk) {
  TcBodies b;
  double* d = c->bod.p;
  size_t N = (size_t)n;
  b.x = d; b.y = d + N; b.z = d + 2 * N; b.m = d + 3 * N;
  const bool vel = jerk || c->steps;  // the time-step pass needs velocities in the top tree too
  b.vx = vel ? d + 4 * N : nullptr; b.vy = vel ? d + 5 * N : nullptr; b.vz = vel ? d + 6 * N : nullptr;
  b.flags = c->bflags.p;
  b.perm = c->perm.p;
  b.eps2 = c->prm.softening * c->prm.softening;
  // the mixed near field's FP32 splits sit after the seven FP64 arrays (16-byte aligned)
  b.f32 = c->prm.precision != TC_PREC_FP64 ? reinterpret_cast<float4*>(d + 7 * N + (N & 1)) : nullptr;
  return b;
}

static TcOut out_view(tc_ctx* c, int n, bool jerk) {
  TcOut o;
  double* d = c->outs.p;
  size_t N = (size_t)n;
  o.pot = d; o.ax = d + N; o.ay = d + 2 * N; o.az = d + 3 * N;
  o.jx = jerk ? d + 4 * N : nullptr; o.jy = jerk ? d + 5 * N : nullptr; o.jz = jerk ? d + 6 * N : nullptr;
  return o;
}

__global__ void k_identity(int n, int* v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = i;
}

__global__ void k_nan_check(int n, const double* x, const double* y, const double* z, const double* m, unsigned* err) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && !(isfinite(x[i]) && isfinite(y[i]) && isfinite(z[i]) && isfinite(m[i]))) tc_set_err(err, TC_EBIT_NAN);
}

__global__ void k_leaf_list(int ncell, const int* nchild, int* leaves, unsigned* cnt, const int* ncdev = nullptr) {
  if (ncdev) ncell = *ncdev;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool has = i < ncell && nchild[i] == 0;
  unsigned mask = __ballot_sync(0xffffffffu, has);
  int lane = threadIdx.x & 31;
  unsigned base = 0;
  if (lane == 0 && mask) base = atomicAdd(cnt, (unsigned)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (has) leaves[base + __popc(mask & ((1u << lane) - 1u))] = i;
}

// sum over the P2P list of (sink-cell bodies) x (source-cell bodies)
__global__ void k_p2p_count(const unsigned long long* __restrict__ keys, unsigned long long n, int sbits,
                            const int* __restrict__ nbody, const uint8_t* __restrict__ has_sink,
                            unsigned long long* total, const unsigned long long* ndev = nullptr) {
  if (ndev && *ndev < n) n = *ndev;
  unsigned long long loc = 0, mask = (1ull << sbits) - 1ull;
  for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (unsigned long long)gridDim.x * blockDim.x) {
    int t = (int)(keys[k] >> sbits), s = (int)(keys[k] & mask);
    if (has_sink[t]) loc += (unsigned long long)nbody[t] * (unsigned long long)nbody[s];
  }
  for (int o = 16; o > 0; o >>= 1) loc += __shfl_xor_sync(0xffffffffu, loc, o);
  if ((threadIdx.x & 31) == 0 && loc) atomicAdd(total, loc);
}

// ----------------------------------------------------------------------------------------
// per-pair orders with a per-target error budget (tc_order.cuh): the target scale of every cell
// from the previous evaluation's accelerations, then each target's list regrouped by order
// ----------------------------------------------------------------------------------------
// With an order selector on, accepted pairs of a leaf target whose body counts multiply to at
// most this many interactions are summed directly (exact) instead of by an M2L, scaled by
// (p + 1)^3.  At N = 4M, p = 12 the step time is flat from 256 to 1024 (the near field's
// FP32 interactions, about 2.7 ps of the whole GPU each, against about 2 ns per M2L pair) while
// the force error falls (1.28e-8 -> 1.11e-8 RMS at 512); 0 (fixed order, the reference's
// lists) = off.
static long long p2p_instead_max(const tc_params& prm) {
  if (prm.selector <= 0) return 0;
  const double s = (prm.p + 1.0) / 13.0;
  return (long long)(512.0 * s * s * s);
}

// the orders used by an evaluation: h[k] pairs of class k, of order q[k] (ascending)
static void order_stats(tc_ctx* ctx, int p, const unsigned* h, const int* q, int nclass) {
  ctx->n_classes = 0;
  double tot = 0.0, ff = 0.0;
  for (int k = 0; k < nclass; k++) {
    if (!h[k]) continue;
    ctx->class_order[ctx->n_classes] = q[k];
    ctx->class_pairs[ctx->n_classes] = h[k];
    ctx->n_classes++;
    tot += h[k];
    ff += h[k] * std::pow((q[k] + 1.0) / (p + 1.0), 3);
  }
  ctx->flop_frac = tot > 0 ? ff / tot : 1.0;
}

template <int P>
static cudaError_t select_orders(tc_ctx* ctx, TcCells cv, int n, int ntl, const unsigned* ntldev, bool capture) {
  using OC = TcOrderClasses<P>;
  cudaStream_t st = ctx->stream;
  const int nc = capture ? (int)ctx->ccap : ctx->ncell;
  cudaError_t e;
  if ((e = ctx->cell_pn.ensure((size_t)nc * (P + 1))) != cudaSuccess) return e;
  if ((e = ctx->cell_scale.ensure((size_t)nc)) != cudaSuccess) return e;
  if ((e = ctx->body_scale.ensure((size_t)n)) != cudaSuccess) return e;
  if ((e = ctx->m2l_src2.ensure(ctx->m2l_src.n)) != cudaSuccess) return e;
  if ((e = ctx->m2l_off.ensure(ctx->m2l_src.n)) != cudaSuccess) return e;
  if ((e = ctx->cls_rng.ensure((size_t)2 * OC::n * nc)) != cudaSuccess) return e;
  const int* d_ncell = capture ? &((TcLevels*)ctx->d_lv)->ncell : nullptr;
  k_cell_pn<P><<<std::min(nblocks(nc, 128), 148 * 16), 128, 0, st>>>(nc, cv.M, ctx->cell_pn.p, d_ncell);
  k_gather_scale<<<nblocks(n, 256), 256, 0, st>>>(n, ctx->perm.p, ctx->amag.p, ctx->body_scale.p);
  int* d_start = &((TcLevels*)ctx->d_lv)->start[0];
  int* d_count = &((TcLevels*)ctx->d_lv)->count[0];
  const int maxl = capture ? TC_MAX_LEVEL : ctx->max_level;
  const int gc = std::min(nblocks(nc, 128), 148 * 16);
  for (int l = maxl; l >= 0; l--)
    k_min_acc<<<gc, 128, 0, st>>>(l, cv, d_start, d_count, ctx->body_scale.p, ctx->cell_scale.p);
  if ((e = cudaMemsetAsync(ctx->d_hist, 0, 32 * sizeof(unsigned), st)) != cudaSuccess) return e;
  TcClassOrders co;
  for (int i = 0; i < TC_MAX_CLASSES; i++) {
    co.q[i] = i < OC::n ? OC::q[i] : P;
    co.below[i] = 0;
  }
  for (int l = 0; l < TcClassLaunches<P>::n; l++) {
    const int f = TcClassLaunches<P>::first(l), e2 = TcClassLaunches<P>::first(l + 1);
    for (int i = f; i < e2; i++) co.below[i] = OC::q[e2 - 1] - OC::q[i];
  }
  double fact[2 * TC_PMAX_DEV + 2];
  fact[0] = 1.0;
  for (int i = 1; i < 2 * TC_PMAX_DEV + 2; i++) fact[i] = fact[i - 1] * (double)i;
  for (int k = 0; k <= TC_PMAX_DEV; k++) co.comb[k] = k <= P ? fact[P] * (1.0 / fact[k]) * (1.0 / fact[P - k]) : 0.0;
  const int mode = ctx->prm.selector == 2 ? 2 : 1;
  if (mode == 2) {
    if ((e = ctx->cell_feat.ensure((size_t)nc * 5)) != cudaSuccess) return e;
    k_cell_feat<P><<<std::min(nblocks(nc, 128), 148 * 16), 128, 0, st>>>(nc, cv, ctx->cell_pn.p, ctx->cell_feat.p,
                                                                         d_ncell);
  }
  const int grid = capture ? 148 * 8 : std::max(1, std::min(nblocks(ntl, 4), 148 * 8));
  k_select_order<P><<<grid, 128, 0, st>>>(ctx->m2l_tl.p, ntl, ctx->m2l_start.p, ctx->m2l_src.p, ctx->m2l_src2.p,
                                          ctx->m2l_off.p, ctx->cls_rng.p, ctx->cls_rng.p + (size_t)OC::n * nc, nc,
                                          cv, ctx->cell_pn.p, ctx->cell_scale.p, ctx->prm.selector_tol, mode,
                                          ctx->mlp_w.p, ctx->mlp_norm, OC::n, co, ctx->cell_feat.p, ctx->d_hist,
                                          ntldev);
  ctx->launches += 4 + maxl;
  return cudaGetLastError();
}

// one M2L launch per order class over the class ranges that select_orders wrote: persistent
// grids (one CTA per SM) taking targets from a counter, the target count read on the device
template <int P, bool JERK, int I = 0>
static void m2l_class_launches(tc_ctx* ctx, TcCells cv, int ntl, const unsigned* ntldev, int nc) {
  using OC = TcOrderClasses<P>;
  using CL = TcClassLaunches<P>;
  if constexpr (I < CL::n) {
    constexpr int F = CL::first(I), E = CL::first(I + 1);  // classes [F, E), at the order of E - 1
    constexpr int Q = OC::q[E - 1];
    const size_t smem = (size_t)TcM2LSmem<Q>::TOTAL * sizeof(double);
    unsigned* next = ctx->d_small + 11;
    cudaMemsetAsync(next, 0, sizeof(unsigned), ctx->stream);
    k_m2l<P, Q, JERK><<<ctx->nsm, tc_m2l_threads<Q>(), smem, ctx->stream>>>(
        ctx->m2l_tl.p, ntl, ctx->cls_rng.p + (size_t)F * nc, ctx->m2l_src2.p, cv, ntldev, next,
        ctx->cls_rng.p + (size_t)(OC::n + E - 1) * nc);
    ctx->launches++;
    m2l_class_launches<P, JERK, I + 1>(ctx, cv, ntl, ntldev, nc);
  }
}

template <int P, int I = 0>
static void set_class_attrs() {
  using OC = TcOrderClasses<P>;
  if constexpr (I < OC::n) {
    constexpr int Q = OC::q[I];
    const int smem = (int)(TcM2LSmem<Q>::TOTAL * sizeof(double));
    cudaFuncSetAttribute(k_m2l<P, Q, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(k_m2l<P, Q, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    set_class_attrs<P, I + 1>();
  }
}

// ----------------------------------------------------------------------------------------
// learned selector: training data from the FMM, then Adam on the GPU
// ----------------------------------------------------------------------------------------
template <int P, int I>
struct TcClassPairs {
  static void run(int K, const int* pt, const int* ps, TcCells cv, double* Lcls, cudaStream_t st) {
    if constexpr (I < TcOrderClasses<P>::n) {
      constexpr int Q = TcOrderClasses<P>::q[I];
      constexpr int NTQ = (Q + 1) * (Q + 1), G = TcM2LGroups<Q>::G;
      size_t smem = (size_t)(NTQ * 32 + NTQ * 32 * G) * sizeof(double);
      cudaFuncSetAttribute(k_m2l_pairs<P, Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      k_m2l_pairs<P, Q><<<(K + 31) / 32, 128, smem, st>>>(K, pt, ps, cv, Lcls + (size_t)I * K * (P + 1) * (P + 1));
      TcClassPairs<P, I + 1>::run(K, pt, ps, cv, Lcls, st);
    }
  }
};

static void mlp_init_weights(std::vector<float>& w, int nout, unsigned long long seed) {
  std::mt19937_64 rng(seed);
  auto fill = [&](float* a, int fan_out, int fan_in) {
    float lim = sqrtf(6.f / (float)(fan_in + fan_out));
    std::uniform_real_distribution<float> U(-lim, lim);
    for (int i = 0; i < fan_out * fan_in; i++) a[i] = U(rng);
    for (int i = 0; i < fan_out; i++) a[fan_out * fan_in + i] = 0.f;
  };
  w.assign(tc_mlp_nparam(nout), 0.f);
  float* p = w.data();
  fill(p, kMlpH, kMlpIn);
  p += kMlpH * kMlpIn + kMlpH;
  fill(p, kMlpH, kMlpH);
  p += kMlpH * kMlpH + kMlpH;
  fill(p, kMlpH, kMlpH);
  p += kMlpH * kMlpH + kMlpH;
  fill(p, nout, kMlpH);
}

// gradient descent on (feat, lab) resident on the device; returns final losses
static cudaError_t mlp_fit(int ntrain, int nval, int nout, const float* d_feat, const float* d_lab, float* d_w,
                           const TcMlpNorm& norm, int iters, cudaStream_t st, double* train_loss, double* val_loss) {
  const int np = tc_mlp_nparam(nout);
  float *g = nullptr, *m1 = nullptr, *m2 = nullptr, *loss = nullptr, *gs = nullptr;
  cudaError_t e = cudaMalloc((void**)&g, np * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc((void**)&gs, np * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc((void**)&m1, np * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc((void**)&m2, np * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc((void**)&loss, 2 * sizeof(float));
  if (e == cudaSuccess) {
    cudaMemsetAsync(g, 0, np * sizeof(float), st);
    cudaMemsetAsync(m1, 0, np * sizeof(float), st);
    cudaMemsetAsync(m2, 0, np * sizeof(float), st);
    int blocks = std::min(148 * 2, (ntrain + 255) / 256);
    for (int it = 1; it <= iters; it++) {
      float lr = 3e-3f * (it < iters / 2 ? 1.f : (it < 3 * iters / 4 ? 0.3f : 0.1f));
      k_mlp_grad<<<blocks, 256, 0, st>>>(ntrain, nout, d_feat, d_lab, d_w, norm, g, loss);
      k_mlp_adam<<<(np + 255) / 256, 256, 0, st>>>(np, d_w, g, m1, m2, lr, 0.9f, 0.999f, 1e-8f, it);
    }
    cudaMemsetAsync(loss, 0, 2 * sizeof(float), st);
    cudaMemsetAsync(gs, 0, np * sizeof(float), st);
    k_mlp_grad<<<blocks, 256, 0, st>>>(ntrain, nout, d_feat, d_lab, d_w, norm, gs, loss);
    if (nval > 0)
      k_mlp_grad<<<std::min(148, (nval + 255) / 256), 256, 0, st>>>(nval, nout, d_feat + (size_t)ntrain * kMlpIn,
                                                                     d_lab + (size_t)ntrain * nout, d_w, norm, gs,
                                                                     loss + 1);
    float hl[2] = {0, 0};
    e = cudaMemcpyAsync(hl, loss, sizeof(hl), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    *train_loss = hl[0];
    *val_loss = hl[1];
  }
  cudaFree(g); cudaFree(gs); cudaFree(m1); cudaFree(m2); cudaFree(loss);
  return e == cudaSuccess ? cudaGetLastError() : e;
}

template <int P>
static tc_status train_selector(tc_ctx* ctx, int nsamples, int iters, unsigned long long seed, tc_train_report* rep) {
  using OC = TcOrderClasses<P>;
  constexpr int NTP = (P + 1) * (P + 1);
  cudaStream_t st = ctx->stream;
  const bool jerk = ctx->prm.variant == TC_VARIANT_JERKS;
  TcCells cv = cells_view(ctx, NTP);
  TcBodies b = bodies_view(ctx, ctx->n, jerk);
  const int K = (int)std::min<unsigned long long>((unsigned long long)nsamples, ctx->n_m2l);
  if (K < 16) return TC_ERR_ARG;
  // the fixed-order evaluation left the sorted (target, source) list in m2l
  std::vector<long long> idx(K);
  std::mt19937_64 rng(seed);
  std::uniform_int_distribution<unsigned long long> U(0, ctx->n_m2l - 1);
  for (int k = 0; k < K; k++) idx[k] = (long long)U(rng);
  long long* d_idx = nullptr;
  int *pt = nullptr, *ps = nullptr;
  double* Lcls = nullptr;
  float *d_feat = nullptr, *d_lab = nullptr;
  const int nc = ctx->ncell;
  TC_CK(ctx->cell_pn.ensure((size_t)nc * (P + 1)));
  TC_CK(cudaMalloc((void**)&d_idx, K * sizeof(long long)));
  TC_CK(cudaMalloc((void**)&pt, K * sizeof(int)));
  TC_CK(cudaMalloc((void**)&ps, K * sizeof(int)));
  TC_CK(cudaMalloc((void**)&Lcls, (size_t)OC::n * K * NTP * sizeof(double)));
  TC_CK(cudaMalloc((void**)&d_feat, (size_t)K * kMlpIn * sizeof(float)));
  TC_CK(cudaMalloc((void**)&d_lab, (size_t)K * OC::n * sizeof(float)));
  TC_CK(cudaMemcpyAsync(d_idx, idx.data(), K * sizeof(long long), cudaMemcpyHostToDevice, st));
  k_gather_pairs<<<(K + 255) / 256, 256, 0, st>>>(K, ctx->m2l.p, d_idx, ctx->sbits, pt, ps);
  k_cell_pn<P><<<nblocks(nc, 128), 128, 0, st>>>(nc, cv.M, ctx->cell_pn.p);
  TcClassPairs<P, 0>::run(K, pt, ps, cv, Lcls, st);
  k_pair_eval<P><<<K, 128, 0, st>>>(K, OC::n, pt, ps, b, cv, ctx->cell_pn.p, Lcls, d_lab);
  k_pair_features<P><<<(K + 255) / 256, 256, 0, st>>>(K, pt, ps, cv, ctx->cell_pn.p, d_feat);
  ctx->train_feat.resize((size_t)K * kMlpIn);
  ctx->train_lab.resize((size_t)K * OC::n);
  TC_CK(cudaMemcpyAsync(ctx->train_feat.data(), d_feat, ctx->train_feat.size() * sizeof(float),
                        cudaMemcpyDeviceToHost, st));
  TC_CK(cudaMemcpyAsync(ctx->train_lab.data(), d_lab, ctx->train_lab.size() * sizeof(float), cudaMemcpyDeviceToHost,
                        st));
  TC_CK(cudaStreamSynchronize(st));
  ctx->train_n = K;
  // standardisation from the training part
  const int ntrain = (K * 4) / 5, nval = K - ntrain;
  TcMlpNorm norm;
  double lab_mean = 0;
  for (int i = 0; i < kMlpIn; i++) {
    double s1 = 0, s2 = 0;
    for (int k = 0; k < ntrain; k++) {
      double v = ctx->train_feat[(size_t)k * kMlpIn + i];
      s1 += v;
      s2 += v * v;
    }
    double mu = s1 / ntrain, var = std::max(s2 / ntrain - mu * mu, 1e-12);
    norm.mean[i] = (float)mu;
    norm.inv_std[i] = (float)(1.0 / sqrt(var));
  }
  for (int k = 0; k < ntrain * OC::n; k++) lab_mean += ctx->train_lab[k];
  norm.out_mean = (float)(lab_mean / (ntrain * OC::n));
  std::vector<float> w;
  mlp_init_weights(w, OC::n, seed ^ 0x9e3779b97f4a7c15ull);
  TC_CK(ctx->mlp_w.ensure(w.size()));
  TC_CK(cudaMemcpyAsync(ctx->mlp_w.p, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice, st));
  double tl = 0, vl = 0;
  TC_CK(mlp_fit(ntrain, nval, OC::n, d_feat, d_lab, ctx->mlp_w.p, norm, iters, st, &tl, &vl));
  ctx->mlp_norm = norm;
  ctx->mlp_nout = OC::n;
  ctx->mlp_ready = true;
  cudaFree(d_idx); cudaFree(pt); cudaFree(ps); cudaFree(Lcls); cudaFree(d_feat); cudaFree(d_lab);
  if (rep) {
    rep->samples = K;
    rep->iters = iters;
    rep->n_classes = OC::n;
    for (int i = 0; i < 6; i++) rep->class_order[i] = i < OC::n ? OC::at(i) : 0;
    rep->train_loss = tl;
    rep->val_loss = vl;
  }
  return TC_OK;
}

// ----------------------------------------------------------------------------------------
// per-order evaluation body
// ----------------------------------------------------------------------------------------
template <int P, bool JERK>
static tc_status run_fmm(tc_ctx* ctx, int n) {
  constexpr int NT = (P + 1) * (P + 1);
  cudaStream_t st = ctx->stream;
  const tc_params& prm = ctx->prm;
  TcBodies b = bodies_view(ctx, n, JERK);
  ctx->ncell = 0;
  // ---- tree levels
  TcCells cv = cells_view(ctx, NT);
  k_tree_root<<<1, 1, 0, st>>>(n, cv, ctx->d_root, ctx->d_lv);
  ctx->launches += 1 + 3 * (TC_MAX_LEVEL + 1);
  int tgrid = 148 * 8;
  for (int l = 0; l < TC_MAX_LEVEL + 1; l++) {
    k_tree_split<<<tgrid, 128, 0, st>>>(l, prm.ncrit, b, cv, ctx->d_lv, ctx->split_off.p, ctx->d_err);
    k_tree_scan<<<1, 1024, 0, st>>>(l, cv, ctx->d_lv, (int)ctx->ccap, ctx->d_err);
    k_tree_emit<<<tgrid, 128, 0, st>>>(l, cv, ctx->d_lv, ctx->split_off.p, ctx->d_root);
  }
  TC_CK(cudaMemcpyAsync(&ctx->lv, ctx->d_lv, sizeof(TcLevels), cudaMemcpyDeviceToHost, st));
  unsigned herr = 0;
  TC_CK(cudaMemcpyAsync(&herr, ctx->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  TC_CK(cudaStreamSynchronize(st));
  if (herr & TC_EBIT_NAN) return TC_ERR_NAN_INPUT;
  if (herr & TC_EBIT_CELL_CAP) return TC_ERR_CAPACITY;
  ctx->tree_flags = herr;
  ctx->ncell = ctx->lv.ncell;
  int maxl = 0;
  for (int l = 0; l <= TC_MAX_LEVEL; l++)
    if (ctx->lv.count[l] > 0) maxl = l;
  ctx->max_level = maxl;
  if (ctx->events) cudaEventRecord(ctx->ev[1], st);
  // ---- expansions
  size_t ne = (size_t)ctx->ncell * NT;
  TC_CK(ctx->expn.ensure(ne * (JERK ? 4 : 2)));
  ctx->expn_stride = (size_t)ctx->ncell;
  cv = cells_view(ctx, NT);
  TC_CK(cudaMemsetAsync(cv.L, 0, ne * sizeof(double), st));
  if (JERK) TC_CK(cudaMemsetAsync(cv.Ld, 0, ne * sizeof(double), st));
  // ---- upward, deepest level first
  int* d_start = &((TcLevels*)ctx->d_lv)->start[0];
  int* d_count = &((TcLevels*)ctx->d_lv)->count[0];
  ctx->launches += maxl + 3;
  {
    int g = nblocks(ctx->ncell, kUpWarps);
    if (g > 148 * 16) g = 148 * 16;
    k_leaf_balls<<<g, kUpWarps * 32, 0, st>>>(ctx->ncell, b, cv, ctx->d_err);
    g = nblocks(ctx->ncell, kP2MWarps);
    if (g > 148 * 16) g = 148 * 16;
    k_p2m_leaves<P, JERK><<<g, kP2MWarps * 32, 0, st>>>(ctx->ncell, b, cv);
  }
  for (int l = maxl; l >= 0; l--) {
    int cnt = ctx->lv.count[l];
    int g = nblocks(cnt, TcTransW<P>::W);
    if (g > 148 * 16) g = 148 * 16;
    k_upward_level<P, JERK><<<g, TcTransW<P>::W * 32, 0, st>>>(l, b, cv, d_start, d_count, ctx->d_err);
  }
  if (ctx->events) cudaEventRecord(ctx->ev[2], st);
  // ---- traversal, list sort and per-target offsets (lists of the acceptance test `mac` over the
  // cells `cvm`: the error-MAC pre-pass runs it on the geometric cells first)
  int sbits = 1;
  while ((1 << sbits) < ctx->ncell) sbits++;
  ctx->sbits = sbits;
  double theta2 = prm.theta * prm.theta;
  unsigned hs[4];
  auto build_lists = [&](const TcCells& cvm, const TcMac& mac) -> tc_status {
  for (int attempt = 0; attempt < 6; attempt++) {
    size_t want_m = ctx->mcap ? ctx->mcap : (size_t)ctx->ncell * 640 + 65536;
    size_t want_p = ctx->pcap ? ctx->pcap : (size_t)ctx->ncell * 240 + 65536;
    size_t want_f = ctx->fcap ? ctx->fcap : (size_t)ctx->ncell * 256 + 65536;
    TC_CK(ctx->front[0].ensure(want_f));
    TC_CK(ctx->front[1].ensure(want_f));
    TC_CK(ctx->m2l.ensure(want_m));
    TC_CK(ctx->p2p.ensure(want_p));
    ctx->mcap = ctx->m2l.n;
    ctx->pcap = ctx->p2p.n;
    ctx->fcap = ctx->front[0].n < ctx->front[1].n ? ctx->front[0].n : ctx->front[1].n;
    TC_CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(unsigned), st));
    k_trav_init<<<1, 1, 0, st>>>(ctx->front[0].p, ctx->d_cnt);
    int nsteps = 2 * (maxl + 1) + 2;
    ctx->launches += 1 + nsteps;
    for (int s = 0; s < nsteps; s++)
      k_trav_step<<<148 * 8, 256, 0, st>>>(s, ctx->front[s & 1].p, ctx->front[(s + 1) & 1].p, ctx->fcap, ctx->d_cnt,
                                           cvm, theta2, prm.variant == TC_VARIANT_TOP, sbits, ctx->m2l.p, ctx->mcap,
                                           ctx->p2p.p, ctx->pcap, ctx->d_err, mac);
    TcTravCounters hc;
    TC_CK(cudaMemcpyAsync(&hc, ctx->d_cnt, sizeof(hc), cudaMemcpyDeviceToHost, st));
    TC_CK(cudaMemcpyAsync(&herr, ctx->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    TC_CK(cudaStreamSynchronize(st));
    bool grow = false;
    if (herr & TC_EBIT_M2L_CAP) { ctx->mcap = (size_t)(hc.n_m2l * 1.25) + 4096; grow = true; }
    if (herr & TC_EBIT_P2P_CAP) { ctx->pcap = (size_t)(hc.n_p2p * 1.25) + 4096; grow = true; }
    if (herr & TC_EBIT_FRONTIER_CAP) { ctx->fcap = ctx->fcap * 4; grow = true; }
    unsigned long long left = hc.frontier[nsteps % 3];
    if (left != 0) { ctx->err = "traversal did not finish"; return TC_ERR_CAPACITY; }
    if (!grow) {
      ctx->n_m2l = hc.n_m2l;
      ctx->n_p2p = hc.n_p2p;
      break;
    }
    if (attempt == 5) return TC_ERR_CAPACITY;
  }
  // ---- sort lists and build per-target offsets
  int kbits = 2 * sbits;
  {
    size_t nm = ctx->n_m2l, np = ctx->n_p2p;
    size_t mx = nm > np ? nm : np;
    if (mx < (size_t)n) mx = (size_t)n;
    size_t hist_need = 257 * ((mx + kRsTile - 1) / kRsTile + 1) + 1024;
    TC_CK(ctx->hist.ensure(hist_need));
    TC_CK(ctx->m2l_alt.ensure(nm + 1));
    TC_CK(ctx->p2p_alt.ensure(np + 1));
    ctx->launches += radix_sort(ctx->m2l.p, nullptr, ctx->m2l_alt.p, nullptr, (int)nm, kbits, ctx->hist.p, st);
    ctx->launches += radix_sort(ctx->p2p.p, nullptr, ctx->p2p_alt.p, nullptr, (int)np, kbits, ctx->hist.p, st);
    ctx->launches += 5;
    TC_CK(ctx->m2l_start.ensure(ctx->ncell + 1));
    TC_CK(ctx->p2p_start.ensure(ctx->ncell + 1));
    TC_CK(ctx->m2l_src.ensure(nm + 1));
    TC_CK(ctx->p2p_src.ensure(np + 1));
    TC_CK(ctx->m2l_tl.ensure(ctx->ncell));
    TC_CK(ctx->p2p_tl.ensure(ctx->ncell));
    TC_CK(ctx->leaves.ensure(ctx->ncell));
    k_list_csr<<<148 * 8, 256, 0, st>>>(ctx->m2l.p, nm, ctx->ncell, sbits, ctx->m2l_start.p, ctx->m2l_src.p);
    k_list_csr<<<148 * 8, 256, 0, st>>>(ctx->p2p.p, np, ctx->ncell, sbits, ctx->p2p_start.p, ctx->p2p_src.p);
    TC_CK(cudaMemsetAsync(ctx->d_small, 0, 4 * sizeof(unsigned), st));
    TC_CK(cudaMemsetAsync(&ctx->d_cnt->frontier[0], 0, sizeof(unsigned long long), st));
    k_p2p_count<<<148 * 4, 256, 0, st>>>(ctx->p2p.p, np, sbits, cv.nbody, cv.has_sink, &ctx->d_cnt->frontier[0]);
    ctx->launches++;
    k_list_targets<<<nblocks(ctx->ncell, 256), 256, 0, st>>>(ctx->m2l_start.p, ctx->ncell, ctx->m2l_tl.p, ctx->d_small);
    k_list_targets<<<nblocks(ctx->ncell, 256), 256, 0, st>>>(ctx->p2p_start.p, ctx->ncell, ctx->p2p_tl.p, ctx->d_small + 1);
    k_leaf_list<<<nblocks(ctx->ncell, 256), 256, 0, st>>>(ctx->ncell, cv.nchild, ctx->leaves.p, ctx->d_small + 2);
  }
  TC_CK(cudaMemcpyAsync(hs, ctx->d_small, sizeof(hs), cudaMemcpyDeviceToHost, st));
  TC_CK(cudaMemcpyAsync(&ctx->n_inter, &ctx->d_cnt->frontier[0], sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  TC_CK(cudaStreamSynchronize(st));
    return TC_OK;
  };
  TcMac mac;  // theta
  mac.p2p_max = p2p_instead_max(prm);
  if (ctx->emac) {
    // ---- low-order pre-pass on the geometric cells -> acc_old (integrator.h:476-493;
    // taichi_with_jerks/integrator.h:326-360)
    const int nc = ctx->ncell;
    TC_CK(ctx->low_rgeo.ensure(nc));
    TC_CK(ctx->low_m9.ensure((size_t)nc * kLowNT));
    TC_CK(ctx->low_l9.ensure((size_t)nc * kLowNT));
    TC_CK(ctx->acc_old.ensure(n));
    TC_CK(ctx->cell_of.ensure(n));
    TC_CK(ctx->min_acc.ensure(nc));
    TC_CK(ctx->pn_ref.ensure((size_t)nc * (P + 1)));
    const int gc = std::min(nblocks(nc, 128), 148 * 16);
    const int gb = std::min(nblocks(n, 128), 148 * 16);
    k_low_rgeo<<<gc, 128, 0, st>>>(nc, cv.level, ctx->d_root, ctx->low_rgeo.p);
    k_low_p2m<<<gc, 128, 0, st>>>(nc, b, cv, ctx->low_m9.p);
    for (int l = maxl; l >= 0; l--) k_low_m2m<<<gc, 128, 0, st>>>(l, cv, d_start, d_count, ctx->low_m9.p);
    TcCells geo = cv;
    geo.X = cv.gx; geo.Y = cv.gy; geo.Z = cv.gz; geo.R = ctx->low_rgeo.p;
    TcMac low;
    low.mode = 1;
    tc_status rl = build_lists(geo, low);
    if (rl != TC_OK) return rl;
    TC_CK(cudaMemsetAsync(ctx->low_l9.p, 0, sizeof(double) * (size_t)nc * kLowNT, st));
    k_low_m2l<<<gc, 128, 0, st>>>(nc, cv, ctx->m2l_start.p, ctx->m2l_src.p, ctx->low_m9.p, ctx->low_l9.p);
    k_low_cell_of<<<gc, 128, 0, st>>>(nc, cv, ctx->cell_of.p);
    if (JERK) {
      TC_CK(ctx->low_f.ensure(3 * (size_t)n));
      k_low_p2p_jerks<<<gb, 128, 0, st>>>(n, b, cv, ctx->cell_of.p, ctx->p2p_start.p, ctx->p2p_src.p, ctx->low_f.p);
    } else {
      k_low_p2p<<<gb, 128, 0, st>>>(n, b, cv, ctx->cell_of.p, ctx->p2p_start.p, ctx->p2p_src.p, ctx->acc_old.p);
    }
    for (int l = 0; l < maxl; l++) k_low_l2l<<<gc, 128, 0, st>>>(l, cv, d_start, d_count, ctx->low_l9.p);
    if (JERK)
      k_low_l2p_jerks<<<gb, 128, 0, st>>>(n, b, cv, ctx->cell_of.p, ctx->low_l9.p, ctx->low_f.p, ctx->acc_old.p);
    else
      k_low_l2p<<<gb, 128, 0, st>>>(n, b, cv, ctx->cell_of.p, ctx->low_l9.p, ctx->acc_old.p);
    // ---- MAC inputs: min_acc (bottom-up) and Pn of the reference's form
    for (int l = maxl; l >= 0; l--)
      k_min_acc<<<gc, 128, 0, st>>>(l, cv, d_start, d_count, ctx->acc_old.p, ctx->min_acc.p);
    k_cell_pn_ref<P><<<gc, 128, 0, st>>>(nc, cv.M, ctx->pn_ref.p);
    ctx->launches += 7 + 3 * (maxl + 1);
    mac.mode = JERK ? 3 : 2;
    mac.p = P;
    mac.fa = ctx->emac_fa;
    mac.pn = ctx->pn_ref.p;
    mac.min_acc = ctx->min_acc.p;
    // combinator_coef[P][k] = P! / (k! (P-k)!) as the reference forms it (kernel_fast_lean.h:139)
    double fact[2 * TC_PMAX_DEV + 2];
    fact[0] = 1.0;
    for (int i = 1; i < 2 * TC_PMAX_DEV + 2; i++) fact[i] = fact[i - 1] * (double)i;
    for (int k = 0; k <= P; k++) mac.comb[k] = fact[P] * (1.0 / fact[k]) * (1.0 / fact[P - k]);
  }
  {
    tc_status rh = build_lists(cv, mac);
    if (rh != TC_OK) return rh;
  }
  ctx->nleaf = (int)hs[2];
  if (ctx->events) cudaEventRecord(ctx->ev[3], st);
  // ---- far field and near field
  TcOut o = out_view(ctx, n, JERK);
  TC_CK(cudaMemsetAsync(ctx->outs.p, 0, sizeof(double) * (size_t)n * (JERK ? 7 : 4), st));
  const bool mixed = prm.precision == TC_PREC_MIXED_M2L;              // FP32 far field
  const bool mixed_p2p = prm.precision != TC_PREC_FP64;               // FP32 near field
  ctx->n_classes = 1;
  ctx->class_order[0] = P;
  ctx->class_pairs[0] = (long long)ctx->n_m2l;
  ctx->flop_frac = 1.0;
  if (ctx->steps) {
    // time-step pass: no far field (the reference skips M2L when get_steps is set)
  } else if (hs[0] > 0) {
    const int* m2l_src = ctx->m2l_src.p;
    bool classes = false;
    if (prm.selector > 0 && !mixed && TcOrderClasses<P>::n > 1 && ctx->amag_n == n &&
        (prm.selector == 1 || ctx->mlp_ready)) {
      cudaError_t ce = select_orders<P>(ctx, cv, n, (int)hs[0], nullptr, false);
      if (ce != cudaSuccess) return cuda_fail(ctx, ce, "order selection");
      m2l_class_launches<P, JERK>(ctx, cv, (int)hs[0], nullptr, ctx->ncell);
      unsigned h[32];
      TC_CK(cudaMemcpyAsync(h, ctx->d_hist, sizeof(h), cudaMemcpyDeviceToHost, st));
      TC_CK(cudaStreamSynchronize(st));
      order_stats(ctx, P, h, TcOrderClasses<P>::q, TcOrderClasses<P>::n);
      classes = true;
    }
    if (classes) {
      // done: one launch per order class
    } else
    if (mixed && P <= TC_TC_QMAX) {
      if constexpr (P <= TC_TC_QMAX) {
        TC_CK(tc_ensure_bins<P>(ctx));
        TC_CK(cudaMemsetAsync(ctx->d_small + 9, 0, sizeof(unsigned), st));
        int grid = std::min((int)hs[0], ctx->nsm);
        k_m2l_tc<P, P, JERK><<<grid, 128, TcTcSmem<P>::TOTAL, st>>>(ctx->m2l_tl.p, (int)hs[0], ctx->m2l_start.p,
                                                                     ctx->m2l_src.p, cv, ctx->tc_bins.p,
                                                                     ctx->d_small + 9, ctx->d_err, ctx->wait_limit);
      }
    } else if (mixed) {
      size_t smem = (size_t)TcM2LMixSmem<P>::BYTES;
      k_m2l_mixed<P, JERK><<<hs[0], tc_m2lx_threads<P>(), smem, st>>>(ctx->m2l_tl.p, (int)hs[0], ctx->m2l_start.p,
                                                                        ctx->m2l_src.p, cv);
    } else {
      size_t smem = (size_t)TcM2LSmem<P>::TOTAL * sizeof(double);
      k_m2l<P, P, JERK><<<hs[0], tc_m2l_threads<P>(), smem, st>>>(ctx->m2l_tl.p, (int)hs[0], ctx->m2l_start.p,
                                                                     m2l_src, cv);
    }
    ctx->launches++;
  }
  if (ctx->events) cudaEventRecord(ctx->ev[4], st);
  // ---- downward, before the near field (the mixed near field reads the far-field
  // acceleration); nothing to add in the time-step pass, where every local expansion is zero
  if (!ctx->steps) {
    ctx->launches += maxl + (ctx->nleaf > 0);
    for (int l = 1; l <= maxl; l++) {
      int cnt = ctx->lv.count[l];
      int g = nblocks(cnt, TcTransW<P>::W);
      if (g > 148 * 16) g = 148 * 16;
      k_l2l_level<P, JERK><<<g, TcTransW<P>::W * 32, 0, st>>>(l, cv, d_start, d_count);
    }
    if (ctx->nleaf > 0) {
      int g = nblocks(ctx->nleaf, kUpWarps);
      if (g > 148 * 32) g = 148 * 32;
      k_l2p<P, JERK><<<g, kUpWarps * 32, 0, st>>>(ctx->leaves.p, ctx->nleaf, b, cv, o);
    }
  }
  if (ctx->events) cudaEventRecord(ctx->ev[5], st);
  if (ctx->steps) {
    TC_CK(ctx->tsum.ensure((size_t)n));
    TC_CK(cudaMemsetAsync(ctx->tsum.p, 0, sizeof(double) * (size_t)n, st));
  }
  if (hs[1] > 0 && ctx->steps) {
    if constexpr (!JERK) {
      const int ntl = (int)hs[1];
      int nsplit = p2p_nsplit(n);  // few target leaves: source chunks folded in order, as k_p2p
      if (nsplit > 1 && ctx->p2p_part.ensure((size_t)nsplit * 5 * n) != cudaSuccess) nsplit = 1;
      if (nsplit > 1) {
        k_p2p_steps<<<nblocks(ntl * nsplit, kP2PWarps), kP2PWarps * 32, 0, st>>>(
            ctx->p2p_tl.p, ntl, ctx->p2p_start.p, ctx->p2p_src.p, b, cv, o, ctx->dt_param, ctx->tsum.p, nsplit,
            ctx->p2p_part.p, n);
        k_p2p_steps_join<<<nblocks(ntl, kP2PWarps), kP2PWarps * 32, 0, st>>>(ctx->p2p_tl.p, ntl, b, cv, o,
                                                                             ctx->tsum.p, nsplit, ctx->p2p_part.p, n);
        ctx->launches++;
      } else {
        k_p2p_steps<<<nblocks(ntl, kP2PWarps), kP2PWarps * 32, 0, st>>>(ctx->p2p_tl.p, ntl, ctx->p2p_start.p,
                                                                        ctx->p2p_src.p, b, cv, o, ctx->dt_param,
                                                                        ctx->tsum.p);
      }
      ctx->launches++;
    }
  } else if (hs[1] > 0) {
    int g = nblocks(hs[1], kP2PWarps);
    if (mixed_p2p) {
      k_body_f32<JERK><<<nblocks(n, 256), 256, 0, st>>>(n, b);
      ctx->launches++;
      k_p2p_mixed<JERK><<<g, kP2PWarps * 32, 0, st>>>(ctx->p2p_tl.p, (int)hs[1], ctx->p2p_start.p, ctx->p2p_src.p, b,
                                                       cv, o, kP2PExclFrac);
    } else {
      // few target leaves (small n): split each leaf's sources over up to 16 warps, then fold
      // the chunks in order (k_p2p_join); the split depends on n only, as in the graph path
      const int ntl = (int)hs[1];
      int nsplit = p2p_nsplit(n);
      constexpr int NC = JERK ? 7 : 4;
      if (nsplit > 1 && ctx->p2p_part.ensure((size_t)nsplit * NC * n) != cudaSuccess) nsplit = 1;
      if (nsplit > 1) {
        k_p2p<JERK><<<nblocks(ntl * nsplit, kP2PWarps), kP2PWarps * 32, 0, st>>>(
            ctx->p2p_tl.p, ntl, ctx->p2p_start.p, ctx->p2p_src.p, b, cv, o, nullptr, nsplit, ctx->p2p_part.p, n);
        k_p2p_join<JERK><<<g, kP2PWarps * 32, 0, st>>>(ctx->p2p_tl.p, ntl, b, cv, o, nsplit, ctx->p2p_part.p, n);
        ctx->launches++;
      } else {
        k_p2p<JERK><<<g, kP2PWarps * 32, 0, st>>>(ctx->p2p_tl.p, ntl, ctx->p2p_start.p, ctx->p2p_src.p, b, cv, o);
      }
    }
    ctx->launches++;
  }
  if (ctx->events) cudaEventRecord(ctx->ev[6], st);
  return TC_OK;
}

// timing event inside a capture: an external record node, so the replay records it
static inline void graph_event(tc_ctx* ctx, int i, cudaStream_t st) {
  if (ctx->events) cudaEventRecordWithFlags(ctx->ev[i], st, cudaEventRecordExternal);
}

// first failing stage of a capture (a launch that fails is left out of the graph without
// invalidating the capture, so every stage is checked)
static void graph_check(tc_ctx* ctx, const char* stage) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess && ctx->gfail.empty()) ctx->gfail = std::string(stage) + ": " + cudaGetErrorString(e);
}

// Device-sized form of run_fmm for a captured CUDA graph (tc_set_graph): no host reads.  Every
// launch is sized by the capacities fixed when the graph was planned (ccap cells, mcap / pcap
// list entries, fcap frontier pairs) and reads its count on the device (levels, list sizes,
// target and leaf counts); loops over levels run to TC_MAX_LEVEL (empty levels exit at once).
// An overflow sets d_err bits (the tree then stays consistent, the lists are clamped), which
// the host reads after the replay before it uses the outputs.  FP64 / MIXED far field, fixed
// order, no time-step pass.
template <int P, bool JERK>
static void run_fmm_graph(tc_ctx* ctx, int n) {
  constexpr int NT = (P + 1) * (P + 1);
  cudaStream_t st = ctx->stream;
  const tc_params& prm = ctx->prm;
  TcBodies b = bodies_view(ctx, n, JERK);
  TcCells cv = cells_view(ctx, NT);
  const int ccap = (int)ctx->ccap;
  const int* d_ncell = &ctx->d_lv->ncell;
  int* d_start = &ctx->d_lv->start[0];
  int* d_count = &ctx->d_lv->count[0];
  long long L = 0;
  // ---- tree levels (as run_fmm)
  k_tree_root<<<1, 1, 0, st>>>(n, cv, ctx->d_root, ctx->d_lv);
  const int tgrid = 148 * 8;
  for (int l = 0; l < TC_MAX_LEVEL + 1; l++) {
    k_tree_split<<<tgrid, 128, 0, st>>>(l, prm.ncrit, b, cv, ctx->d_lv, ctx->split_off.p, ctx->d_err);
    k_tree_scan<<<1, 1024, 0, st>>>(l, cv, ctx->d_lv, ccap, ctx->d_err);
    k_tree_emit<<<tgrid, 128, 0, st>>>(l, cv, ctx->d_lv, ctx->split_off.p, ctx->d_root);
  }
  L += 1 + 3 * (TC_MAX_LEVEL + 1);
  graph_check(ctx, "tree");
  graph_event(ctx, 1, st);
  // ---- expansions (capacity-strided) and upward pass
  const size_t ne = (size_t)ccap * NT;
  cudaMemsetAsync(cv.L, 0, ne * sizeof(double), st);
  if (JERK) cudaMemsetAsync(cv.Ld, 0, ne * sizeof(double), st);
  {
    int g = std::min(nblocks(ccap, kUpWarps), 148 * 16);
    k_leaf_balls<<<g, kUpWarps * 32, 0, st>>>(ccap, b, cv, ctx->d_err, ctx->d_lv);
    g = std::min(nblocks(ccap, kP2MWarps), 148 * 16);
    k_p2m_leaves<P, JERK><<<g, kP2MWarps * 32, 0, st>>>(ccap, b, cv, ctx->d_lv);
  }
  for (int l = TC_MAX_LEVEL; l >= 0; l--)
    k_upward_level<P, JERK><<<148 * 16, TcTransW<P>::W * 32, 0, st>>>(l, b, cv, d_start, d_count, ctx->d_err);
  L += 2 + TC_MAX_LEVEL + 1;
  graph_check(ctx, "upward pass");
  graph_event(ctx, 2, st);
  // ---- traversal
  const int sbits = ctx->gsbits;
  const double theta2 = prm.theta * prm.theta;
  k_trav_init<<<1, 1, 0, st>>>(ctx->front[0].p, ctx->d_cnt);
  const int nsteps = 2 * (TC_MAX_LEVEL + 1) + 2;
  {
    TcMac mac;  // theta
    mac.p2p_max = p2p_instead_max(prm);
    for (int s = 0; s < nsteps; s++)
      k_trav_step<<<148 * 8, 256, 0, st>>>(s, ctx->front[s & 1].p, ctx->front[(s + 1) & 1].p, ctx->fcap, ctx->d_cnt,
                                           cv, theta2, prm.variant == TC_VARIANT_TOP, sbits, ctx->m2l.p, ctx->mcap,
                                           ctx->p2p.p, ctx->pcap, ctx->d_err, mac);
  }
  L += 1 + nsteps;
  graph_check(ctx, "traversal");
  // ---- sort lists (counts on the device) and per-target offsets
  const int kbits = 2 * sbits;
  unsigned long long *km = nullptr, *kp = nullptr;
  L += radix_sort(ctx->m2l.p, nullptr, ctx->m2l_alt.p, nullptr, (int)ctx->mcap, kbits, ctx->hist.p, st, 0,
                  &ctx->d_cnt->n_m2l, &km);
  L += radix_sort(ctx->p2p.p, nullptr, ctx->p2p_alt.p, nullptr, (int)ctx->pcap, kbits, ctx->hist.p, st, 0,
                  &ctx->d_cnt->n_p2p, &kp);
  k_list_csr<<<148 * 8, 256, 0, st>>>(km, ctx->mcap, ccap, sbits, ctx->m2l_start.p, ctx->m2l_src.p,
                                      &ctx->d_cnt->n_m2l, d_ncell);
  k_list_csr<<<148 * 8, 256, 0, st>>>(kp, ctx->pcap, ccap, sbits, ctx->p2p_start.p, ctx->p2p_src.p,
                                      &ctx->d_cnt->n_p2p, d_ncell);
  cudaMemsetAsync(ctx->d_small, 0, 4 * sizeof(unsigned), st);
  cudaMemsetAsync(&ctx->d_cnt->frontier[0], 0, sizeof(unsigned long long), st);
  k_p2p_count<<<148 * 4, 256, 0, st>>>(kp, ctx->pcap, sbits, cv.nbody, cv.has_sink, &ctx->d_cnt->frontier[0],
                                       &ctx->d_cnt->n_p2p);
  k_list_targets<<<nblocks(ccap, 256), 256, 0, st>>>(ctx->m2l_start.p, ccap, ctx->m2l_tl.p, ctx->d_small, d_ncell);
  k_list_targets<<<nblocks(ccap, 256), 256, 0, st>>>(ctx->p2p_start.p, ccap, ctx->p2p_tl.p, ctx->d_small + 1,
                                                     d_ncell);
  k_leaf_list<<<nblocks(ccap, 256), 256, 0, st>>>(ccap, cv.nchild, ctx->leaves.p, ctx->d_small + 2, d_ncell);
  L += 6;
  graph_check(ctx, "list sort and offsets");
  graph_event(ctx, 3, st);
  // ---- far field and near field
  TcOut o = out_view(ctx, n, JERK);
  cudaMemsetAsync(ctx->outs.p, 0, sizeof(double) * (size_t)n * (JERK ? 7 : 4), st);
  cudaMemsetAsync(ctx->d_small + 10, 0, sizeof(unsigned), st);
  if (TcOrderClasses<P>::n < 2) ctx->gselect = false;  // one class: nothing to select
  if (ctx->gselect) {  // per-pair orders (the previous replay left |a| in ctx->amag)
    for (int i = 0; i < TcOrderClasses<P>::n; i++) ctx->gcls_q[i] = TcOrderClasses<P>::q[i];
    ctx->gcls_n = TcOrderClasses<P>::n;
    select_orders<P>(ctx, cv, n, ccap, ctx->d_small, true);
    m2l_class_launches<P, JERK>(ctx, cv, ccap, ctx->d_small, ccap);
    L += 4 + TC_MAX_LEVEL + TcClassLaunches<P>::n;
    graph_check(ctx, "order selection");
  } else {
    k_m2l<P, P, JERK><<<ctx->nsm, tc_m2l_threads<P>(), (size_t)TcM2LSmem<P>::TOTAL * sizeof(double), st>>>(
        ctx->m2l_tl.p, ccap, ctx->m2l_start.p, ctx->m2l_src.p, cv, ctx->d_small, ctx->d_small + 10);
  }
  graph_check(ctx, "M2L");
  graph_event(ctx, 4, st);
  // ---- downward (before the near field: the mixed near field reads the far-field acceleration)
  for (int l = 1; l <= TC_MAX_LEVEL; l++)
    k_l2l_level<P, JERK><<<148 * 16, TcTransW<P>::W * 32, 0, st>>>(l, cv, d_start, d_count);
  {
    const int g = std::min(nblocks(ccap, kUpWarps), 148 * 32);
    k_l2p<P, JERK><<<g, kUpWarps * 32, 0, st>>>(ctx->leaves.p, ccap, b, cv, o, ctx->d_small + 2);
  }
  L += TC_MAX_LEVEL + 1;
  graph_check(ctx, "downward pass");
  graph_event(ctx, 5, st);
  {
    const int g = nblocks(ccap, kP2PWarps);  // a warp per target slot; warps past the count exit
    if (prm.precision != TC_PREC_FP64) {
      k_body_f32<JERK><<<nblocks(n, 256), 256, 0, st>>>(n, b);
      L++;
    }
    if (prm.precision != TC_PREC_FP64)
      k_p2p_mixed<JERK><<<g, kP2PWarps * 32, 0, st>>>(ctx->p2p_tl.p, ccap, ctx->p2p_start.p, ctx->p2p_src.p, b, cv, o,
                                                       kP2PExclFrac, ctx->d_small + 1);
    else {
      const int nsplit = p2p_nsplit(n);
      if (nsplit > 1) {  // the same chunks as the direct launches (p2p_part sized by graph_plan)
        k_p2p<JERK><<<nblocks(ccap * nsplit, kP2PWarps), kP2PWarps * 32, 0, st>>>(
            ctx->p2p_tl.p, ccap, ctx->p2p_start.p, ctx->p2p_src.p, b, cv, o, ctx->d_small + 1, nsplit,
            ctx->p2p_part.p, n);
        k_p2p_join<JERK><<<g, kP2PWarps * 32, 0, st>>>(ctx->p2p_tl.p, ccap, b, cv, o, nsplit, ctx->p2p_part.p, n,
                                                        ctx->d_small + 1);
        L++;
      } else {
        k_p2p<JERK><<<g, kP2PWarps * 32, 0, st>>>(ctx->p2p_tl.p, ccap, ctx->p2p_start.p, ctx->p2p_src.p, b, cv, o,
                                                   ctx->d_small + 1);
      }
    }
  }
  L += 2;
  graph_check(ctx, "P2P");
  graph_event(ctx, 6, st);
  ctx->glaunches += L;
}

typedef void (*graph_fn)(tc_ctx*, int);

typedef tc_status (*run_fn)(tc_ctx*, int);

// RMS relative acceleration error of the last evaluation (Morton-order outputs) at nt seeded
// bodies against FP64 direct sums
static tc_status judge(tc_ctx* ctx, int n, int nt, bool jerk, double* rms) {
  cudaStream_t st = ctx->stream;
  std::vector<int> idx(nt);
  std::mt19937_64 rng(ctx->prm.judge_seed);
  std::uniform_int_distribution<int> U(0, n - 1);
  for (int k = 0; k < nt; k++) idx[k] = U(rng);
  TC_CK(ctx->judge_idx.ensure(nt));
  const int nchunk = std::max(1, std::min(4 * ctx->nsm, n / 1024));
  TC_CK(ctx->judge_out.ensure(7 * (size_t)nt + 8 * (size_t)nt * nchunk));
  TC_CK(cudaMemcpyAsync(ctx->judge_idx.p, idx.data(), nt * sizeof(int), cudaMemcpyHostToDevice, st));
  TcBodies b = bodies_view(ctx, n, jerk);
  TcOut o = out_view(ctx, n, jerk);
  double* part = ctx->judge_out.p + 7 * (size_t)nt;
  k_direct_targets<false><<<dim3(nchunk, (nt + kJudgeTile - 1) / kJudgeTile), kJudgeTile, 0, st>>>(
      n, nt, nchunk, ctx->judge_idx.p, b, part);
  k_direct_targets_sum<<<nblocks(nt, 128), 128, 0, st>>>(nt, nchunk, ctx->judge_idx.p, part, o, ctx->judge_out.p);
  ctx->launches += 2;
  std::vector<double> ref(7 * (size_t)nt);
  TC_CK(cudaMemcpyAsync(ref.data(), ctx->judge_out.p, ref.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  TC_CK(cudaStreamSynchronize(st));
  double s = 0.0;
  for (int k = 0; k < nt; k++) {
    const double* r = &ref[7 * (size_t)k];
    double ex = r[4] - r[1], ey = r[5] - r[2], ez = r[6] - r[3];
    double an = r[1] * r[1] + r[2] * r[2] + r[3] * r[3];
    s += (ex * ex + ey * ey + ez * ez) / (an > 0 ? an : 1.0);
  }
  *rms = sqrt(s / nt);
  return TC_OK;
}

template <int P>
static void set_m2l_attrs() {
  set_class_attrs<P>();
  size_t smem = (size_t)TcM2LSmem<P>::TOTAL * sizeof(double);
  cudaFuncSetAttribute(k_m2l<P, P, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaFuncSetAttribute(k_m2l<P, P, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if constexpr (P <= TC_TC_QMAX) {
    cudaFuncSetAttribute(k_m2l_tc<P, P, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, TcTcSmem<P>::TOTAL);
    cudaFuncSetAttribute(k_m2l_tc<P, P, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, TcTcSmem<P>::TOTAL);
  }
  size_t smx = (size_t)TcM2LMixSmem<P>::BYTES;
  cudaFuncSetAttribute(k_m2l_mixed<P, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx);
  cudaFuncSetAttribute(k_m2l_mixed<P, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx);
}

#define TC_ORDERS(X) X(4) X(6) X(8) X(10) X(12) X(16)

static run_fn pick(int p, bool jerk) {
  switch (p) {
#define TC_CASE(P) \
  case P:          \
    return jerk ? run_fmm<P, true> : run_fmm<P, false>;
    TC_ORDERS(TC_CASE)
#undef TC_CASE
    default:
      return nullptr;
  }
}

static graph_fn pick_graph(int p, bool jerk) {
  switch (p) {
#define TC_CASE(P) \
  case P:          \
    return jerk ? run_fmm_graph<P, true> : run_fmm_graph<P, false>;
    TC_ORDERS(TC_CASE)
#undef TC_CASE
    default:
      return nullptr;
  }
}

static void set_attrs(int p) {
  switch (p) {
#define TC_CASE(P) \
  case P:          \
    set_m2l_attrs<P>(); \
    break;
    TC_ORDERS(TC_CASE)
#undef TC_CASE
    default:
      break;
  }
}

__global__ void k_kick_drift(int n, double* x, double* y, double* z, double* vx, double* vy, double* vz,
                             const double* ax, const double* ay, const double* az, double dk, double dd) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double u = vx[i] + ax[i] * dk, v = vy[i] + ay[i] * dk, w = vz[i] + az[i] * dk;
  vx[i] = u; vy[i] = v; vz[i] = w;
  if (dd != 0.0) {
    x[i] += u * dd; y[i] += v * dd; z[i] += w * dd;
  }
}

// the closing kick of a captured leapfrog step: skipped when the evaluation before it overflowed a
// capacity (its accelerations are invalid; the host re-runs the evaluation and this kick)
__global__ void k_kick_guarded(int n, double* vx, double* vy, double* vz, const double* ax, const double* ay,
                               const double* az, double dk, const unsigned* err, unsigned mask) {
  if (*err & mask) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  vx[i] += ax[i] * dk;
  vy[i] += ay[i] * dk;
  vz[i] += az[i] * dk;
}

// Hermite 4th-order predictor (Makino & Aarseth 1992) in FP64: saves x0, v0, a0, j0 into
// save[12 n] (x y z, vx vy vz, ax ay az, jx jy jz) and writes the predicted x, v
__global__ void k_hermite_predict(int n, double* __restrict__ x, double* __restrict__ y, double* __restrict__ z,
                                  double* __restrict__ vx, double* __restrict__ vy, double* __restrict__ vz,
                                  const double* __restrict__ ax, const double* __restrict__ ay,
                                  const double* __restrict__ az, const double* __restrict__ jx,
                                  const double* __restrict__ jy, const double* __restrict__ jz,
                                  double* __restrict__ save, double dt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double* const X[3] = {x, y, z};
  double* const V[3] = {vx, vy, vz};
  const double* const A[3] = {ax, ay, az};
  const double* const J[3] = {jx, jy, jz};
  for (int d = 0; d < 3; d++) {
    const double x0 = X[d][i], v0 = V[d][i], a0 = A[d][i], j0 = J[d][i];
    save[(size_t)d * n + i] = x0;
    save[(size_t)(3 + d) * n + i] = v0;
    save[(size_t)(6 + d) * n + i] = a0;
    save[(size_t)(9 + d) * n + i] = j0;
    X[d][i] = x0 + dt * (v0 + dt * (a0 / 2 + dt * (j0 / 6)));
    V[d][i] = v0 + dt * (a0 + dt * (j0 / 2));
  }
}

// Hermite 4th-order corrector with the accelerations and jerks a1, j1 at the predicted state
__global__ void k_hermite_correct(int n, double* __restrict__ x, double* __restrict__ y, double* __restrict__ z,
                                  double* __restrict__ vx, double* __restrict__ vy, double* __restrict__ vz,
                                  const double* __restrict__ ax, const double* __restrict__ ay,
                                  const double* __restrict__ az, const double* __restrict__ jx,
                                  const double* __restrict__ jy, const double* __restrict__ jz,
                                  const double* __restrict__ save, double dt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double* const X[3] = {x, y, z};
  double* const V[3] = {vx, vy, vz};
  const double* const A[3] = {ax, ay, az};
  const double* const J[3] = {jx, jy, jz};
  for (int d = 0; d < 3; d++) {
    const double x0 = save[(size_t)d * n + i], v0 = save[(size_t)(3 + d) * n + i];
    const double a0 = save[(size_t)(6 + d) * n + i], j0 = save[(size_t)(9 + d) * n + i];
    const double a1 = A[d][i], j1 = J[d][i];
    const double v1 = v0 + dt / 2 * (a0 + a1) + dt * dt / 12 * (j0 - j1);
    V[d][i] = v1;
    X[d][i] = x0 + dt / 2 * (v0 + v1) + dt * dt / 12 * (a0 - a1);
  }
}

template <typename T>
__global__ void k_fma_probe(T* out, int iters) {
  T a0 = (T)threadIdx.x * (T)1e-3, a1 = a0 + (T)1, a2 = a0 + (T)2, a3 = a0 + (T)3;
  T a4 = a0 + (T)4, a5 = a0 + (T)5, a6 = a0 + (T)6, a7 = a0 + (T)7;
  const T b = (T)0.999999, c = (T)1e-7;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 16; k++) {
      a0 = a0 * b + c; a1 = a1 * b + c; a2 = a2 * b + c; a3 = a3 * b + c;
      a4 = a4 * b + c; a5 = a5 * b + c; a6 = a6 * b + c; a7 = a7 * b + c;
    }
  }
  if (a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7 == (T)-1) out[0] = a0;
}

// ----------------------------------------------------------------------------------------
// Scratch of tc_evaluate_direct_noalloc: a fixed static device array instead of cudaMalloc.
// Layout: 7 body arrays (x y z m vx vy vz) | 7 output arrays, each TC_NOALLOC_MAX_N doubles.
// ----------------------------------------------------------------------------------------
static __device__ __align__(256) double g_noalloc_scratch[14 * TC_NOALLOC_MAX_N];
static __device__ __align__(256) int g_noalloc_index[TC_NOALLOC_MAX_N];
static __device__ __align__(256) uint8_t g_noalloc_flags[TC_NOALLOC_MAX_N];

struct TcNoallocDev {
  double* scratch = nullptr;
  int* index = nullptr;
  uint8_t* flags = nullptr;
};
static TcNoallocDev g_noalloc_dev[64];
static std::mutex g_noalloc_mu;  // guards the one-time fill of g_noalloc_dev

// Direct-sum evaluation over working storage the caller provides: S entries per array in
// `scratch` (14 arrays: x y z m vx vy vz | pot ax ay az jx jy jz), `index` and `flags`
// (n <= S).  Shared by tc_evaluate_direct_noalloc (the static array) and the block-time-step
// integrator's direct kicks (the context's own buffers, so contexts never share storage).
static cudaError_t direct_with_scratch(int n, const double* x, const double* y, const double* z, const double* vx,
                                       const double* vy, const double* vz, const double* m,
                                       const unsigned char* flags, double* ax, double* ay, double* az, double* pot,
                                       double* jx, double* jy, double* jz, int jerk, cudaStream_t st,
                                       double* scratch, int* index, uint8_t* fl, size_t S, double eps2 = 0.0) {
  TcBodies b;
  b.x = scratch; b.y = scratch + S; b.z = scratch + 2 * S; b.m = scratch + 3 * S;
  b.vx = jerk ? scratch + 4 * S : nullptr; b.vy = jerk ? scratch + 5 * S : nullptr;
  b.vz = jerk ? scratch + 6 * S : nullptr;
  b.flags = fl;
  b.perm = index;
  b.eps2 = eps2;
  TcOut o;
  o.pot = scratch + 7 * S; o.ax = scratch + 8 * S; o.ay = scratch + 9 * S; o.az = scratch + 10 * S;
  o.jx = jerk ? scratch + 11 * S : nullptr; o.jy = jerk ? scratch + 12 * S : nullptr;
  o.jz = jerk ? scratch + 13 * S : nullptr;
  k_identity<<<nblocks(n, 256), 256, 0, st>>>(n, index);
  k_gather_bodies<<<nblocks(n, 256), 256, 0, st>>>(n, index, x, y, z, m, vx, vy, vz, flags, b);
  if (jerk)
    k_direct<true><<<nblocks(n, 128), 128, 0, st>>>(n, b, o);
  else
    k_direct<false><<<nblocks(n, 128), 128, 0, st>>>(n, b, o);
  k_scatter_out<<<nblocks(n, 256), 256, 0, st>>>(n, index, o, pot, ax, ay, az, jerk ? jx : nullptr, jy, jz);
  return cudaGetLastError();
}

// ----------------------------------------------------------------------------------------
// C ABI
// ----------------------------------------------------------------------------------------
extern "C" {

void tc_default_params(tc_params* prm) {
  memset(prm, 0, sizeof(*prm));
  prm->p = 12;
  prm->ncrit = 64;
  prm->theta = 0.4;
  prm->variant = TC_VARIANT_JERKS;
  prm->precision = TC_PREC_FP64;
  prm->direct_below = -1;
  prm->device = 0;
  prm->selector = 0;
  prm->selector_tol = 1e-9;
  prm->judge_n = 0;
  prm->judge_tol = 0.0;
  prm->judge_seed = 12345;
}

int tc_pmax(void) { return TC_PMAX; }

int tc_order_supported(int p) { return pick(p, false) != nullptr; }

int tc_tc_bins(int q, float* out, int cap) {
  std::vector<float> img;
  switch (q) {
    case 4: tc_build_bins<4>(img); break;
    case 6: tc_build_bins<6>(img); break;
    case 8: tc_build_bins<8>(img); break;
    case 10: tc_build_bins<10>(img); break;
    case 12: tc_build_bins<12>(img); break;
    default: return -1;
  }
  if (out) memcpy(out, img.data(), sizeof(float) * std::min((size_t)std::max(cap, 0), img.size()));
  return (int)img.size();
}

const char* tc_status_string(tc_status s) {
  switch (s) {
    case TC_OK: return "ok";
    case TC_ERR_ARG: return "invalid argument";
    case TC_ERR_CUDA: return "CUDA error";
    case TC_ERR_CAPACITY: return "capacity exceeded";
    case TC_ERR_NAN_INPUT: return "non-finite position or mass";
    case TC_ERR_DEPTH: return "tree depth limit reached";
    case TC_ERR_UNSUPPORTED: return "unsupported option";
    case TC_ERR_TIMEOUT: return "device-side wait timed out";
  }
  return "unknown status";
}

const char* tc_last_error_string(tc_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

tc_status tc_create(const tc_params* prm, tc_ctx** out) {
  if (!prm || !out) return TC_ERR_ARG;
  *out = nullptr;
  if (prm->p < 1 || prm->p > TC_PMAX || !tc_order_supported(prm->p)) return TC_ERR_UNSUPPORTED;
  if (prm->ncrit < 1 || !(prm->theta > 0.0) || (prm->variant != TC_VARIANT_TOP && prm->variant != TC_VARIANT_JERKS))
    return TC_ERR_ARG;
  if (prm->precision != TC_PREC_FP64 && prm->precision != TC_PREC_MIXED && prm->precision != TC_PREC_MIXED_M2L)
    return TC_ERR_ARG;
  if (!(prm->softening >= 0.0) || !std::isfinite(prm->softening)) return TC_ERR_ARG;
  tc_ctx* ctx = new tc_ctx();
  ctx->prm = *prm;
  memset(&ctx->stats, 0, sizeof(ctx->stats));
  cudaError_t e = cudaSetDevice(prm->device);
  if (e == cudaSuccess) e = init_constants(prm->device);
  if (e == cudaSuccess) e = cudaMalloc((void**)&ctx->d_root, sizeof(TcRootInfo));
  if (e == cudaSuccess) e = cudaMalloc((void**)&ctx->d_lv, sizeof(TcLevels));
  if (e == cudaSuccess) e = cudaMalloc((void**)&ctx->d_cnt, sizeof(TcTravCounters));
  if (e == cudaSuccess) e = cudaMalloc((void**)&ctx->d_err, sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMalloc((void**)&ctx->d_small, 16 * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMalloc((void**)&ctx->d_hist, 32 * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, ctx->prm.device);
  if (e == cudaSuccess) {
    for (int i = 0; i < 8 && e == cudaSuccess; i++) e = cudaEventCreate(&ctx->ev[i]);
    ctx->events = e == cudaSuccess;
  }
  if (e != cudaSuccess) {
    tc_destroy(ctx);
    return TC_ERR_CUDA;
  }
  set_attrs(prm->p);
  *out = ctx;
  return TC_OK;
}

static void graph_drop(tc_ctx* ctx);

tc_status tc_destroy(tc_ctx* ctx) {
  if (!ctx) return TC_ERR_ARG;
  cudaSetDevice(ctx->prm.device);
  ctx->in_d.release(); ctx->in_f.release(); ctx->out_d.release();
  ctx->keys.release(); ctx->keys_alt.release(); ctx->vals.release(); ctx->vals_alt.release(); ctx->hist.release();
  ctx->bod.release(); ctx->bflags.release(); ctx->perm.release(); ctx->outs.release();
  ctx->cint.release(); ctx->cdbl.release(); ctx->csink.release(); ctx->split_off.release(); ctx->expn.release();
  ctx->front[0].release(); ctx->front[1].release();
  ctx->m2l.release(); ctx->m2l_alt.release(); ctx->p2p.release(); ctx->p2p_alt.release();
  ctx->m2l_start.release(); ctx->m2l_src.release(); ctx->p2p_start.release(); ctx->p2p_src.release();
  ctx->m2l_tl.release(); ctx->p2p_tl.release(); ctx->leaves.release(); ctx->bpart.release();
  ctx->cell_pn.release(); ctx->cls_start.release(); ctx->cls_tl.release(); ctx->mlp_w.release();
  ctx->judge_idx.release(); ctx->judge_out.release();
  ctx->ds_bod.release(); ctx->ds_out.release(); ctx->ds_flags.release(); ctx->ds_idx.release(); ctx->ds_tgt.release();
  ctx->tsum.release(); ctx->diag.release(); ctx->p2p_part.release();
  ctx->ev_d.release(); ctx->ev_u.release(); ctx->ev_i.release(); ctx->ev_f.release();
  ctx->amag.release(); ctx->body_scale.release(); ctx->cell_scale.release(); ctx->m2l_src2.release();
  ctx->m2l_off.release(); ctx->cls_rng.release(); ctx->cell_feat.release(); ctx->kd_scratch.release(); ctx->kd_index.release(); ctx->kd_flags.release();
  ctx->low_f.release();
  if (ctx->d_root) cudaFree(ctx->d_root);
  if (ctx->d_lv) cudaFree(ctx->d_lv);
  if (ctx->d_cnt) cudaFree(ctx->d_cnt);
  if (ctx->d_err) cudaFree(ctx->d_err);
  if (ctx->d_small) cudaFree(ctx->d_small);
  if (ctx->d_hist) cudaFree(ctx->d_hist);
  if (ctx->events)
    for (int i = 0; i < 8; i++) cudaEventDestroy(ctx->ev[i]);
  graph_drop(ctx);
  if (ctx->gstream) cudaStreamDestroy(ctx->gstream);
  if (ctx->hstat) cudaFreeHost(ctx->hstat);
  if (ctx->hjudge) cudaFreeHost(ctx->hjudge);
  delete ctx;
  return TC_OK;
}

tc_status tc_set_stream(tc_ctx* ctx, void* stream) {
  if (!ctx) return TC_ERR_ARG;
  ctx->stream = (cudaStream_t)stream;
  return TC_OK;
}

// statistics of the last evaluation and its status from the error bits
static tc_status finish_stats(tc_ctx* ctx, int n, unsigned herr) {
  tc_stats& S = ctx->stats;
  S.n_bodies = n;
  S.n_cells = ctx->ncell;
  S.n_leaves = ctx->nleaf;
  S.n_m2l = (long long)ctx->n_m2l;
  S.n_p2p = (long long)ctx->n_p2p;
  S.max_level = ctx->max_level;
  S.n_p2p_inter = ctx->direct ? (long long)n * n : (long long)ctx->n_inter;
  S.n_launches = ctx->launches;
  S.flags = herr | ctx->tree_flags;
  S.n_classes = ctx->n_classes;
  for (int i = 0; i < 16; i++) {
    S.class_order[i] = i < ctx->n_classes ? ctx->class_order[i] : 0;
    S.class_pairs[i] = i < ctx->n_classes ? ctx->class_pairs[i] : 0;
  }
  S.m2l_flop_fraction = ctx->flop_frac;
  S.judge_rms = ctx->judge_rms;
  S.judge_redo = ctx->judge_redo;
  if (ctx->events) {
    float t[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    bool ok = true;
    for (int i = 1; i < 8; i++) ok = ok && cudaEventElapsedTime(&t[i], ctx->ev[i - 1], ctx->ev[i]) == cudaSuccess;
    ok = ok && cudaEventElapsedTime(&t[0], ctx->ev[0], ctx->ev[7]) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      for (int i = 0; i < 8; i++) t[i] = 0.f;
    }
    S.ms_total = t[0]; S.ms_tree = t[1]; S.ms_upward = t[2]; S.ms_traverse = t[3]; S.ms_m2l = t[4];
    S.ms_downward = t[5]; S.ms_p2p = t[6];  // the downward pass runs before the near field
  }
  if (herr & TC_EBIT_TIMEOUT) {
    ctx->err = "a device-side wait of the tensor-core far field gave up";
    return TC_ERR_TIMEOUT;
  }
  if ((herr | ctx->tree_flags) & TC_EBIT_NAN) return TC_ERR_NAN_INPUT;
  if ((herr | ctx->tree_flags) & TC_EBIT_DEPTH) return TC_ERR_DEPTH;
  return TC_OK;
}


static tc_status evaluate_impl(tc_ctx* ctx, int n, const double* x, const double* y, const double* z,
                               const double* vx, const double* vy, const double* vz, const double* m,
                               const unsigned char* flags, double* ax, double* ay, double* az, double* pot,
                               double* jx, double* jy, double* jz, int mem, double* timestep);

static tc_status evaluate_graph(tc_ctx* ctx, int n, const double* x, const double* y, const double* z,
                                const double* vx, const double* vy, const double* vz, const double* m,
                                const unsigned char* flags, double* ax, double* ay, double* az, double* pot,
                                double* jx, double* jy, double* jz, int mem, double step_dt = 0.0);

tc_status tc_evaluate(tc_ctx* ctx, int n, const double* x, const double* y, const double* z, const double* vx,
                      const double* vy, const double* vz, const double* m, const unsigned char* flags, double* ax,
                      double* ay, double* az, double* pot, double* jx, double* jy, double* jz, int mem) {
  if (!ctx) return TC_ERR_ARG;
  ctx->steps = false;
  if (ctx->graph_on) return evaluate_graph(ctx, n, x, y, z, vx, vy, vz, m, flags, ax, ay, az, pot, jx, jy, jz, mem);
  return evaluate_impl(ctx, n, x, y, z, vx, vy, vz, m, flags, ax, ay, az, pot, jx, jy, jz, mem, nullptr);
}

tc_status tc_evaluate_steps(tc_ctx* ctx, int n, const double* x, const double* y, const double* z, const double* vx,
                            const double* vy, const double* vz, const double* m, const unsigned char* flags,
                            double dt_param, double* ax, double* ay, double* az, double* pot, double* timestep,
                            int mem) {
  if (!ctx || !vx || !vy || !vz || !timestep) return TC_ERR_ARG;
  if (ctx->prm.variant != TC_VARIANT_TOP) return TC_ERR_UNSUPPORTED;
  ctx->steps = true;
  ctx->dt_param = dt_param;
  tc_status r = evaluate_impl(ctx, n, x, y, z, vx, vy, vz, m, flags, ax, ay, az, pot, nullptr, nullptr, nullptr, mem,
                              timestep);
  ctx->steps = false;
  return r;
}

static tc_status evaluate_impl(tc_ctx* ctx, int n, const double* x, const double* y, const double* z,
                               const double* vx, const double* vy, const double* vz, const double* m,
                               const unsigned char* flags, double* ax, double* ay, double* az, double* pot,
                               double* jx, double* jy, double* jz, int mem, double* timestep) {
  if (!ctx || n <= 0 || !x || !y || !z || !m || !ax || !ay || !az || !pot) return TC_ERR_ARG;
  const bool jerk = ctx->prm.variant == TC_VARIANT_JERKS;
  if (jerk && (!vx || !vy || !vz)) return TC_ERR_ARG;
  if (mem != TC_MEM_HOST && mem != TC_MEM_DEVICE) return TC_ERR_ARG;
  TC_CK(cudaSetDevice(ctx->prm.device));
  cudaGetLastError();  // an error left by an earlier, unrelated call is not this evaluation's
  cudaStream_t st = ctx->stream;
  ctx->n = n;
  ctx->launches = 0;
  ctx->tree_flags = 0;
  size_t N = (size_t)n;
  if (ctx->events) cudaEventRecord(ctx->ev[0], st);
  // ---- inputs on the device
  const double *dx = x, *dy = y, *dz = z, *dm = m, *dvx = vx, *dvy = vy, *dvz = vz;
  const uint8_t* df = flags;
  if (mem == TC_MEM_HOST) {
    TC_CK(ctx->in_d.ensure(7 * N));
    double* s = ctx->in_d.p;
    const double* src[7] = {x, y, z, m, vx, vy, vz};
    for (int a = 0; a < 7; a++) {
      if (!src[a]) continue;
      TC_CK(cudaMemcpyAsync(s + a * N, src[a], N * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    dx = s; dy = s + N; dz = s + 2 * N; dm = s + 3 * N;
    dvx = vx ? s + 4 * N : nullptr; dvy = vy ? s + 5 * N : nullptr; dvz = vz ? s + 6 * N : nullptr;
    if (flags) {
      TC_CK(ctx->in_f.ensure(N));
      TC_CK(cudaMemcpyAsync(ctx->in_f.p, flags, N, cudaMemcpyHostToDevice, st));
      df = ctx->in_f.p;
    }
  }
  // ---- buffers sized by N
  TC_CK(ctx->keys.ensure(N)); TC_CK(ctx->keys_alt.ensure(N));
  TC_CK(ctx->vals.ensure(N)); TC_CK(ctx->vals_alt.ensure(N));
  TC_CK(ctx->bod.ensure(ctx->prm.precision != TC_PREC_FP64 ? 13 * N + 2 : 7 * N));
  TC_CK(ctx->bflags.ensure(N)); TC_CK(ctx->perm.ensure(N));
  TC_CK(ctx->outs.ensure(7 * N));
  TC_CK(ctx->hist.ensure(257 * ((N + kRsTile - 1) / kRsTile + 1) + 1024));
  TC_CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(unsigned), st));
  int direct_below = ctx->prm.direct_below;
  if (direct_below < 0) direct_below = jerk ? 8000 : ctx->prm.ncrit;
  ctx->direct = n < direct_below && !ctx->steps;  // the time-step pass always builds the tree
  TcBodies b = bodies_view(ctx, n, jerk);
  TcOut o = out_view(ctx, n, jerk);
  tc_status rs = TC_OK;
  if (ctx->direct) {
    k_nan_check<<<nblocks(n, 256), 256, 0, st>>>(n, dx, dy, dz, dm, ctx->d_err);
    k_identity<<<nblocks(n, 256), 256, 0, st>>>(n, ctx->vals.p);
    k_gather_bodies<<<nblocks(n, 256), 256, 0, st>>>(n, ctx->vals.p, dx, dy, dz, dm, dvx, dvy, dvz, df, b);
    if (jerk)
      k_direct<true><<<nblocks(n, 128), 128, 0, st>>>(n, b, o);
    else
      k_direct<false><<<nblocks(n, 128), 128, 0, st>>>(n, b, o);
    ctx->launches += 4;
    ctx->ncell = 0; ctx->nleaf = 0; ctx->n_m2l = 0; ctx->n_p2p = 0; ctx->max_level = 0;
    if (ctx->events)
      for (int i = 1; i <= 6; i++) cudaEventRecord(ctx->ev[i], st);
  } else {
    size_t grow_c = 0;  // cell capacity asked for by a retry after a cell overflow
    for (int attempt = 0; attempt < 4; attempt++) {
      // cells for this n (kept at least as large as what the context already holds), or what a
      // retry asks for; the buffers are grown whenever the capacity grows
      size_t want_c = (size_t)(2 * N / (size_t)(ctx->prm.ncrit > 8 ? 8 : ctx->prm.ncrit) + 1024);
      if (want_c > 2 * N + 1024) want_c = 2 * N + 1024;
      if (want_c < ctx->ccap) want_c = ctx->ccap;
      if (want_c < grow_c) want_c = grow_c;
      if (ctx->ccap < want_c || !ctx->cint.p) {
        TC_CK(ctx->cint.ensure(6 * want_c));
        TC_CK(ctx->cdbl.ensure(7 * want_c));
        TC_CK(ctx->csink.ensure(want_c));
        TC_CK(ctx->split_off.ensure(8 * want_c));
        ctx->ccap = want_c;
      }
      int nb = 148 * 4;
      TC_CK(ctx->bpart.ensure(6 * nb));
      k_bounds_partial<<<nb, 256, 0, st>>>(n, dx, dy, dz, dm, ctx->bpart.p, ctx->d_err);
      k_bounds_final<<<1, 1, 0, st>>>(nb, ctx->bpart.p, ctx->d_root, ctx->prm.use_shift, ctx->prm.shift_u[0],
                                      ctx->prm.shift_u[1], ctx->prm.shift_u[2]);
      k_morton<<<nblocks(n, 256), 256, 0, st>>>(n, dx, dy, dz, ctx->d_root, ctx->keys.p, ctx->vals.p);
      ctx->launches += 4 + radix_sort(ctx->keys.p, ctx->vals.p, ctx->keys_alt.p, ctx->vals_alt.p, n, 63, ctx->hist.p, st);
      k_gather_bodies<<<nblocks(n, 256), 256, 0, st>>>(n, ctx->vals.p, dx, dy, dz, dm, dvx, dvy, dvz, df, b);
      run_fn f = pick(ctx->prm.p, jerk);
      if (!f) return TC_ERR_UNSUPPORTED;
      rs = f(ctx, n);
      if (rs == TC_ERR_CAPACITY && ctx->ncell == 0) {
        grow_c = 2 * ctx->ccap + 1024;
        continue;
      }
      break;
    }
    if (rs != TC_OK) return rs;
  }
  // ---- judge: FP64 direct sums at seeded bodies; a rejected selector step is redone at fixed p
  ctx->judge_rms = 0.0;
  ctx->judge_redo = 0;
  if (ctx->prm.judge_n > 0 && !ctx->steps) {
    int nt = std::min(ctx->prm.judge_n, n);
    double rms = 0.0;
    tc_status js = judge(ctx, n, nt, jerk, &rms);
    if (js != TC_OK) return js;
    ctx->judge_rms = rms;
    if (!ctx->direct && ctx->prm.selector > 0 && ctx->prm.judge_tol > 0 && rms > ctx->prm.judge_tol) {
      int sel = ctx->prm.selector;
      ctx->prm.selector = 0;
      run_fn f = pick(ctx->prm.p, jerk);
      rs = f(ctx, n);
      ctx->prm.selector = sel;
      if (rs != TC_OK) return rs;
      js = judge(ctx, n, nt, jerk, &rms);
      if (js != TC_OK) return js;
      ctx->judge_rms = rms;
      ctx->judge_redo = 1;
    }
  }
  // ---- outputs to the caller's order
  double *opot = pot, *oax = ax, *oay = ay, *oaz = az, *ojx = jx, *ojy = jy, *ojz = jz;
  double* ots = timestep;
  if (mem == TC_MEM_HOST) {
    TC_CK(ctx->out_d.ensure(8 * N));
    double* s = ctx->out_d.p;
    opot = s; oax = s + N; oay = s + 2 * N; oaz = s + 3 * N;
    ojx = jx ? s + 4 * N : nullptr; ojy = jx ? s + 5 * N : nullptr; ojz = jx ? s + 6 * N : nullptr;
    ots = s + 7 * N;
  }
  k_scatter_out<<<nblocks(n, 256), 256, 0, st>>>(n, ctx->perm.p, o, opot, oax, oay, oaz, ojx, ojy, ojz);
  ctx->launches++;
  const bool keep_amag = ctx->prm.selector > 0 && !timestep && !ctx->direct;
  if (keep_amag) {  // the next evaluation's per-target error budget
    TC_CK(ctx->amag.ensure(N));
    k_amag<<<nblocks(n, 256), 256, 0, st>>>(n, oax, oay, oaz, ctx->amag.p);
    ctx->launches++;
  }
  if (timestep) {
    k_scatter_one<<<nblocks(n, 256), 256, 0, st>>>(n, ctx->perm.p, ctx->tsum.p, ots);
    ctx->launches++;
  }
  if (ctx->events) cudaEventRecord(ctx->ev[7], st);
  unsigned herr = 0;
  TC_CK(cudaMemcpyAsync(&herr, ctx->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  if (mem == TC_MEM_HOST) {
    double* s = ctx->out_d.p;
    double* dst[7] = {pot, ax, ay, az, jx, jy, jz};
    for (int a = 0; a < 7; a++) {
      if (!dst[a] || (a >= 4 && !jx)) continue;
      TC_CK(cudaMemcpyAsync(dst[a], s + a * N, N * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    if (timestep) TC_CK(cudaMemcpyAsync(timestep, s + 7 * N, N * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  TC_CK(cudaStreamSynchronize(st));
  TC_CK(cudaGetLastError());
  ctx->amag_n = keep_amag ? n : -1;
  return finish_stats(ctx, n, herr);
}

// ---------------------------------------------------------------------------------------
// The evaluation as one CUDA graph (tc_set_graph).  A call that cannot replay (first call,
// other pointers, sizes or parameters, or a capacity overflow reported by the last replay)
// runs the normal path, whose results it returns, and then plans and captures: capacities
// with headroom over that evaluation, every buffer allocated, the judge's targets uploaded,
// and the whole device-sized sequence (inputs, tree, FMM, judge kernels, outputs and a status
// block) recorded into a graph on a private stream.  A matching call replays the graph and
// reads the status block: an overflow bit re-runs the call on the normal path (and re-plans).
// ---------------------------------------------------------------------------------------
static void graph_drop(tc_ctx* ctx) {
  if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
  if (ctx->graph) cudaGraphDestroy(ctx->graph);
  ctx->gexec = nullptr;
  ctx->graph = nullptr;
  ctx->gvalid = false;
}

// Every device buffer and capacity a captured graph has baked into its launches.  Any other
// call on the context (tc_evaluate_steps, tc_direct_sums, tc_train_selector, an evaluation of
// another n) may grow, and so free and reallocate, one of them; a replay is only valid while
// the signature is unchanged.
static void graph_signature(const tc_ctx* c, std::vector<const void*>& s) {
  s.clear();
  const void* bufs[] = {c->in_d.p,     c->in_f.p,      c->out_d.p,     c->keys.p,      c->keys_alt.p,
                        c->vals.p,     c->vals_alt.p,  c->hist.p,      c->bod.p,       c->bflags.p,
                        c->perm.p,     c->outs.p,      c->cint.p,      c->cdbl.p,      c->csink.p,
                        c->split_off.p, c->expn.p,     c->front[0].p,  c->front[1].p,  c->m2l.p,
                        c->m2l_alt.p,  c->p2p.p,       c->p2p_alt.p,   c->m2l_start.p, c->m2l_src.p,
                        c->p2p_start.p, c->p2p_src.p,  c->m2l_tl.p,    c->p2p_tl.p,    c->leaves.p,
                        c->judge_idx.p, c->judge_out.p, c->p2p_part.p, c->bpart.p,     c->tc_bins.p,
                        c->amag.p,      c->body_scale.p, c->cell_scale.p, c->m2l_src2.p, c->m2l_off.p,
                        c->cell_pn.p,   c->mlp_w.p,      c->cls_rng.p,    c->cell_feat.p};
  s.assign(bufs, bufs + sizeof(bufs) / sizeof(bufs[0]));
  const size_t caps[] = {c->ccap, c->mcap, c->pcap, c->fcap, c->expn.n, c->p2p_part.n};
  for (size_t v : caps) s.push_back((const void*)(uintptr_t)v);
}

constexpr unsigned kGraphCapBits = TC_EBIT_CELL_CAP | TC_EBIT_M2L_CAP | TC_EBIT_P2P_CAP | TC_EBIT_FRONTIER_CAP;

static bool graph_key_equal(const TcGraphKey& a, const TcGraphKey& b) {
  if (a.n != b.n || a.mem != b.mem || a.step_dt != b.step_dt) return false;
  for (int i = 0; i < 15; i++)
    if (a.ptr[i] != b.ptr[i]) return false;
  return memcmp(&a.prm, &b.prm, sizeof(tc_params)) == 0;
}

static bool host_pinned(const void* p) {
  if (!p) return true;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// the captured sequence; ctx->stream is the capture stream
static void graph_issue(tc_ctx* ctx, int n, const double* const* in, const unsigned char* flags, double* const* outp,
                        int mem, bool jerk, graph_fn f) {
  cudaStream_t st = ctx->stream;
  const size_t N = (size_t)n;
  long long L = 0;
  graph_event(ctx, 0, st);
  const double *dx = in[0], *dy = in[1], *dz = in[2], *dm = in[3], *dvx = in[4], *dvy = in[5], *dvz = in[6];
  const uint8_t* df = flags;
  if (mem == TC_MEM_HOST) {
    double* s = ctx->in_d.p;
    for (int a = 0; a < 7; a++)
      if (in[a]) cudaMemcpyAsync(s + a * N, in[a], N * sizeof(double), cudaMemcpyHostToDevice, st);
    dx = s; dy = s + N; dz = s + 2 * N; dm = s + 3 * N;
    dvx = in[4] ? s + 4 * N : nullptr; dvy = in[5] ? s + 5 * N : nullptr; dvz = in[6] ? s + 6 * N : nullptr;
    if (flags) {
      cudaMemcpyAsync(ctx->in_f.p, flags, N, cudaMemcpyHostToDevice, st);
      df = ctx->in_f.p;
    }
  }
  const double sdt = ctx->gstep_dt;
  if (sdt != 0.0) {  // leapfrog step: kick by the previous accelerations and drift, in place
    k_kick_drift<<<nblocks(n, 256), 256, 0, st>>>(n, (double*)in[0], (double*)in[1], (double*)in[2], (double*)in[4],
                                                  (double*)in[5], (double*)in[6], outp[0], outp[1], outp[2],
                                                  0.5 * sdt, sdt);
    L++;
  }
  cudaMemsetAsync(ctx->d_err, 0, sizeof(unsigned), st);
  TcBodies b = bodies_view(ctx, n, jerk);
  const int nb = 148 * 4;
  k_bounds_partial<<<nb, 256, 0, st>>>(n, dx, dy, dz, dm, ctx->bpart.p, ctx->d_err);
  k_bounds_final<<<1, 1, 0, st>>>(nb, ctx->bpart.p, ctx->d_root, ctx->prm.use_shift, ctx->prm.shift_u[0],
                                  ctx->prm.shift_u[1], ctx->prm.shift_u[2]);
  k_morton<<<nblocks(n, 256), 256, 0, st>>>(n, dx, dy, dz, ctx->d_root, ctx->keys.p, ctx->vals.p);
  L += 4 + radix_sort(ctx->keys.p, ctx->vals.p, ctx->keys_alt.p, ctx->vals_alt.p, n, 63, ctx->hist.p, st);
  k_gather_bodies<<<nblocks(n, 256), 256, 0, st>>>(n, ctx->vals.p, dx, dy, dz, dm, dvx, dvy, dvz, df, b);
  graph_check(ctx, "inputs and Morton sort");
  f(ctx, n);
  graph_check(ctx, "FMM");
  TcOut o = out_view(ctx, n, jerk);
  const int nt = ctx->gjudge_nt;
  if (nt > 0) {
    const int nchunk = std::max(1, std::min(4 * ctx->nsm, n / 1024));
    double* part = ctx->judge_out.p + 7 * (size_t)nt;
    k_direct_targets<false><<<dim3(nchunk, (nt + kJudgeTile - 1) / kJudgeTile), kJudgeTile, 0, st>>>(
        n, nt, nchunk, ctx->judge_idx.p, b, part);
    k_direct_targets_sum<<<nblocks(nt, 128), 128, 0, st>>>(nt, nchunk, ctx->judge_idx.p, part, o, ctx->judge_out.p);
    cudaMemcpyAsync(ctx->hjudge, ctx->judge_out.p, 7 * (size_t)nt * sizeof(double), cudaMemcpyDeviceToHost, st);
    L += 2;
  }
  double *opot = outp[3], *oax = outp[0], *oay = outp[1], *oaz = outp[2], *ojx = outp[4], *ojy = outp[5],
         *ojz = outp[6];
  if (mem == TC_MEM_HOST) {
    double* s = ctx->out_d.p;
    opot = s; oax = s + N; oay = s + 2 * N; oaz = s + 3 * N;
    ojx = outp[4] ? s + 4 * N : nullptr; ojy = outp[4] ? s + 5 * N : nullptr; ojz = outp[4] ? s + 6 * N : nullptr;
  }
  k_scatter_out<<<nblocks(n, 256), 256, 0, st>>>(n, ctx->perm.p, o, opot, oax, oay, oaz, ojx, ojy, ojz);
  L += 1;
  if (ctx->prm.selector > 0) {  // the next replay's per-target error budget
    k_amag<<<nblocks(n, 256), 256, 0, st>>>(n, oax, oay, oaz, ctx->amag.p);
    L++;
  }
  if (sdt != 0.0) {  // closing kick by the new accelerations (not after a capacity overflow)
    k_kick_guarded<<<nblocks(n, 256), 256, 0, st>>>(n, (double*)in[4], (double*)in[5], (double*)in[6], outp[0],
                                                    outp[1], outp[2], 0.5 * sdt, ctx->d_err, kGraphCapBits);
    L++;
  }
  graph_event(ctx, 7, st);
  if (mem == TC_MEM_HOST) {
    double* s = ctx->out_d.p;
    double* dst[7] = {outp[3], outp[0], outp[1], outp[2], outp[4], outp[5], outp[6]};
    for (int a = 0; a < 7; a++)
      if (dst[a] && (a < 4 || outp[4])) cudaMemcpyAsync(dst[a], s + a * N, N * sizeof(double), cudaMemcpyDeviceToHost, st);
  }
  TcGraphStatus* h = ctx->hstat;
  cudaMemcpyAsync(&h->err, ctx->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(h->small, ctx->d_small, 4 * sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  if (ctx->gselect) cudaMemcpyAsync(h->hist, ctx->d_hist, 32 * sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&h->lv, ctx->d_lv, sizeof(TcLevels), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&h->cnt, ctx->d_cnt, sizeof(TcTravCounters), cudaMemcpyDeviceToHost, st);
  graph_check(ctx, "judge, outputs and status");
  ctx->glaunches += L;
}

// after a successful normal evaluation of the same call: plan capacities and capture
static void graph_plan(tc_ctx* ctx, int n, const TcGraphKey& key, const double* const* in, const unsigned char* flags,
                       double* const* outp, int mem, bool jerk) {
  graph_drop(ctx);
  if (ctx->direct || ctx->prm.precision == TC_PREC_MIXED_M2L || ctx->emac) return;
  if (ctx->prm.selector == 2 && !ctx->mlp_ready) return;
  graph_fn f = pick_graph(ctx->prm.p, jerk);
  if (!f) return;
  if (mem == TC_MEM_HOST) {
    for (int a = 0; a < 7; a++)
      if (!host_pinned(in[a]) || !host_pinned(outp[a])) return;  // pageable memory cannot be captured
    if (!host_pinned(flags)) return;
  }
  const int NT = TC_NTERM(ctx->prm.p);
  const size_t N = (size_t)n;
  // capacities: 25 % over this evaluation
  size_t ccap = std::max(ctx->ccap, (size_t)(ctx->ncell * 1.25) + 1024);
  if (ccap > 2 * N + 1024) ccap = std::max(ctx->ccap, 2 * N + 1024);
  if (ctx->cint.ensure(6 * ccap) || ctx->cdbl.ensure(7 * ccap) || ctx->csink.ensure(ccap) ||
      ctx->split_off.ensure(8 * ccap))
    return;
  ctx->ccap = ccap;
  size_t mcap = std::max(ctx->mcap, (size_t)(ctx->n_m2l * 1.25) + 4096);
  size_t pcap = std::max(ctx->pcap, (size_t)(ctx->n_p2p * 1.25) + 4096);
  size_t fcap = (size_t)(ctx->fcap * 1.25) + 4096;
  if (ctx->m2l.ensure(mcap) || ctx->p2p.ensure(pcap) || ctx->front[0].ensure(fcap) || ctx->front[1].ensure(fcap)) return;
  ctx->mcap = ctx->m2l.n;
  ctx->pcap = ctx->p2p.n;
  ctx->fcap = std::min(ctx->front[0].n, ctx->front[1].n);
  size_t mx = std::max(std::max(ctx->mcap, ctx->pcap), N);
  if (ctx->m2l_alt.ensure(ctx->mcap + 1) || ctx->p2p_alt.ensure(ctx->pcap + 1) ||
      ctx->hist.ensure(257 * ((mx + kRsTile - 1) / kRsTile + 1) + 1024) || ctx->m2l_start.ensure(ccap + 1) ||
      ctx->p2p_start.ensure(ccap + 1) || ctx->m2l_src.ensure(ctx->mcap + 1) || ctx->p2p_src.ensure(ctx->pcap + 1) ||
      ctx->m2l_tl.ensure(ccap) || ctx->p2p_tl.ensure(ccap) || ctx->leaves.ensure(ccap) ||
      ctx->expn.ensure(ccap * NT * (jerk ? 4 : 2)) || ctx->bpart.ensure(6 * 148 * 4) ||
      (p2p_nsplit(n) > 1 && ctx->p2p_part.ensure((size_t)p2p_nsplit(n) * (jerk ? 7 : 4) * N)))
    return;
  if (ctx->prm.selector > 0 &&
      (ctx->cell_pn.ensure(ccap * (ctx->prm.p + 1)) || ctx->cell_scale.ensure(ccap) || ctx->body_scale.ensure(N) ||
       ctx->amag.ensure(N) || ctx->m2l_src2.ensure(ctx->m2l_src.n) || ctx->m2l_off.ensure(ctx->m2l_src.n) ||
       ctx->cls_rng.ensure((size_t)2 * TC_MAX_CLASSES * ccap) || ctx->cell_feat.ensure(ccap * 5)))
    return;
  // orders are selected in the graph once an evaluation of these bodies left its |a| behind
  ctx->gselect = ctx->prm.selector > 0 && ctx->amag_n == n;
  int sb = 1;
  while (((size_t)1 << sb) < ccap) sb++;
  ctx->gsbits = sb;
  // judge targets (the same seeded bodies as the normal path's judge)
  ctx->gjudge_nt = 0;
  if (ctx->prm.judge_n > 0) {
    const int nt = std::min(ctx->prm.judge_n, n);
    std::vector<int> idx(nt);
    std::mt19937_64 rng(ctx->prm.judge_seed);
    std::uniform_int_distribution<int> U(0, n - 1);
    for (int k = 0; k < nt; k++) idx[k] = U(rng);
    const int nchunk = std::max(1, std::min(4 * ctx->nsm, n / 1024));
    if (ctx->judge_idx.ensure(nt) || ctx->judge_out.ensure(7 * (size_t)nt + 8 * (size_t)nt * nchunk)) return;
    if (cudaMemcpy(ctx->judge_idx.p, idx.data(), nt * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) return;
    if (ctx->hjudge_cap < 7 * (size_t)nt) {
      if (ctx->hjudge) cudaFreeHost(ctx->hjudge);
      ctx->hjudge = nullptr;
      ctx->hjudge_cap = 0;
      if (cudaMallocHost((void**)&ctx->hjudge, 7 * (size_t)nt * sizeof(double)) != cudaSuccess) return;
      ctx->hjudge_cap = 7 * (size_t)nt;
    }
    ctx->gjudge_nt = nt;
  }
  if (!ctx->hstat && cudaMallocHost((void**)&ctx->hstat, sizeof(TcGraphStatus)) != cudaSuccess) {
    ctx->hstat = nullptr;
    return;
  }
  if (!ctx->gstream && cudaStreamCreateWithFlags(&ctx->gstream, cudaStreamNonBlocking) != cudaSuccess) {
    ctx->gstream = nullptr;
    return;
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return;
  // capture
  cudaStream_t saved = ctx->stream;
  const size_t saved_stride = ctx->expn_stride;
  ctx->stream = ctx->gstream;
  ctx->expn_stride = ccap;
  ctx->glaunches = 0;
  ctx->gfail.clear();
  cudaGraph_t g = nullptr;
  cudaGetLastError();
  cudaError_t e = cudaStreamBeginCapture(ctx->gstream, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    graph_issue(ctx, n, in, flags, outp, mem, jerk, f);
    e = cudaStreamEndCapture(ctx->gstream, &g);
  } else {
    ctx->gfail = std::string("begin capture: ") + cudaGetErrorString(e);
  }
  ctx->stream = saved;
  ctx->expn_stride = saved_stride;
  if (e != cudaSuccess || !g || !ctx->gfail.empty()) {
    if (ctx->gfail.empty()) ctx->gfail = std::string("end capture: ") + cudaGetErrorString(e);
    cudaGetLastError();
    if (g) cudaGraphDestroy(g);
    return;
  }
  if (cudaGraphInstantiate(&ctx->gexec, g, 0) != cudaSuccess) {
    cudaGetLastError();
    cudaGraphDestroy(g);
    ctx->gexec = nullptr;
    return;
  }
  ctx->graph = g;
  ctx->gkey = key;
  graph_signature(ctx, ctx->gsig);
  ctx->gvalid = true;
  graph_check(ctx, "instantiate");
  if (!ctx->gfail.empty()) graph_drop(ctx);
}

static tc_status evaluate_graph(tc_ctx* ctx, int n, const double* x, const double* y, const double* z,
                                const double* vx, const double* vy, const double* vz, const double* m,
                                const unsigned char* flags, double* ax, double* ay, double* az, double* pot,
                                double* jx, double* jy, double* jz, int mem, double step_dt) {
  TcGraphKey key;
  key.n = n;
  key.mem = mem;
  key.step_dt = step_dt;
  const void* ptrs[15] = {x, y, z, vx, vy, vz, m, flags, ax, ay, az, pot, jx, jy, jz};
  for (int i = 0; i < 15; i++) key.ptr[i] = ptrs[i];
  key.prm = ctx->prm;
  const bool jerk = ctx->prm.variant == TC_VARIANT_JERKS;
  if (ctx->gvalid) {
    std::vector<const void*> sig;
    graph_signature(ctx, sig);
    if (sig != ctx->gsig) graph_drop(ctx);  // a buffer it launches on was reallocated since the capture
  }
  if (ctx->gvalid && graph_key_equal(key, ctx->gkey)) {
    TC_CK(cudaSetDevice(ctx->prm.device));
    TC_CK(cudaGraphLaunch(ctx->gexec, ctx->stream));
    TC_CK(cudaStreamSynchronize(ctx->stream));
    const TcGraphStatus& h = *ctx->hstat;
    if (!(h.err & kGraphCapBits)) {
      ctx->n = n;
      ctx->direct = 0;
      ctx->ncell = h.lv.ncell;
      ctx->nleaf = (int)h.small[2];
      ctx->n_m2l = h.cnt.n_m2l;
      ctx->n_p2p = h.cnt.n_p2p;
      ctx->n_inter = h.cnt.frontier[0];
      ctx->lv = h.lv;
      int maxl = 0;
      for (int l = 0; l <= TC_MAX_LEVEL; l++)
        if (h.lv.count[l] > 0) maxl = l;
      ctx->max_level = maxl;
      ctx->sbits = ctx->gsbits;
      ctx->expn_stride = ctx->ccap;
      ctx->launches = ctx->glaunches;
      ctx->tree_flags = 0;
      ctx->n_classes = 1;
      ctx->class_order[0] = ctx->prm.p;
      ctx->class_pairs[0] = (long long)ctx->n_m2l;
      ctx->flop_frac = 1.0;
      if (ctx->gselect) order_stats(ctx, ctx->prm.p, h.hist, ctx->gcls_q, ctx->gcls_n);
      if (ctx->prm.selector > 0) ctx->amag_n = n;  // the replay left its |a| for the next one
      ctx->judge_redo = 0;
      ctx->judge_rms = 0.0;
      if (ctx->gjudge_nt > 0) {
        double sacc = 0.0;
        for (int k = 0; k < ctx->gjudge_nt; k++) {
          const double* r = ctx->hjudge + 7 * (size_t)k;
          double ex = r[4] - r[1], ey = r[5] - r[2], ez = r[6] - r[3];
          double an = r[1] * r[1] + r[2] * r[2] + r[3] * r[3];
          sacc += (ex * ex + ey * ey + ez * ez) / (an > 0 ? an : 1.0);
        }
        ctx->judge_rms = sqrt(sacc / ctx->gjudge_nt);
      }
      if (ctx->gselect && step_dt == 0.0 && ctx->prm.judge_tol > 0 && ctx->judge_rms > ctx->prm.judge_tol) {
        // the judge rejected the selected orders: redo this evaluation at the fixed order (a
        // step's kicks are already applied, so a captured step only reports judge_rms)
        const int sel = ctx->prm.selector;
        ctx->prm.selector = 0;
        tc_status rr = evaluate_impl(ctx, n, x, y, z, vx, vy, vz, m, flags, ax, ay, az, pot, jx, jy, jz, mem, nullptr);
        ctx->prm.selector = sel;
        ctx->amag_n = n;
        if (rr == TC_OK) ctx->judge_redo = 1;
        return rr;
      }
      return finish_stats(ctx, n, h.err);
    }
    ctx->gvalid = false;  // a capacity overflowed: re-run on the normal path and re-plan
    if (step_dt != 0.0) {
      // the replay already kicked and drifted (and skipped its closing kick): redo the
      // evaluation and the closing kick only
      tc_status rs = evaluate_impl(ctx, n, x, y, z, vx, vy, vz, m, flags, ax, ay, az, pot, jx, jy, jz, mem, nullptr);
      if (rs != TC_OK) return rs;
      k_kick_drift<<<nblocks(n, 256), 256, 0, ctx->stream>>>(n, (double*)x, (double*)y, (double*)z, (double*)vx,
                                                             (double*)vy, (double*)vz, ax, ay, az, 0.5 * step_dt,
                                                             0.0);
      const double* in[7] = {x, y, z, m, vx, vy, vz};
      double* outp[7] = {ax, ay, az, pot, jx, jy, jz};
      ctx->gstep_dt = step_dt;
      graph_plan(ctx, n, key, in, flags, outp, mem, jerk);
      ctx->gstep_dt = 0.0;
      return TC_OK;
    }
  }
  if (step_dt != 0.0)
    k_kick_drift<<<nblocks(n, 256), 256, 0, ctx->stream>>>(n, (double*)x, (double*)y, (double*)z, (double*)vx,
                                                           (double*)vy, (double*)vz, ax, ay, az, 0.5 * step_dt,
                                                           step_dt);
  tc_status rs = evaluate_impl(ctx, n, x, y, z, vx, vy, vz, m, flags, ax, ay, az, pot, jx, jy, jz, mem, nullptr);
  if (rs == TC_OK && step_dt != 0.0)
    k_kick_drift<<<nblocks(n, 256), 256, 0, ctx->stream>>>(n, (double*)x, (double*)y, (double*)z, (double*)vx,
                                                           (double*)vy, (double*)vz, ax, ay, az, 0.5 * step_dt, 0.0);
  if (rs == TC_OK) {
    const double* in[7] = {x, y, z, m, vx, vy, vz};
    double* outp[7] = {ax, ay, az, pot, jx, jy, jz};
    ctx->gstep_dt = step_dt;
    graph_plan(ctx, n, key, in, flags, outp, mem, jerk);
    ctx->gstep_dt = 0.0;
  }
  return rs;
}

tc_status tc_set_error_mac(tc_ctx* ctx, int on, double force_accuracy) {
  if (!ctx || (on && !(force_accuracy > 0.0))) return TC_ERR_ARG;
  ctx->emac = on != 0;
  ctx->emac_fa = force_accuracy;
  graph_drop(ctx);  // a captured graph used the theta MAC
  return TC_OK;
}

tc_status tc_get_acc_old(tc_ctx* ctx, double* acc_old) {
  if (!ctx || !acc_old) return TC_ERR_ARG;
  if (!ctx->emac || !ctx->acc_old.p || ctx->direct) return TC_ERR_UNSUPPORTED;
  std::vector<double> a(ctx->n);
  std::vector<int> perm(ctx->n);
  TC_CK(cudaMemcpy(a.data(), ctx->acc_old.p, ctx->n * sizeof(double), cudaMemcpyDeviceToHost));
  TC_CK(cudaMemcpy(perm.data(), ctx->perm.p, ctx->n * sizeof(int), cudaMemcpyDeviceToHost));
  for (int i = 0; i < ctx->n; i++) acc_old[perm[i]] = a[i];
  return TC_OK;
}

tc_status tc_set_graph(tc_ctx* ctx, int on) {
  if (!ctx) return TC_ERR_ARG;
  cudaSetDevice(ctx->prm.device);
  ctx->graph_on = on != 0;
  if (!ctx->graph_on) graph_drop(ctx);
  return TC_OK;
}

int tc_graph_ready(const tc_ctx* ctx) { return ctx && ctx->gvalid ? 1 : 0; }

const char* tc_graph_note(const tc_ctx* ctx) { return ctx ? ctx->gfail.c_str() : ""; }

tc_status tc_direct_sums(tc_ctx* ctx, int n, const double* x, const double* y, const double* z, const double* vx,
                         const double* vy, const double* vz, const double* m, const unsigned char* flags, int nt,
                         const int* targets, double* out, int mem) {
  if (!ctx || n <= 0 || nt <= 0 || !x || !y || !z || !m || !targets || !out) return TC_ERR_ARG;
  if (mem != TC_MEM_HOST && mem != TC_MEM_DEVICE) return TC_ERR_ARG;
  const bool jerk = vx && vy && vz;
  for (int k = 0; k < nt; k++)
    if (targets[k] < 0 || targets[k] >= n) return TC_ERR_ARG;
  TC_CK(cudaSetDevice(ctx->prm.device));
  cudaStream_t st = ctx->stream;
  const size_t N = (size_t)n;
  const double *dx = x, *dy = y, *dz = z, *dm = m, *dvx = vx, *dvy = vy, *dvz = vz;
  const uint8_t* df = flags;
  if (mem == TC_MEM_HOST) {
    TC_CK(ctx->in_d.ensure(7 * N));
    double* s = ctx->in_d.p;
    const double* src[7] = {x, y, z, m, vx, vy, vz};
    for (int a = 0; a < 7; a++) {
      if (!src[a]) continue;
      TC_CK(cudaMemcpyAsync(s + a * N, src[a], N * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    dx = s; dy = s + N; dz = s + 2 * N; dm = s + 3 * N;
    dvx = vx ? s + 4 * N : nullptr; dvy = vy ? s + 5 * N : nullptr; dvz = vz ? s + 6 * N : nullptr;
    if (flags) {
      TC_CK(ctx->in_f.ensure(N));
      TC_CK(cudaMemcpyAsync(ctx->in_f.p, flags, N, cudaMemcpyHostToDevice, st));
      df = ctx->in_f.p;
    }
  }
  // bodies in caller order, in buffers of their own (the last evaluation's state is kept)
  TC_CK(ctx->ds_bod.ensure(7 * N));
  TC_CK(ctx->ds_flags.ensure(N));
  TC_CK(ctx->ds_idx.ensure(N));
  TcBodies b;
  double* bb = ctx->ds_bod.p;
  b.x = bb; b.y = bb + N; b.z = bb + 2 * N; b.m = bb + 3 * N;
  b.vx = bb + 4 * N; b.vy = bb + 5 * N; b.vz = bb + 6 * N;
  b.flags = ctx->ds_flags.p;
  b.perm = ctx->ds_idx.p;
  b.eps2 = ctx->prm.softening * ctx->prm.softening;
  k_identity<<<nblocks(n, 256), 256, 0, st>>>(n, ctx->ds_idx.p);
  k_gather_bodies<<<nblocks(n, 256), 256, 0, st>>>(n, ctx->ds_idx.p, dx, dy, dz, dm, dvx, dvy, dvz, df, b);
  const int nchunk = std::max(1, std::min(4 * ctx->nsm, n / 1024));
  TC_CK(ctx->ds_tgt.ensure(nt));
  TC_CK(ctx->ds_out.ensure(7 * (size_t)nt + 8 * (size_t)nt * nchunk));
  TC_CK(cudaMemcpyAsync(ctx->ds_tgt.p, targets, nt * sizeof(int), cudaMemcpyHostToDevice, st));
  double* part = ctx->ds_out.p + 7 * (size_t)nt;
  const dim3 grid(nchunk, (nt + kJudgeTile - 1) / kJudgeTile);
  if (jerk)
    k_direct_targets<true><<<grid, kJudgeTile, 0, st>>>(n, nt, nchunk, ctx->ds_tgt.p, b, part);
  else
    k_direct_targets<false><<<grid, kJudgeTile, 0, st>>>(n, nt, nchunk, ctx->ds_tgt.p, b, part);
  k_direct_targets_out<<<nblocks(nt, 128), 128, 0, st>>>(nt, nchunk, part, ctx->ds_out.p);
  TC_CK(cudaMemcpyAsync(out, ctx->ds_out.p, 7 * (size_t)nt * sizeof(double), cudaMemcpyDeviceToHost, st));
  TC_CK(cudaStreamSynchronize(st));
  TC_CK(cudaGetLastError());
  return TC_OK;
}

tc_status tc_kick_drift(tc_ctx* ctx, int n, double* x, double* y, double* z, double* vx, double* vy, double* vz,
                        const double* ax, const double* ay, const double* az, double dt_kick, double dt_drift) {
  if (!ctx || n <= 0 || !x || !y || !z || !vx || !vy || !vz || !ax || !ay || !az) return TC_ERR_ARG;
  TC_CK(cudaSetDevice(ctx->prm.device));
  k_kick_drift<<<nblocks(n, 256), 256, 0, ctx->stream>>>(n, x, y, z, vx, vy, vz, ax, ay, az, dt_kick, dt_drift);
  TC_CK(cudaGetLastError());
  return TC_OK;
}

tc_status tc_set_wait_limit(tc_ctx* ctx, long long cycles) {
  if (!ctx) return TC_ERR_ARG;
  ctx->wait_limit = cycles > 0 ? cycles : kTcWaitLimit;
  graph_drop(ctx);
  return TC_OK;
}

tc_status tc_step_leapfrog(tc_ctx* ctx, int n, double* x, double* y, double* z, double* vx, double* vy, double* vz,
                           const double* m, double* ax, double* ay, double* az, double* pot, double* jx, double* jy,
                           double* jz, double dt) {
  if (!ctx || n <= 0 || !x || !y || !z || !vx || !vy || !vz || !m || !ax || !ay || !az || !pot ||
      !(dt != 0.0) || !std::isfinite(dt))
    return TC_ERR_ARG;
  TC_CK(cudaSetDevice(ctx->prm.device));
  ctx->steps = false;
  if (ctx->graph_on)
    return evaluate_graph(ctx, n, x, y, z, vx, vy, vz, m, nullptr, ax, ay, az, pot, jx, jy, jz, TC_MEM_DEVICE, dt);
  k_kick_drift<<<nblocks(n, 256), 256, 0, ctx->stream>>>(n, x, y, z, vx, vy, vz, ax, ay, az, 0.5 * dt, dt);
  TC_CK(cudaGetLastError());
  tc_status r = evaluate_impl(ctx, n, x, y, z, vx, vy, vz, m, nullptr, ax, ay, az, pot, jx, jy, jz, TC_MEM_DEVICE,
                              nullptr);
  if (r != TC_OK) return r;
  k_kick_drift<<<nblocks(n, 256), 256, 0, ctx->stream>>>(n, x, y, z, vx, vy, vz, ax, ay, az, 0.5 * dt, 0.0);
  TC_CK(cudaGetLastError());
  return TC_OK;
}

tc_status tc_system_diagnostics(tc_ctx* ctx, int n, const double* m, const double* x, const double* y,
                                const double* z, const double* vx, const double* vy, const double* vz,
                                const double* pot, double* out) {
  if (!ctx || n <= 0 || !m || !x || !y || !z || !vx || !vy || !vz || !pot || !out) return TC_ERR_ARG;
  TC_CK(cudaSetDevice(ctx->prm.device));
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->prm.device);
  const int nblk = std::max(1, std::min(3 * nsm, (n + kDiagThreads - 1) / kDiagThreads));  // one wave: 3 CTAs per SM
  TC_CK(ctx->diag.ensure((size_t)nblk * kDiagQ * 2 + kDiagQ));
  double* res = ctx->diag.p + (size_t)nblk * kDiagQ * 2;
  cudaStream_t st = ctx->stream;
  k_sys_diag_part<<<nblk, kDiagThreads, 0, st>>>(n, m, x, y, z, vx, vy, vz, pot, ctx->diag.p);
  k_sys_diag_final<<<1, kDiagThreads, 0, st>>>(nblk, ctx->diag.p, res);
  TC_CK(cudaGetLastError());
  TC_CK(cudaMemcpyAsync(out, res, kDiagQ * sizeof(double), cudaMemcpyDeviceToHost, st));
  TC_CK(cudaStreamSynchronize(st));
  return TC_OK;
}

tc_status tc_drift_compensated(tc_ctx* ctx, int n, double* x, double* y, double* z, double* ex, double* ey,
                               double* ez, const double* vx, const double* vy, const double* vz, double dt) {
  if (!ctx || n <= 0 || !x || !y || !z || !ex || !ey || !ez || !vx || !vy || !vz) return TC_ERR_ARG;
  TC_CK(cudaSetDevice(ctx->prm.device));
  k_drift_compsum<<<nblocks(n, 256), 256, 0, ctx->stream>>>(n, x, y, z, ex, ey, ez, vx, vy, vz, dt);
  TC_CK(cudaGetLastError());
  return TC_OK;
}

tc_status tc_hermite_predict(tc_ctx* ctx, int n, double* x, double* y, double* z, double* vx, double* vy, double* vz,
                             const double* ax, const double* ay, const double* az, const double* jx,
                             const double* jy, const double* jz, double* save, double dt) {
  if (!ctx || n <= 0 || !x || !y || !z || !vx || !vy || !vz || !ax || !ay || !az || !jx || !jy || !jz || !save)
    return TC_ERR_ARG;
  TC_CK(cudaSetDevice(ctx->prm.device));
  k_hermite_predict<<<nblocks(n, 256), 256, 0, ctx->stream>>>(n, x, y, z, vx, vy, vz, ax, ay, az, jx, jy, jz, save,
                                                              dt);
  TC_CK(cudaGetLastError());
  return TC_OK;
}

tc_status tc_hermite_correct(tc_ctx* ctx, int n, double* x, double* y, double* z, double* vx, double* vy, double* vz,
                             const double* ax, const double* ay, const double* az, const double* jx,
                             const double* jy, const double* jz, const double* save, double dt) {
  if (!ctx || n <= 0 || !x || !y || !z || !vx || !vy || !vz || !ax || !ay || !az || !jx || !jy || !jz || !save)
    return TC_ERR_ARG;
  TC_CK(cudaSetDevice(ctx->prm.device));
  k_hermite_correct<<<nblocks(n, 256), 256, 0, ctx->stream>>>(n, x, y, z, vx, vy, vz, ax, ay, az, jx, jy, jz, save,
                                                              dt);
  TC_CK(cudaGetLastError());
  return TC_OK;
}

double tc_probe_peak(tc_ctx* ctx, int kind) {
  if (!ctx || (kind != 0 && kind != 1)) return -1.0;
  if (cudaSetDevice(ctx->prm.device) != cudaSuccess) return -1.0;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->prm.device);
  void* out = nullptr;
  if (cudaMalloc(&out, 64) != cudaSuccess) return -1.0;
  int blocks = nsm * 8, threads = 256, iters = 4096;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int r = 0; r < 4; r++) {
    cudaEventRecord(e0, ctx->stream);
    if (kind == 0)
      k_fma_probe<double><<<blocks, threads, 0, ctx->stream>>>((double*)out, iters);
    else
      k_fma_probe<float><<<blocks, threads, 0, ctx->stream>>>((float*)out, iters);
    cudaEventRecord(e1, ctx->stream);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0 && ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (cudaGetLastError() != cudaSuccess) return -1.0;
  double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
  return flops / (best * 1e-3) / 1e9;
}

tc_status tc_evaluate_direct_noalloc(int n, const double* x, const double* y, const double* z, const double* vx,
                                     const double* vy, const double* vz, const double* m, const unsigned char* flags,
                                     double* ax, double* ay, double* az, double* pot, double* jx, double* jy,
                                     double* jz, int jerk, void* stream) {
  if (n <= 0 || !x || !y || !z || !m || !ax || !ay || !az || !pot) return TC_ERR_ARG;
  if (jerk && (!vx || !vy || !vz || !jx || !jy || !jz)) return TC_ERR_ARG;
  if (n > TC_NOALLOC_MAX_N) return TC_ERR_CAPACITY;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return TC_ERR_CUDA;
  TcNoallocDev D;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_dev[dev].scratch) {  // once per device: device addresses of the static arrays
      TcNoallocDev f;
      if (cudaGetSymbolAddress((void**)&f.scratch, g_noalloc_scratch) != cudaSuccess ||
          cudaGetSymbolAddress((void**)&f.index, g_noalloc_index) != cudaSuccess ||
          cudaGetSymbolAddress((void**)&f.flags, g_noalloc_flags) != cudaSuccess)
        return TC_ERR_CUDA;
      g_noalloc_dev[dev] = f;
    }
    D = g_noalloc_dev[dev];
  }
  return direct_with_scratch(n, x, y, z, vx, vy, vz, m, flags, ax, ay, az, pot, jx, jy, jz, jerk,
                             (cudaStream_t)stream, D.scratch, D.index, D.flags, TC_NOALLOC_MAX_N) == cudaSuccess
             ? TC_OK
             : TC_ERR_CUDA;
}

tc_status tc_train_selector(tc_ctx* ctx, int n, const double* x, const double* y, const double* z, const double* vx,
                            const double* vy, const double* vz, const double* m, int mem, int nsamples, int iters,
                            unsigned long long seed, tc_train_report* rep) {
  if (!ctx || n <= 0 || nsamples <= 0 || iters < 0) return TC_ERR_ARG;
  if (ctx->prm.p != 12 && ctx->prm.p != 16) return TC_ERR_UNSUPPORTED;
  auto t0 = std::chrono::steady_clock::now();
  const bool jerk = ctx->prm.variant == TC_VARIANT_JERKS;
  // a fixed-order evaluation builds the tree, the expansions and the lists
  int sel = ctx->prm.selector;
  int db = ctx->prm.direct_below;
  ctx->prm.selector = 0;
  ctx->prm.direct_below = 0;
  size_t N = (size_t)n;
  tc_status rs;
  if (mem == TC_MEM_HOST) {
    std::vector<double> o(7 * N);
    rs = tc_evaluate(ctx, n, x, y, z, vx, vy, vz, m, nullptr, o.data(), o.data() + N, o.data() + 2 * N,
                     o.data() + 3 * N, jerk ? o.data() + 4 * N : nullptr, jerk ? o.data() + 5 * N : nullptr,
                     jerk ? o.data() + 6 * N : nullptr, mem);
  } else {
    double* o = nullptr;
    if (cudaMalloc((void**)&o, 7 * N * sizeof(double)) != cudaSuccess) {
      ctx->prm.selector = sel;
      ctx->prm.direct_below = db;
      return TC_ERR_CUDA;
    }
    rs = tc_evaluate(ctx, n, x, y, z, vx, vy, vz, m, nullptr, o, o + N, o + 2 * N, o + 3 * N, jerk ? o + 4 * N : nullptr,
                     jerk ? o + 5 * N : nullptr, jerk ? o + 6 * N : nullptr, mem);
    cudaFree(o);
  }
  ctx->prm.selector = sel;
  ctx->prm.direct_below = db;
  if (rs != TC_OK) return rs;
  tc_status r2 = ctx->prm.p == 12 ? train_selector<12>(ctx, nsamples, iters, seed, rep)
                                  : train_selector<16>(ctx, nsamples, iters, seed, rep);
  if (rep) rep->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return r2;
}

tc_status tc_set_selector(tc_ctx* ctx, int selector, double tol) {
  if (!ctx || selector < 0 || selector > 2 || !(tol > 0.0)) return TC_ERR_ARG;
  if (selector == 2 && !ctx->mlp_ready) return TC_ERR_ARG;
  ctx->prm.selector = selector;
  ctx->prm.selector_tol = tol;
  return TC_OK;
}

tc_status tc_get_selector_data(tc_ctx* ctx, float* feat, float* labels, int* n, int* n_classes) {
  if (!ctx || !n) return TC_ERR_ARG;
  *n = ctx->train_n;
  if (n_classes) *n_classes = ctx->mlp_nout;
  if (feat && !ctx->train_feat.empty()) memcpy(feat, ctx->train_feat.data(), ctx->train_feat.size() * sizeof(float));
  if (labels && !ctx->train_lab.empty()) memcpy(labels, ctx->train_lab.data(), ctx->train_lab.size() * sizeof(float));
  return TC_OK;
}

int tc_selector_nparam(tc_ctx* ctx) {
  if (!ctx) return -1;
  int nout = ctx->prm.p == 12 ? TcOrderClasses<12>::n : ctx->prm.p == 16 ? TcOrderClasses<16>::n : 0;
  return nout ? tc_mlp_nparam(nout) : 0;
}

tc_status tc_get_selector_weights(tc_ctx* ctx, float* w, float* norm) {
  if (!ctx || !ctx->mlp_ready) return TC_ERR_ARG;
  if (w) TC_CK(cudaMemcpy(w, ctx->mlp_w.p, tc_mlp_nparam(ctx->mlp_nout) * sizeof(float), cudaMemcpyDeviceToHost));
  if (norm) {
    memcpy(norm, ctx->mlp_norm.mean, kMlpIn * sizeof(float));
    memcpy(norm + kMlpIn, ctx->mlp_norm.inv_std, kMlpIn * sizeof(float));
    norm[2 * kMlpIn] = ctx->mlp_norm.out_mean;
  }
  return TC_OK;
}

tc_status tc_set_selector_weights(tc_ctx* ctx, const float* w, const float* norm) {
  int np = tc_selector_nparam(ctx);
  if (!ctx || !w || !norm || np <= 0) return TC_ERR_ARG;
  TC_CK(cudaSetDevice(ctx->prm.device));
  TC_CK(ctx->mlp_w.ensure(np));
  TC_CK(cudaMemcpy(ctx->mlp_w.p, w, np * sizeof(float), cudaMemcpyHostToDevice));
  memcpy(ctx->mlp_norm.mean, norm, kMlpIn * sizeof(float));
  memcpy(ctx->mlp_norm.inv_std, norm + kMlpIn, kMlpIn * sizeof(float));
  ctx->mlp_norm.out_mean = norm[2 * kMlpIn];
  ctx->mlp_nout = ctx->prm.p == 12 ? TcOrderClasses<12>::n : TcOrderClasses<16>::n;
  ctx->mlp_ready = true;
  return TC_OK;
}

tc_status tc_mlp_loss_grad(int ns, int n_out, const float* feat, const float* labels, const float* w,
                           const float* norm, float* grad, float* loss) {
  if (ns <= 0 || n_out <= 0 || n_out > kMlpOutMax || !feat || !labels || !w || !norm || !grad || !loss)
    return TC_ERR_ARG;
  tc_ctx* ctx = nullptr;
  const int np = tc_mlp_nparam(n_out);
  float *df = nullptr, *dl = nullptr, *dw = nullptr, *dg = nullptr, *dloss = nullptr;
  TcMlpNorm nm;
  memcpy(nm.mean, norm, kMlpIn * sizeof(float));
  memcpy(nm.inv_std, norm + kMlpIn, kMlpIn * sizeof(float));
  nm.out_mean = norm[2 * kMlpIn];
  TC_CK(cudaMalloc((void**)&df, (size_t)ns * kMlpIn * sizeof(float)));
  TC_CK(cudaMalloc((void**)&dl, (size_t)ns * n_out * sizeof(float)));
  TC_CK(cudaMalloc((void**)&dw, np * sizeof(float)));
  TC_CK(cudaMalloc((void**)&dg, np * sizeof(float)));
  TC_CK(cudaMalloc((void**)&dloss, sizeof(float)));
  TC_CK(cudaMemcpy(df, feat, (size_t)ns * kMlpIn * sizeof(float), cudaMemcpyHostToDevice));
  TC_CK(cudaMemcpy(dl, labels, (size_t)ns * n_out * sizeof(float), cudaMemcpyHostToDevice));
  TC_CK(cudaMemcpy(dw, w, np * sizeof(float), cudaMemcpyHostToDevice));
  TC_CK(cudaMemset(dg, 0, np * sizeof(float)));
  TC_CK(cudaMemset(dloss, 0, sizeof(float)));
  k_mlp_grad<<<std::min(148, (ns + 255) / 256), 256>>>(ns, n_out, df, dl, dw, nm, dg, dloss);
  TC_CK(cudaGetLastError());
  TC_CK(cudaMemcpy(grad, dg, np * sizeof(float), cudaMemcpyDeviceToHost));
  TC_CK(cudaMemcpy(loss, dloss, sizeof(float), cudaMemcpyDeviceToHost));
  cudaFree(df); cudaFree(dl); cudaFree(dw); cudaFree(dg); cudaFree(dloss);
  return TC_OK;
}

// the selector's own inference (tensor cores, a warp per 32 samples), as k_select_order runs it
__global__ void __launch_bounds__(128) k_mlp_predict(int ns, int nout, const float* __restrict__ feat,
                                                     const float* __restrict__ w, TcMlpNorm norm,
                                                     float* __restrict__ pred) {
  __shared__ TcMlpTc T;
  __shared__ float act[4][32 * kMlpActS];
  tc_mlp_tc_load(T, w, nout, threadIdx.x, blockDim.x);
  __syncthreads();
  const int k = blockIdx.x * blockDim.x + threadIdx.x, wi = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float x[kMlpIn], y[kMlpOutMax];
  for (int i = 0; i < kMlpIn; i++)
    x[i] = k < ns ? (feat[(size_t)k * kMlpIn + i] - norm.mean[i]) * norm.inv_std[i] : 0.f;
  tc_mlp_infer_tc<kMlpOutMax>(T, act[wi], x, y, lane);
  if (k < ns)
    for (int j = 0; j < nout; j++) pred[(size_t)k * nout + j] = y[j] + norm.out_mean;
}

tc_status tc_mlp_predict(int ns, int n_out, const float* feat, const float* w, const float* norm, float* pred) {
  if (ns <= 0 || n_out <= 0 || n_out > kMlpOutMax || !feat || !w || !norm || !pred) return TC_ERR_ARG;
  tc_ctx* ctx = nullptr;
  const int np = tc_mlp_nparam(n_out);
  float *df = nullptr, *dw = nullptr, *dp = nullptr;
  TcMlpNorm nm;
  memcpy(nm.mean, norm, kMlpIn * sizeof(float));
  memcpy(nm.inv_std, norm + kMlpIn, kMlpIn * sizeof(float));
  nm.out_mean = norm[2 * kMlpIn];
  TC_CK(cudaMalloc((void**)&df, (size_t)ns * kMlpIn * sizeof(float)));
  TC_CK(cudaMalloc((void**)&dw, np * sizeof(float)));
  TC_CK(cudaMalloc((void**)&dp, (size_t)ns * n_out * sizeof(float)));
  TC_CK(cudaMemcpy(df, feat, (size_t)ns * kMlpIn * sizeof(float), cudaMemcpyHostToDevice));
  TC_CK(cudaMemcpy(dw, w, np * sizeof(float), cudaMemcpyHostToDevice));
  k_mlp_predict<<<(ns + 127) / 128, 128>>>(ns, n_out, df, dw, nm, dp);
  TC_CK(cudaGetLastError());
  TC_CK(cudaMemcpy(pred, dp, (size_t)ns * n_out * sizeof(float), cudaMemcpyDeviceToHost));
  cudaFree(df); cudaFree(dw); cudaFree(dp);
  return TC_OK;
}

tc_status tc_get_stats(tc_ctx* ctx, tc_stats* st) {
  if (!ctx || !st) return TC_ERR_ARG;
  *st = ctx->stats;
  return TC_OK;
}

tc_status tc_get_cells(tc_ctx* ctx, int* begin, int* nbody, int* nchild, int* child, int* level, double* X,
                       double* R, int* perm) {
  if (!ctx) return TC_ERR_ARG;
  int nc = ctx->ncell;
  size_t cc = ctx->ccap;
  if (nc > 0) {
    int* ci = ctx->cint.p;
    int* dsts[5] = {begin, nbody, nchild, child, level};
    int offs[5] = {0, 1, 2, 3, 5};
    for (int a = 0; a < 5; a++)
      if (dsts[a]) TC_CK(cudaMemcpy(dsts[a], ci + offs[a] * cc, nc * sizeof(int), cudaMemcpyDeviceToHost));
    if (X) {
      std::vector<double> t(nc);
      for (int d = 0; d < 3; d++) {
        TC_CK(cudaMemcpy(t.data(), ctx->cdbl.p + (3 + d) * cc, nc * sizeof(double), cudaMemcpyDeviceToHost));
        for (int i = 0; i < nc; i++) X[3 * i + d] = t[i];
      }
    }
    if (R) TC_CK(cudaMemcpy(R, ctx->cdbl.p + 6 * cc, nc * sizeof(double), cudaMemcpyDeviceToHost));
  }
  if (perm) TC_CK(cudaMemcpy(perm, ctx->perm.p, ctx->n * sizeof(int), cudaMemcpyDeviceToHost));
  return TC_OK;
}

tc_status tc_get_lists(tc_ctx* ctx, int kind, int* tgt, int* src) {
  if (!ctx || (kind != 0 && kind != 1)) return TC_ERR_ARG;
  unsigned long long cnt = kind ? ctx->n_p2p : ctx->n_m2l;
  if (!cnt) return TC_OK;
  std::vector<unsigned long long> k(cnt);
  TC_CK(cudaMemcpy(k.data(), kind ? ctx->p2p.p : ctx->m2l.p, cnt * sizeof(unsigned long long),
                   cudaMemcpyDeviceToHost));
  unsigned long long mask = (1ull << ctx->sbits) - 1ull;
  unsigned long long kmask = (1ull << (2 * ctx->sbits)) - 1ull;  // drop an order-class prefix
  for (auto& v : k) v &= kmask;
  std::sort(k.begin(), k.end());
  for (unsigned long long i = 0; i < cnt; i++) {
    if (tgt) tgt[i] = (int)(k[i] >> ctx->sbits);
    if (src) src[i] = (int)(k[i] & mask);
  }
  return TC_OK;
}

tc_status tc_get_expansions(tc_ctx* ctx, double* M, double* Md, double* L, double* Ld) {
  if (!ctx) return TC_ERR_ARG;
  int NT = TC_NTERM(ctx->prm.p);
  size_t ne = (size_t)ctx->ncell * NT;
  if (!ne) return TC_OK;
  TcCells cv = cells_view(ctx, NT);
  if (M) TC_CK(cudaMemcpy(M, cv.M, ne * sizeof(double), cudaMemcpyDeviceToHost));
  if (L) TC_CK(cudaMemcpy(L, cv.L, ne * sizeof(double), cudaMemcpyDeviceToHost));
  if (Md && cv.Md) TC_CK(cudaMemcpy(Md, cv.Md, ne * sizeof(double), cudaMemcpyDeviceToHost));
  if (Ld && cv.Ld) TC_CK(cudaMemcpy(Ld, cv.Ld, ne * sizeof(double), cudaMemcpyDeviceToHost));
  return TC_OK;
}

}  // extern "C"

#include "tc_integrate.cuh"
