// Per-pair expansion order with a per-target error budget.
//
// Every M2L pair (t, s) may be evaluated at an order q <= P instead of the fixed P.  The budget of
// a pair is a fraction `tol` of the target's acceleration: the order is the smallest q whose
// predicted truncation error -- the absolute acceleration error of the pair's contribution -- is
// at most tol * A_t, where A_t is the least acceleration magnitude among the target cell's bodies
// (the role the cell's min_acc plays in the reference's error-controlled MAC,
// traverse_eager.h:82-96).  A_t comes from the previous evaluation of the same bodies (caller
// indices), so a time-stepping caller pays nothing for it; an evaluation without one runs at the
// fixed order.  The predictions:
//   analytic: the reference's MAC estimate with the order q in place of P (traverse_eager.h:82-96,
//     Dehnen 2014): 8 max(Rt, Rs) / (Rt + Rs) r^-(q+2) sum_k C(q, k) Pn_s[q-k] Rt^k, with Pn the
//     per-degree multipole power (integrator.h:527-539);
//   learned: the MLP of tc_mlp.cuh, which predicts log10 of each class's error relative to the
//     source's monopole acceleration M_s / r^2, rescaled to an absolute error; a warp's 32 pairs
//     go through it together on the tensor cores (tc_mlp_infer_tc).
// Each target's source list is then stably regrouped by order class (one warp per target) and
// the classes run as the M2L launches of TcClassLaunches (k_m2l<P, Q>, each with its balanced
// per-degree work split) over per-target ranges, each source entry carrying how far its pair's
// order lies below its launch's; the launches are persistent grids that read their counts on
// the device, so nothing here synchronises with the host and the selection is part of the
// captured graph.
#pragma once
#include "tc_mlp.cuh"

namespace tc {

constexpr int kOrderMin = 3;  // lowest order a pair may get

// the orders of the classes (TcOrderClasses) and the binomials C(P, k) of the estimate as the
// reference forms them (kernel_fast_lean.h:139)
struct TcClassOrders {
  int q[TC_MAX_CLASSES];
  int below[TC_MAX_CLASSES];  // per class: its launch's order minus its own (source-entry top bits)
  double comb[TC_PMAX_DEV + 1];
};

// |a| of each body in caller order (the next evaluation's error budget)
__global__ void k_amag(int n, const double* __restrict__ ax, const double* __restrict__ ay,
                       const double* __restrict__ az, double* __restrict__ amag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) amag[i] = sqrt(ax[i] * ax[i] + ay[i] * ay[i] + az[i] * az[i]);
}

// the previous |a| of the body now at sorted position i
__global__ void k_gather_scale(int n, const int* __restrict__ perm, const double* __restrict__ amag,
                               double* __restrict__ sc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) sc[i] = amag[perm[i]];
}

// Class (index into TcClassOrders) of one pair by the analytic selector (mode 1), which
// evaluates the reference's estimate once, at the full order P,
//   E_P = 8 max(Rt, Rs) / (Rt + Rs) r^-(P+2) sum_k C(P, k) Pn_s[P-k] Rt^k,
// and scales it to lower orders by the convergence ratio rho = (Rt + Rs) / r of the pair
// (E_q ~ E_P rho^(q-P), the geometric decay of the estimate's leading term), so the order is
// q = P - floor(ln(budget / E_P) / ln(1 / rho)), rounded up to the next class.
template <int P>
__device__ __forceinline__ int tc_pair_class(const TcCells& c, int t, int s, const double* __restrict__ pn,
                                             double budget, int nclass, const int* cls_order, const double* comb) {
  if (!(budget > 0.0)) return nclass - 1;
  const double dx = c.X[t] - c.X[s], dy = c.Y[t] - c.Y[s], dz = c.Z[t] - c.Z[s];
  const double r2 = dx * dx + dy * dy + dz * dz, r = sqrt(r2);
  const double* pns = pn + (size_t)s * (P + 1);
  const double rt = c.R[t], rs = c.R[s];
  double sum = 0.0, rk = 1.0;
#pragma unroll
  for (int k = 0; k <= P; k++) {
    sum += comb[k] * pns[P - k] * rk;
    rk *= rt;
  }
  double rp = r2;  // r^(P+2)
#pragma unroll
  for (int k = 0; k < P; k++) rp *= r;
  const double ep = 8.0 * fmax(rt, rs) / (rt + rs) * sum / rp;
  if (!(ep > budget)) {
    const double rho = (rt + rs) / r;
    int q = kOrderMin;
    if (rho > 0.0 && rho < 1.0 && ep > 0.0) q = P - (int)floor(log(budget / ep) / -log(rho));
    for (int i = 0; i < nclass; i++)
      if (cls_order[i] >= q) return i;
  }
  return nclass - 1;
}

// Class of one pair by the learned selector (mode 2), warp-wide: every lane of the warp calls it
// (with some valid pair) and the 32 pairs go through the network together on the tensor cores.
// Features as tc_pair_features: the geometry per pair, the rest per cell (featc).
template <int P>
__device__ __forceinline__ int tc_pair_class_mlp(const TcCells& c, int t, int s, const double* __restrict__ pn,
                                                 double budget, const TcMlpTc& T, float* act, const TcMlpNorm& norm,
                                                 const float* __restrict__ featc, int lane) {
  constexpr int NO = TcOrderClasses<P>::n;
  // the features and the budget in FP32 (the network itself runs on TF32 operands)
  const double dx = c.X[t] - c.X[s], dy = c.Y[t] - c.Y[s], dz = c.Z[t] - c.Z[s];
  const float r2 = (float)(dx * dx + dy * dy + dz * dz), lr = 0.5f * logf(r2);
  float x[kMlpIn], y[NO];
  x[0] = logf((float)c.R[t]) - lr;
  x[1] = logf((float)c.R[s]) - lr;
#pragma unroll
  for (int j = 0; j < 5; j++) x[2 + j] = featc[(size_t)s * 5 + j];
  x[7] = featc[(size_t)t * 5 + 4];
#pragma unroll
  for (int i = 0; i < kMlpIn; i++) x[i] = (x[i] - norm.mean[i]) * norm.inv_std[i];
  tc_mlp_infer_tc<NO>(T, act, x, y, lane);
  if (!(budget > 0.0)) return NO - 1;
  // log10 of the budget relative to the source's monopole acceleration
  const float lim = (logf((float)budget) + logf(r2) - logf(fmaxf((float)pn[(size_t)s * (P + 1)], 1e-37f))) *
                    0.43429448f;
#pragma unroll
  for (int i = 0; i < NO - 1; i++)
    if (y[i] + norm.out_mean <= lim) return i;
  return NO - 1;
}

// One warp per target of the M2L target list: every pair's class (pass 1, kept in `cls`), then
// the target's entries regrouped by class, lowest order first, stably, into src_out (pass 2):
// class k of target t occupies [cbeg[k * cstride + t], cend[k * cstride + t]), cstride being the
// cell capacity of those arrays (the M2L launches index them with the same stride).  hist[k]
// counts the pairs of class k.
template <int P>
__global__ void __launch_bounds__(128) k_select_order(const int* __restrict__ tlist, int ntl,
                                                      const int* __restrict__ tstart, const int* __restrict__ src_in,
                                                      int* __restrict__ src_out, uint8_t* __restrict__ cls,
                                                      int* __restrict__ cbeg, int* __restrict__ cend, int cstride,
                                                      const TcCells c, const double* __restrict__ pn,
                                                      const double* __restrict__ cell_scale, double tol, int mode,
                                                      const float* __restrict__ w, TcMlpNorm norm, int nclass,
                                                      TcClassOrders co, const float* __restrict__ featc,
                                                      unsigned* __restrict__ hist, const unsigned* ntldev = nullptr) {
  __shared__ TcMlpTc T;
  __shared__ float act[4][32 * kMlpActS];
  __shared__ unsigned cnt[4][32], base[4][32];
  __shared__ unsigned sh[32];
  if (ntldev) ntl = (int)*ntldev;  // device-sized launch (graph)
  const int wi = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (mode == 2) tc_mlp_tc_load(T, w, nclass, threadIdx.x, blockDim.x);
  if (threadIdx.x < 32) sh[threadIdx.x] = 0;
  __syncthreads();
  for (int k = blockIdx.x * 4 + wi; k < ntl; k += gridDim.x * 4) {
    const int t = tlist[k];
    const int beg = tstart[t], end = tstart[t + 1];
    const double budget = tol * cell_scale[t];
    cnt[wi][lane] = 0;
    __syncwarp();
    for (int q0 = beg; q0 < end; q0 += 32) {
      const int e = q0 + lane;
      const bool ok = e < end;
      int ci;
      if (mode == 2) {  // warp-wide: lanes past the end run the target's first pair
        const int s = src_in[ok ? e : beg] & kM2LSrcMask;
        ci = tc_pair_class_mlp<P>(c, t, s, pn, budget, T, act[wi], norm, featc, lane);
      } else {
        ci = ok ? tc_pair_class<P>(c, t, src_in[e] & kM2LSrcMask, pn, budget, nclass, co.q, co.comb) : 0;
      }
      if (ok) {
        cls[e] = (uint8_t)ci;
        atomicAdd(&cnt[wi][ci], 1u);
      }
    }
    __syncwarp();
    // exclusive prefix over the classes (lane = class)
    const unsigned v = cnt[wi][lane];
    unsigned incl = v;
    for (int d = 1; d < 32; d <<= 1) {
      const unsigned u = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += u;
    }
    base[wi][lane] = incl - v;
    if (lane < nclass) {
      cbeg[(size_t)lane * cstride + t] = beg + (int)(incl - v);
      cend[(size_t)lane * cstride + t] = beg + (int)incl;
    }
    if (v) atomicAdd(&sh[lane], v);
    __syncwarp();
    for (int q0 = beg; q0 < end; q0 += 32) {
      const int e = q0 + lane;
      const bool ok = e < end;
      const int ci = ok ? cls[e] : 31;
      const unsigned peers = __match_any_sync(0xffffffffu, ci);
      const unsigned rank = __popc(peers & ((1u << lane) - 1u));
      if (ok) src_out[beg + base[wi][ci] + rank] = (src_in[e] & kM2LSrcMask) | (co.below[ci] << kM2LOrderShift);
      __syncwarp();
      if (ok && rank == 0) base[wi][ci] += __popc(peers);
      __syncwarp();
    }
  }
  __syncthreads();
  if (threadIdx.x < 32 && sh[threadIdx.x]) atomicAdd(&hist[threadIdx.x], sh[threadIdx.x]);
}

}  // namespace tc
