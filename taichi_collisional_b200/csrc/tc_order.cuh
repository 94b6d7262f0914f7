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
//     source's monopole acceleration M_s / r^2, rescaled to an absolute error.
// Each target's source list is then stably regrouped by order (one warp per target), and every
// entry carries its order in the top bits of the source index (kM2LOrderShift), so one M2L launch
// serves all orders: a batch of 32 pairs runs at the largest order among them.  Nothing here
// synchronises with the host, so the selection is part of the captured graph.
#pragma once
#include "tc_mlp.cuh"

namespace tc {

constexpr int kOrderMin = 3;  // lowest order a pair may get

// the orders the learned selector's outputs stand for (TcOrderClasses)
struct TcClassOrders {
  int q[TC_MAX_CLASSES];
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

// absolute truncation-error estimate of an order-q M2L for the pair (the reference's estimate)
__device__ __forceinline__ double tc_est_abs_err(double r, double rt, double rs, const double* pns, int q) {
  double sum = 0.0, rk = 1.0, binom = 1.0;
  for (int k = 0; k <= q; k++) {
    sum += binom * pns[q - k] * rk;
    rk *= rt;
    binom = binom * (q - k) / (k + 1);
  }
  return 8.0 * fmax(rt, rs) / (rt + rs) * sum * pow(r, -(double)(q + 2));
}

// order of one pair (mode 1 analytic, 2 learned)
template <int P>
__device__ __forceinline__ int tc_pair_order(const TcCells& c, int t, int s, const double* __restrict__ pn,
                                             double budget, int mode, const float* sw, const TcMlpNorm& norm,
                                             int nclass, const int* cls_order) {
  if (!(budget > 0.0)) return P;
  const double dx = c.X[t] - c.X[s], dy = c.Y[t] - c.Y[s], dz = c.Z[t] - c.Z[s];
  const double r = sqrt(dx * dx + dy * dy + dz * dz);
  const double* pns = pn + (size_t)s * (P + 1);
  if (mode == 2) {
    float x[kMlpIn], a1[kMlpH], a2[kMlpH], a3[kMlpH], y[kMlpOutMax];
    tc_pair_features(c, t, s, pn, P, x);
    for (int i = 0; i < kMlpIn; i++) x[i] = (x[i] - norm.mean[i]) * norm.inv_std[i];
    tc_mlp_forward<true>(sw, nclass, x, a1, a2, a3, y);
    // log10 of the budget relative to the source's monopole acceleration
    const double mono = fmax(pns[0], 1e-300) / (r * r);
    const float lim = (float)log10(budget / mono);
    for (int i = 0; i < nclass - 1; i++)
      if (y[i] + norm.out_mean <= lim) return cls_order[i];
    return P;
  }
  for (int q = kOrderMin; q < P; q++)
    if (tc_est_abs_err(r, c.R[t], c.R[s], pns, q) <= budget) return q;
  return P;
}

// One warp per target of the M2L target list: every pair's order (pass 1, kept in `off` as
// P - q), then the target's entries regrouped by order, stably, into src_out with the order in
// the top bits (pass 2).  hist[P - q] counts the pairs of each order.
template <int P>
__global__ void __launch_bounds__(128) k_select_order(const int* __restrict__ tlist, int ntl,
                                                      const int* __restrict__ tstart, const int* __restrict__ src_in,
                                                      int* __restrict__ src_out, uint8_t* __restrict__ off,
                                                      const TcCells c, const double* __restrict__ pn,
                                                      const double* __restrict__ cell_scale, double tol, int mode,
                                                      const float* __restrict__ w, TcMlpNorm norm, int nclass,
                                                      TcClassOrders cls, unsigned* __restrict__ hist,
                                                      const unsigned* ntldev = nullptr) {
  __shared__ float sw[kMlpParamMax];
  __shared__ unsigned cnt[4][32], base[4][32];
  __shared__ unsigned sh[32];
  if (ntldev) ntl = (int)*ntldev;  // device-sized launch (graph)
  const int wi = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (mode == 2)
    for (int i = threadIdx.x; i < tc_mlp_nparam(nclass); i += blockDim.x) sw[i] = w[i];
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
      if (e < end) {
        const int s = src_in[e] & kM2LSrcMask;
        const int o = P - tc_pair_order<P>(c, t, s, pn, budget, mode, sw, norm, nclass, cls.q);
        off[e] = (uint8_t)o;
        atomicAdd(&cnt[wi][o], 1u);
      }
    }
    __syncwarp();
    // exclusive prefix over the orders (lane = P - q), full orders first
    const unsigned v = cnt[wi][lane];
    unsigned incl = v;
    for (int d = 1; d < 32; d <<= 1) {
      const unsigned u = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += u;
    }
    base[wi][lane] = incl - v;
    if (v) atomicAdd(&sh[lane], v);
    __syncwarp();
    for (int q0 = beg; q0 < end; q0 += 32) {
      const int e = q0 + lane;
      const bool ok = e < end;
      const int o = ok ? off[e] : 31;
      const unsigned peers = __match_any_sync(0xffffffffu, o);
      const unsigned rank = __popc(peers & ((1u << lane) - 1u));
      if (ok) src_out[beg + base[wi][o] + rank] = (src_in[e] & kM2LSrcMask) | (o << kM2LOrderShift);
      __syncwarp();
      if (ok && rank == 0) base[wi][o] += __popc(peers);
      __syncwarp();
    }
  }
  __syncthreads();
  if (threadIdx.x < 32 && sh[threadIdx.x]) atomicAdd(&hist[threadIdx.x], sh[threadIdx.x]);
}

}  // namespace tc
