// Per-pair expansion order for the far field.
//
// Each M2L pair (target t, source s) may use any order q in the context's order classes
// (TcOrderClasses<P>) instead of the fixed P.  Two selectors choose the smallest class whose
// predicted relative error -- |acceleration error| / (M_s / r^2), the error of the pair's
// contribution relative to the source's monopole acceleration -- is at most the tolerance:
//   analytic: the estimate the reference's error-controlled MAC uses
//     (traverse_eager.h:82-96, Dehnen 2014): 8 max(Rt,Rs)/(Rt+Rs) r^-(q+2)
//     sum_k C(q,k) Pn_s[q-k] Rt^k, with Pn the per-degree multipole power
//     (integrator.h:527-539);
//   learned: a small MLP (tc_mlp.cuh) fed with per-pair features.
// Pairs are then stably re-sorted by class, so each class is an ordered (target, source)
// sub-list with its own per-target offsets, and one M2L launch per class adds into L.
#pragma once
#include "tc_common.cuh"

namespace tc {

template <int P>
struct TcOrderClasses {
  static constexpr int n = 1;
  static constexpr int q[1] = {P};
  static __host__ __device__ constexpr int at(int) { return P; }
};
template <>
struct TcOrderClasses<12> {
  static constexpr int n = 5;
  static constexpr int q[5] = {4, 6, 8, 10, 12};
  static __host__ __device__ constexpr int at(int i) { return i < 4 ? 4 + 2 * i : 12; }
};
template <>
struct TcOrderClasses<16> {
  static constexpr int n = 6;
  static constexpr int q[6] = {4, 6, 8, 10, 12, 16};
  static __host__ __device__ constexpr int at(int i) { return i < 5 ? 4 + 2 * i : 16; }
};

#define TC_MAX_CLASSES 6
#define TC_NFEAT 8

// per-cell multipole power Pn[n] = sqrt(sum_m M[n,m]^2 (n+m)!(n-m)!)  (integrator.h:527-539)
template <int P>
__global__ void k_cell_pn(int ncell, const double* __restrict__ M, double* __restrict__ pn) {
  constexpr int NT = (P + 1) * (P + 1);
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
    const double* m = M + (size_t)c * NT;
    for (int n = 0; n <= P; n++) {
      double s = 0.0;
      for (int k = -n; k <= n; k++) {
        int a = k < 0 ? -k : k;
        double v = m[n * n + n + k];
        s += v * v * c_fact[n + a] * c_fact[n - a];
      }
      pn[(size_t)c * (P + 1) + n] = sqrt(s);
    }
  }
}

// pair geometry and source spectrum: the inputs of both selectors
struct TcPairFeat {
  double r, rt, rs, ms;
};

__device__ __forceinline__ TcPairFeat tc_pair_feat(const TcCells& c, int t, int s, const double* pn, int P) {
  TcPairFeat f;
  double dx = c.X[t] - c.X[s], dy = c.Y[t] - c.Y[s], dz = c.Z[t] - c.Z[s];
  f.r = sqrt(dx * dx + dy * dy + dz * dz);
  f.rt = c.R[t];
  f.rs = c.R[s];
  f.ms = fmax(pn[(size_t)s * (P + 1)], 1e-300);
  return f;
}

// relative error estimate of an order-q M2L for this pair (the reference's MAC estimate)
__device__ __forceinline__ double tc_est_rel_err(const TcPairFeat& f, const double* pns, int q) {
  double sum = 0.0, rk = 1.0, binom = 1.0;
  for (int k = 0; k <= q; k++) {
    sum += binom * pns[q - k] * rk;
    rk *= f.rt;
    binom = binom * (q - k) / (k + 1);
  }
  double e = 8.0 * fmax(f.rt, f.rs) / (f.rt + f.rs) * sum * pow(f.r, -(double)(q + 2));
  return e * f.r * f.r / f.ms;
}

// analytic selector: class index per pair (sorted list keys in, class-prefixed keys out)
template <int P>
__global__ void k_select_analytic(const unsigned long long* __restrict__ keys, unsigned long long n, int sbits,
                                  TcCells c, const double* __restrict__ pn, double tol,
                                  unsigned long long* __restrict__ out, unsigned int* __restrict__ hist) {
  using OC = TcOrderClasses<P>;
  __shared__ unsigned int h[TC_MAX_CLASSES];
  if (threadIdx.x < TC_MAX_CLASSES) h[threadIdx.x] = 0;
  __syncthreads();
  const unsigned long long mask = (1ull << sbits) - 1ull;
  for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned long long key = keys[k];
    int t = (int)(key >> sbits), s = (int)(key & mask);
    TcPairFeat f = tc_pair_feat(c, t, s, pn, P);
    const double* pns = pn + (size_t)s * (P + 1);
    int cls = OC::n - 1;
    for (int i = 0; i < OC::n - 1; i++)
      if (tc_est_rel_err(f, pns, OC::at(i)) <= tol) {
        cls = i;
        break;
      }
    out[k] = ((unsigned long long)cls << (2 * sbits)) | key;
    atomicAdd(&h[cls], 1u);
  }
  __syncthreads();
  if (threadIdx.x < TC_MAX_CLASSES && h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], h[threadIdx.x]);
}

// class prefix of a class-tagged key list -> keys without prefix (in place)
__global__ void k_strip_class(unsigned long long* keys, unsigned long long n, int sbits) {
  const unsigned long long mask = (1ull << (2 * sbits)) - 1ull;
  for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (unsigned long long)gridDim.x * blockDim.x)
    keys[k] &= mask;
}

}  // namespace tc
