// Order classes of the learned selector's outputs and the per-cell multipole power.
//
// The learned selector (tc_mlp.cuh, selection in tc_order.cuh) predicts the M2L truncation
// error of a pair at each order of TcOrderClasses<P>; Pn[n] = sqrt(sum_m M[n,m]^2 (n+m)!(n-m)!)
// (integrator.h:527-539) is the source spectrum both selectors read.
#pragma once
#include "tc_common.cuh"

namespace tc {

template <int P>
struct TcOrderClasses {
  static constexpr int n = 1;
  static constexpr int q[1] = {P};
  static __host__ __device__ constexpr int at(int) { return P; }
};
// Each class is one M2L launch over every target that has pairs of it, and a launch pays a fixed
// cost per such target (its accumulators and their ordered sum); at the headline's accuracy
// orders below 8 take about 1 % of the pairs, so the classes start at 8.
template <>
struct TcOrderClasses<12> {
  static constexpr int n = 3;
  static constexpr int q[3] = {8, 10, 12};
  static __host__ __device__ constexpr int at(int i) { return 8 + 2 * i; }
};
template <>
struct TcOrderClasses<16> {
  static constexpr int n = 3;
  static constexpr int q[3] = {10, 12, 16};
  static __host__ __device__ constexpr int at(int i) { return i < 2 ? 10 + 2 * i : 16; }
};

// The M2L launches of the order classes: launch i runs classes [first(i), first(i + 1)), at the
// order of its last class.  A pair of a lower class in a launch carries its own order in its
// source entry, and a 32-pair batch runs at the highest order among its pairs.  At p = 12 the
// two upper classes share a launch: the order-12 class alone is short per target (about 60
// pairs, two batches), which would leave most of a launch's warp groups idle.
template <int P>
struct TcClassLaunches {
  static constexpr int n = TcOrderClasses<P>::n;
  static __host__ __device__ constexpr int first(int i) { return i; }
};
template <>
struct TcClassLaunches<12> {
  static constexpr int n = 2;
  static __host__ __device__ constexpr int first(int i) { return i == 0 ? 0 : (i == 1 ? 1 : 3); }
};

#define TC_MAX_CLASSES 6
#define TC_NFEAT 8

// per-cell multipole power Pn[n] = sqrt(sum_m M[n,m]^2 (n+m)!(n-m)!)  (integrator.h:527-539)
template <int P>
__global__ void k_cell_pn(int ncell, const double* __restrict__ M, double* __restrict__ pn,
                          const int* ncdev = nullptr) {
  constexpr int NT = (P + 1) * (P + 1);
  if (ncdev) ncell = *ncdev;  // device-sized launch (graph)
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

}  // namespace tc
