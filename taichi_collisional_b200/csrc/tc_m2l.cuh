// Rotation-based O(p^3) M2L in FP64, target-stationary.
//
// Restates M2L_rotate (taichi_with_jerks/kernel_fast_lean.h:1130-1371, one-sided; the
// top-level mutual form kernel_fast_lean.h:1034-1295 equals two one-sided calls because the
// reference's visited pair set is symmetric):
//   scale M by (n+|m|)!(n-|m|)!, rotate about z by alpha_z, swap x<->z, rotate by alpha_x,
//   swap, unscale, translate along z, swap, rotate by -alpha_x, swap, rotate by -alpha_z.
// The reference's factorial table stops at (2P-1)! (kernel_fast_lean.h:127), so the scaled
// (P, +-P) entries are zero; that is reproduced here.
//
// Layout: one CTA per target cell; warp g owns the two degrees (g, P-g) of 32 (target,
// source) pairs at a time, one pair per lane, so every per-degree step -- including the
// constant swap matrices, emitted as straight-line code with immediate coefficients --
// runs in registers.  The only exchange is the z-translation, which mixes degrees and goes
// through shared memory (NT x 32 doubles).  Each lane accumulates its pairs' locals in
// registers; one warp reduction per target gives deterministic sums.
#pragma once
#include "swap_tables.h"
#include "tc_harmonics.cuh"

namespace tc {

__constant__ double c_fc[TC_NTERM(TC_PMAX_DEV)];
__constant__ double c_fcinv[TC_NTERM(TC_PMAX_DEV)];

__device__ __forceinline__ void tc_bar_cta() { asm volatile("bar.sync 1, %0;" ::"r"(blockDim.x) : "memory"); }

template <int D>
__device__ __forceinline__ void tc_rot_fwd(double* v, cd e1) {
  cd e = e1;
#pragma unroll
  for (int m = 1; m <= D; m++) {
    double im = v[D - m], re = v[D + m];
    v[D - m] = e.x * im + e.y * re;
    v[D + m] = e.x * re - e.y * im;
    e = e * e1;
  }
}

template <int D>
__device__ __forceinline__ void tc_rot_inv(double* v, cd e1) {
  cd e = e1;
#pragma unroll
  for (int m = 1; m <= D; m++) {
    double im = v[D - m], re = v[D + m];
    v[D - m] = e.x * im - e.y * re;
    v[D + m] = e.x * re + e.y * im;
    e = e * e1;
  }
}

struct TcPairGeo {
  cd ez1, ex1;
  double rinv;
};

__device__ __forceinline__ TcPairGeo tc_pair_geo(double dx, double dy, double dz) {
  TcPairGeo g;
  double rxy2 = dx * dx + dy * dy, rxy = sqrt(rxy2);
  double r = sqrt(rxy2 + dz * dz);
  g.rinv = 1.0 / r;
  g.ez1 = mk(1, 0);
  g.ex1 = mk(dz * g.rinv, -rxy * g.rinv);
  if (rxy > 0) {
    double q = 1.0 / rxy;
    g.ez1 = mk(dy * q, dx * q);
  }
  return g;
}

// forward half for degree D: scaled, rotated into the pair frame, unscaled -> smem
template <int P, int D>
__device__ __forceinline__ void tc_m2l_fwd(const double* __restrict__ Ms, const TcPairGeo& g, double* buf, int lane) {
  double v[2 * D + 1], o[2 * D + 1];
#pragma unroll
  for (int k = 0; k < 2 * D + 1; k++) v[k] = __ldg(Ms + D * D + k) * c_fc[D * D + k];
  if (D == P) {
    v[0] = 0.0;
    v[2 * D] = 0.0;
  }
  tc_rot_fwd<D>(v, g.ez1);
  TcSwapDeg<D>::apply(v, o);
  tc_rot_fwd<D>(o, g.ex1);
  TcSwapDeg<D>::apply(o, v);
#pragma unroll
  for (int k = 0; k < 2 * D + 1; k++) buf[(D * D + k) * 32 + lane] = v[k] * c_fcinv[D * D + k];
}

// translation along z to output degree N, then rotation back; accumulate into acc
template <int P, int N>
__device__ __forceinline__ void tc_m2l_back(const double* buf, int lane, const TcPairGeo& g, double* acc, bool valid) {
  double l[2 * N + 1], o[2 * N + 1];
#pragma unroll
  for (int k = 0; k < 2 * N + 1; k++) l[k] = 0.0;
  const double rinv = g.rinv;
  double pn = rinv;
#pragma unroll
  for (int j = 0; j < N; j++) pn *= rinv;  // rinv^(N+1)
  {
    double s = 0.0, pr = pn;
#pragma unroll
    for (int k = 0; k <= P - N; k++) {
      s += buf[(k * k + k) * 32 + lane] * (c_fact[N + k] * pr);
      pr *= rinv;
    }
    l[N] = s;
  }
  double pm = rinv, sg = -1.0;
  constexpr int MMAX = N < P - N ? N : P - N;
#pragma unroll
  for (int m = 1; m <= MMAX; m++) {
    double pr = pn * pm, sn = 0.0, sp = 0.0;
#pragma unroll
    for (int k = m; k <= P - N; k++) {
      double f = c_fact[N + k] * pr * sg;
      sn += buf[(k * k + k - m) * 32 + lane] * f;
      sp += buf[(k * k + k + m) * 32 + lane] * f;
      pr *= rinv;
    }
    l[N - m] = sn;
    l[N + m] = sp;
    sg = -sg;
    pm *= rinv;
  }
  TcSwapDeg<N>::apply(l, o);
  tc_rot_inv<N>(o, g.ex1);
  TcSwapDeg<N>::apply(o, l);
  tc_rot_inv<N>(l, g.ez1);
  if (valid) {
#pragma unroll
    for (int k = 0; k < 2 * N + 1; k++) acc[k] += l[k];
  }
}

template <int N>
__device__ __forceinline__ void tc_warp_sum_store(double* acc, double* dst) {
#pragma unroll
  for (int k = 0; k < 2 * N + 1; k++) {
    double v = acc[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    acc[k] = v;
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int k = 0; k < 2 * N + 1; k++) dst[N * N + k] = acc[k];
  }
}

template <int P, int G, bool JERK>
__device__ void tc_m2l_group(int t, int s_beg, int s_end, const int* __restrict__ src, const TcCells& c, double* buf) {
  constexpr int NT = (P + 1) * (P + 1);
  constexpr int D1 = G, D2 = P - G;
  constexpr bool TWO = D1 != D2;
  int lane = threadIdx.x & 31;
  double Xt = c.X[t], Yt = c.Y[t], Zt = c.Z[t];
  for (int arr = 0; arr < (JERK ? 2 : 1); arr++) {
    const double* Mbase = arr ? c.Md : c.M;
    double a1[2 * D1 + 1], a2[2 * D2 + 1];
#pragma unroll
    for (int k = 0; k < 2 * D1 + 1; k++) a1[k] = 0.0;
#pragma unroll
    for (int k = 0; k < 2 * D2 + 1; k++) a2[k] = 0.0;
    for (int b0 = s_beg; b0 < s_end; b0 += 32) {
      int idx = b0 + lane;
      bool valid = idx < s_end;
      int s = src[valid ? idx : s_beg];
      TcPairGeo g = tc_pair_geo(Xt - c.X[s], Yt - c.Y[s], Zt - c.Z[s]);
      const double* Ms = Mbase + (size_t)s * NT;
      tc_m2l_fwd<P, D1>(Ms, g, buf, lane);
      if (TWO) tc_m2l_fwd<P, D2>(Ms, g, buf, lane);
      tc_bar_cta();
      tc_m2l_back<P, D1>(buf, lane, g, a1, valid);
      if (TWO) tc_m2l_back<P, D2>(buf, lane, g, a2, valid);
      tc_bar_cta();
    }
    double* Lt = (arr ? c.Ld : c.L) + (size_t)t * NT;
    tc_warp_sum_store<D1>(a1, Lt);
    if (TWO) tc_warp_sum_store<D2>(a2, Lt);
  }
}

template <int P, int G, bool JERK>
struct TcM2LDispatch {
  static __device__ __forceinline__ void run(int g, int t, int sb, int se, const int* src, const TcCells& c, double* buf) {
    if (g == G)
      tc_m2l_group<P, G, JERK>(t, sb, se, src, c, buf);
    else
      TcM2LDispatch<P, G + 1, JERK>::run(g, t, sb, se, src, c, buf);
  }
};
template <int P, bool JERK>
struct TcM2LDispatch<P, P / 2 + 1, JERK> {
  static __device__ __forceinline__ void run(int, int, int, int, const int*, const TcCells&, double*) {}
};

template <int P>
constexpr int tc_m2l_threads() { return 32 * (P / 2 + 1); }

template <int P, bool JERK>
__global__ void __launch_bounds__(tc_m2l_threads<P>()) k_m2l(const int* __restrict__ tlist, int ntl,
                                                               const int* __restrict__ tstart,
                                                               const int* __restrict__ src, TcCells c) {
  extern __shared__ double tc_m2l_buf[];
  int ti = blockIdx.x;
  if (ti >= ntl) return;
  int t = tlist[ti];
  if (!c.has_sink[t]) return;
  int g = threadIdx.x >> 5;
  TcM2LDispatch<P, 0, JERK>::run(g, t, tstart[t], tstart[t + 1], src, c, tc_m2l_buf);
}

}  // namespace tc
