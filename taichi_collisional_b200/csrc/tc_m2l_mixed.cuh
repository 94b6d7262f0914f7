// Mixed-precision rotation M2L: the same O(p^3) scheme as tc_m2l.cuh (rotate about z,
// swap x<->z, rotate, swap, translate along z, and back), with the per-pair work in FP32.
//
// Conditioning.  In the reference's homogeneous scaling (M * (n+|m|)!(n-|m|)!) the swap
// matrices hold integers up to ~2.5e6 * 2^-11 at p = 12 and mix coefficients of very
// different size, which FP32 cannot carry.  Here each source multipole enters as
//   w[n,m] = M[n,m] * F[n,m] / r^n,   F = sqrt((n+|m|)!(n-|m|)!) * (1 for m = 0, sqrt2 else)
// in which every swap T_n = E S_n E^-1 is orthogonal (generated in swap_tables.h) and every
// phase rotation is unitary, so FP32 errors stay at the 1e-7 level of each degree's norm.
// With that scaling the z-translation no longer depends on the pair:
//   u[n,+-m] = sum_k C[n,k,m] w''[k,+-m],  C = (-1)^m (n+k)! / sqrt(D[n,m] D[k,m])
// and the local contribution is L[n,m] = u''[n,m] * (D/F)[n,m] / r^(n+1), accumulated in
// FP64.  Pair geometry (angles, their powers, 1/r) is formed in FP64 from FP64 cell centres
// before any FP32 arithmetic.  The (P, +-P) multipole entries are zeroed as in the FP64 path
// (factorial_table[2P] == 0 in the reference).
#pragma once
#include "tc_m2l.cuh"

namespace tc {

__constant__ double c_mF[TC_NTERM(TC_PMAX_DEV)];
__constant__ double c_mDoF[TC_NTERM(TC_PMAX_DEV)];
__constant__ float c_mC[(TC_PMAX_DEV + 1) * (TC_PMAX_DEV + 1) * (TC_PMAX_DEV + 1)];

#define TC_MC(n, k, m) c_mC[((n) * (TC_PMAX_DEV + 1) + (k)) * (TC_PMAX_DEV + 1) + (m)]

// phase tables: et[(2m)*32+lane] = Re e^{i m a}, et[(2m+1)*32+lane] = Im
template <int D>
__device__ __forceinline__ void tc_rotf_fwd(float* v, const float* et, int lane) {
#pragma unroll
  for (int m = 1; m <= D; m++) {
    float er = et[(2 * m) * 32 + lane], ei = et[(2 * m + 1) * 32 + lane];
    float im = v[D - m], re = v[D + m];
    v[D - m] = er * im + ei * re;
    v[D + m] = er * re - ei * im;
  }
}
template <int D>
__device__ __forceinline__ void tc_rotf_inv(float* v, const float* et, int lane) {
#pragma unroll
  for (int m = 1; m <= D; m++) {
    float er = et[(2 * m) * 32 + lane], ei = et[(2 * m + 1) * 32 + lane];
    float im = v[D - m], re = v[D + m];
    v[D - m] = er * im - ei * re;
    v[D + m] = er * re + ei * im;
  }
}

template <int P>
struct TcM2LMixSmem {
  static constexpr int NT = (P + 1) * (P + 1);
  // in floats: buf (NT*32) | ez table (2(P+1)*32) | ex table (2(P+1)*32) | rinv (double, 32)
  static constexpr int BUF = 0, EZ = NT * 32, EX = EZ + 2 * (P + 1) * 32, RINV = EX + 2 * (P + 1) * 32;
  static constexpr int FLOATS = RINV + 2 * 32;
  // doubles after the floats: acc (NT*32)
  static constexpr int ACC_D = (FLOATS + 1) / 2;
  static constexpr int BYTES = (ACC_D + NT * 32) * 8;
};

template <int P, int D>
__device__ __forceinline__ void tc_m2lx_fwd(const double* __restrict__ Ms, double rinv, const float* ez,
                                            const float* ex, float* buf, int lane) {
  float v[2 * D + 1], o[2 * D + 1];
  double rn = 1.0;
#pragma unroll
  for (int j = 0; j < D; j++) rn *= rinv;
#pragma unroll
  for (int k = 0; k < 2 * D + 1; k++) v[k] = (float)(__ldg(Ms + D * D + k) * (c_mF[D * D + k] * rn));
  if (D == P) {
    v[0] = 0.f;
    v[2 * D] = 0.f;
  }
  tc_rotf_fwd<D>(v, ez, lane);
  TcSwapOrthDeg<D>::apply(v, o);
  tc_rotf_fwd<D>(o, ex, lane);
  TcSwapOrthDeg<D>::apply(o, v);
#pragma unroll
  for (int k = 0; k < 2 * D + 1; k++) buf[(D * D + k) * 32 + lane] = v[k];
}

template <int P, int N>
__device__ __forceinline__ void tc_m2lx_back(const float* buf, const float* ez, const float* ex, double rinv,
                                             int lane, double* acc, bool valid) {
  float l[2 * N + 1], o[2 * N + 1];
#pragma unroll
  for (int k = 0; k < 2 * N + 1; k++) l[k] = 0.f;
  {
    float s = 0.f;
#pragma unroll
    for (int k = 0; k <= P - N; k++) s += buf[(k * k + k) * 32 + lane] * TC_MC(N, k, 0);
    l[N] = s;
  }
  constexpr int MMAX = N < P - N ? N : P - N;
#pragma unroll
  for (int m = 1; m <= MMAX; m++) {
    float sn = 0.f, sp = 0.f;
#pragma unroll
    for (int k = m; k <= P - N; k++) {
      float f = TC_MC(N, k, m);
      sn += buf[(k * k + k - m) * 32 + lane] * f;
      sp += buf[(k * k + k + m) * 32 + lane] * f;
    }
    l[N - m] = sn;
    l[N + m] = sp;
  }
  TcSwapOrthDeg<N>::apply(l, o);
  tc_rotf_inv<N>(o, ex, lane);
  TcSwapOrthDeg<N>::apply(o, l);
  tc_rotf_inv<N>(l, ez, lane);
  if (valid) {
    double rn = rinv;
#pragma unroll
    for (int j = 0; j < N; j++) rn *= rinv;
#pragma unroll
    for (int k = 0; k < 2 * N + 1; k++) acc[(N * N + k) * 32 + lane] += (double)l[k] * (c_mDoF[N * N + k] * rn);
  }
}

template <int P, int G>
struct TcM2LXDispatch {
  static __device__ __forceinline__ void fwd(int g, const double* Ms, double rinv, const float* ez, const float* ex,
                                             float* buf, int lane) {
    if (g == G) {
      tc_m2lx_fwd<P, G>(Ms, rinv, ez, ex, buf, lane);
      if (G != P - G) tc_m2lx_fwd<P, P - G>(Ms, rinv, ez, ex, buf, lane);
    } else {
      TcM2LXDispatch<P, G + 1>::fwd(g, Ms, rinv, ez, ex, buf, lane);
    }
  }
  static __device__ __forceinline__ void back(int g, const float* buf, const float* ez, const float* ex, double rinv,
                                              int lane, double* acc, bool valid) {
    if (g == G) {
      tc_m2lx_back<P, G>(buf, ez, ex, rinv, lane, acc, valid);
      if (G != P - G) tc_m2lx_back<P, P - G>(buf, ez, ex, rinv, lane, acc, valid);
    } else {
      TcM2LXDispatch<P, G + 1>::back(g, buf, ez, ex, rinv, lane, acc, valid);
    }
  }
};
template <int P>
struct TcM2LXDispatch<P, P / 2 + 1> {
  static __device__ __forceinline__ void fwd(int, const double*, double, const float*, const float*, float*, int) {}
  static __device__ __forceinline__ void back(int, const float*, const float*, const float*, double, int, double*,
                                              bool) {}
};

template <int P>
constexpr int tc_m2lx_threads() { return 32 * (P / 2 + 1); }

template <int P, bool JERK>
__global__ void __launch_bounds__(tc_m2lx_threads<P>(), 2) k_m2l_mixed(const int* __restrict__ tlist, int ntl,
                                                                        const int* __restrict__ tstart,
                                                                        const int* __restrict__ src, TcCells c) {
  using SM = TcM2LMixSmem<P>;
  constexpr int NT = SM::NT;
  extern __shared__ double tc_m2lx_smem[];
  float* fs = reinterpret_cast<float*>(tc_m2lx_smem);
  float* buf = fs + SM::BUF;
  float* ez = fs + SM::EZ;
  float* ex = fs + SM::EX;
  double* rinvs = reinterpret_cast<double*>(fs + SM::RINV);
  double* acc = tc_m2lx_smem + SM::ACC_D;
  int ti = blockIdx.x;
  if (ti >= ntl) return;
  int t = tlist[ti];
  if (!c.has_sink[t]) return;
  const int g = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int s_beg = tstart[t], s_end = tstart[t + 1];
  const double Xt = c.X[t], Yt = c.Y[t], Zt = c.Z[t];
  for (int arr = 0; arr < (JERK ? 2 : 1); arr++) {
    const double* Mbase = arr ? c.Md : c.M;
    for (int i = threadIdx.x; i < NT * 32; i += blockDim.x) acc[i] = 0.0;
    for (int b0 = s_beg; b0 < s_end; b0 += 32) {
      int idx = b0 + lane;
      bool valid = idx < s_end;
      int s = src[valid ? idx : s_beg];
      if (g == 0) {
        TcPairGeo pg = tc_pair_geo(Xt - c.X[s], Yt - c.Y[s], Zt - c.Z[s]);
        rinvs[lane] = pg.rinv;
        cd a = mk(1, 0), b = mk(1, 0);
        for (int m = 0; m <= P; m++) {
          ez[(2 * m) * 32 + lane] = (float)a.x;
          ez[(2 * m + 1) * 32 + lane] = (float)a.y;
          ex[(2 * m) * 32 + lane] = (float)b.x;
          ex[(2 * m + 1) * 32 + lane] = (float)b.y;
          a = a * pg.ez1;
          b = b * pg.ex1;
        }
      }
      tc_bar_cta();
      double rinv = rinvs[lane];
      TcM2LXDispatch<P, 0>::fwd(g, Mbase + (size_t)s * NT, rinv, ez, ex, buf, lane);
      tc_bar_cta();
      TcM2LXDispatch<P, 0>::back(g, buf, ez, ex, rinv, lane, acc, valid);
      tc_bar_cta();
    }
    double* Lt = (arr ? c.Ld : c.L) + (size_t)t * NT;
    for (int r = threadIdx.x; r < NT; r += blockDim.x) {
      double v = 0.0;
#pragma unroll 8
      for (int q = 0; q < 32; q++) v += acc[r * 32 + q];
      Lt[r] = v;
    }
    tc_bar_cta();
  }
}

}  // namespace tc
