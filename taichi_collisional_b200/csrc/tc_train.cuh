// Training data for the learned order selector, produced by the FMM itself.
//
// For K (target, source) pairs drawn from a real M2L list: the local expansion at the target
// from the source alone at each order class (the production M2L code path, order Q, without
// the fixed-order quirk), evaluated at the target's bodies (L2P), against the exact P2P
// acceleration from the source's bodies.  The label of (pair, class) is
//   log10( max over target bodies |a_Q - a_exact| / (M_s / r^2) ).
#pragma once
#include "tc_mlp.cuh"
#include "tc_m2l.cuh"
#include "tc_down.cuh"

namespace tc {

// order-Q M2L of 32 sampled pairs per CTA, one pair per lane; L of pair k -> out[k * NTP ..]
template <int P, int Q>
__global__ void __launch_bounds__(128) k_m2l_pairs(int K, const int* __restrict__ pt, const int* __restrict__ ps,
                                                   TcCells c, double* __restrict__ out) {
  constexpr int NTQ = (Q + 1) * (Q + 1), NTP = (P + 1) * (P + 1), G = TcM2LGroups<Q>::G;
  constexpr int CW = TcM2LTmem<Q>::CW;
  constexpr int ALLOC = CW <= 32 ? 32 : CW <= 64 ? 64 : CW <= 128 ? 128 : 256;  // one group
  extern __shared__ double tc_m2lp_smem[];
  __shared__ uint32_t s_tmem;
  double* buf = tc_m2lp_smem;
  double* acc = tc_m2lp_smem + NTQ * 32;  // NTQ x 32 G (columns 0..31 used)
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int k = blockIdx.x * 32 + lane;
  const bool valid = k < K;
  const int t = pt[valid ? k : 0], s = ps[valid ? k : 0];
  if (w == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(&s_tmem)),
                 "r"(ALLOC)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t twarp = s_tmem + ((uint32_t)(32 * w) << 16);
  tc_m2l_zero_warp<Q, false>(w, twarp);
  TcPairGeo pg = tc_pair_geo(c.X[t] - c.X[s], c.Y[t] - c.Y[s], c.Z[t] - c.Z[s]);
  tc_m2l_fwd_warp<Q, false>(w, c.M + (size_t)s * NTP, pg.ez1, pg.ex1, buf, lane, Q);
  __syncthreads();
  tc_m2l_back_warp<Q, false>(w, buf, pg.rinv, lane, pg.ez1, pg.ex1, twarp, valid, Q);
  tc_m2l_readout_warp<Q, false>(w, twarp, acc, lane);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (w == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s_tmem), "r"(ALLOC) : "memory");
  for (int i = 0; i < 32; i++) {
    int kk = blockIdx.x * 32 + i;
    if (kk >= K) break;
    for (int r = threadIdx.x; r < NTP; r += blockDim.x)
      out[(size_t)kk * NTP + r] = r < NTQ ? acc[r * (32 * G) + i] : 0.0;
  }
}

// per pair (one CTA): max relative acceleration error of each class's local expansion; the
// exact acceleration of each target body is computed once and compared with every class
template <int P>
__global__ void __launch_bounds__(128) k_pair_eval(int K, int ncls, const int* __restrict__ pt,
                                                   const int* __restrict__ ps, const TcBodies b, TcCells c,
                                                   const double* __restrict__ pn, const double* __restrict__ Lcls,
                                                   float* __restrict__ logerr) {
  constexpr int NTP = (P + 1) * (P + 1);
  __shared__ cd sl[TC_MAX_CLASSES][NTP];
  __shared__ double sred[TC_MAX_CLASSES][128];
  const int k = blockIdx.x;
  if (k >= K) return;
  const int t = pt[k], s = ps[k];
  const double dxc = c.X[t] - c.X[s], dyc = c.Y[t] - c.Y[s], dzc = c.Z[t] - c.Z[s];
  const double r2c = dxc * dxc + dyc * dyc + dzc * dzc;
  const double amono = fmax(pn[(size_t)s * (P + 1)], 1e-300) / r2c;
  const int tb = c.begin[t], tn = c.nbody[t], sb = c.begin[s], sn = c.nbody[s];
  for (int q = 0; q < ncls; q++) {
    const double* L = Lcls + ((size_t)q * K + k) * NTP;
    for (int i = threadIdx.x; i < NTP; i += blockDim.x) {
      int n = 0;
      while ((n + 1) * (n + 1) <= i) n++;
      sl[q][i] = tc_r2c(L, n, i - n * n - n);
    }
  }
  __syncthreads();
  double emax[TC_MAX_CLASSES];
  for (int q = 0; q < TC_MAX_CLASSES; q++) emax[q] = 0.0;
  for (int i = tb + threadIdx.x; i < tb + tn; i += blockDim.x) {
    double ex = 0, ey = 0, ez = 0;
    for (int j = sb; j < sb + sn; j++) {
      if (!(b.flags[j] & 2)) continue;
      double dx = b.x[j] - b.x[i], dy = b.y[j] - b.y[i], dz = b.z[j] - b.z[i];
      double rr = dx * dx + dy * dy + dz * dz;
      double ri = rsqrt(rr), f = b.m[j] * ri * ri * ri;
      ex += dx * f; ey += dy * f; ez += dz * f;
    }
    for (int q = 0; q < ncls; q++) {
      double a[3];
      tc_l2p_acc<P>(sl[q], c.X[t] - b.x[i], c.Y[t] - b.y[i], c.Z[t] - b.z[i], a);
      double d = sqrt((a[0] - ex) * (a[0] - ex) + (a[1] - ey) * (a[1] - ey) + (a[2] - ez) * (a[2] - ez));
      emax[q] = fmax(emax[q], d);
    }
  }
  for (int q = 0; q < ncls; q++) sred[q][threadIdx.x] = emax[q];
  __syncthreads();
  for (int o = 64; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int q = 0; q < ncls; q++) sred[q][threadIdx.x] = fmax(sred[q][threadIdx.x], sred[q][threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x < ncls) logerr[(size_t)k * ncls + threadIdx.x] = (float)log10(sred[threadIdx.x][0] / amono + 1e-30);
}

// raw features of sampled pairs
template <int P>
__global__ void k_pair_features(int K, const int* __restrict__ pt, const int* __restrict__ ps, TcCells c,
                                const double* __restrict__ pn, float* __restrict__ feat) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  float f[TC_NFEAT];
  tc_pair_features(c, pt[k], ps[k], pn, P, f);
  for (int i = 0; i < TC_NFEAT; i++) feat[(size_t)k * TC_NFEAT + i] = f[i];
}

__global__ void k_gather_pairs(int K, const unsigned long long* __restrict__ keys, const long long* __restrict__ idx,
                               int sbits, int* __restrict__ pt, int* __restrict__ ps) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  unsigned long long key = keys[idx[k]];
  pt[k] = (int)(key >> sbits);
  ps[k] = (int)(key & ((1ull << sbits) - 1ull));
}

}  // namespace tc
