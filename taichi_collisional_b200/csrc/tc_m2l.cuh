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
// Layout: one CTA per target cell, 4 groups of 4 warps (2 at p >= 14); each group takes 32
// (target, source) pairs at a time, one pair per lane.  Warp w of a group owns a fixed set of
// degrees (m2l_schedule.h, balanced by a per-degree cost model) and runs every per-degree
// step -- including the constant swap matrices, emitted as straight-line code with immediate
// coefficients -- in registers.  The only exchange is the z-translation, which mixes
// degrees and goes through shared memory (NT x 32 doubles per group).  Each lane
// accumulates its pairs' locals in its own tensor-memory columns (TcM2LTmem), so shared
// memory holds only the exchange buffers and 16 warps fit on an SM; one fixed-order sum over
// the lanes per coefficient gives deterministic results.  Instruction footprint limits this
// kernel (the code of all degrees exceeds the instruction caches), so each pass applies its
// two swaps through a rolled two-step loop over one copy of the degree's swap code.
#pragma once
#include "swap_tables.h"
#include "tc_harmonics.cuh"
#include "m2l_schedule.h"

namespace tc {

// M2L source lists: bits 0-26 the source cell, bits 27-31 how many orders below the kernel's
// order the pair may be evaluated at (0 = full order; written by the order selectors)
constexpr int kM2LOrderShift = 27;
constexpr int kM2LSrcMask = (1 << kM2LOrderShift) - 1;

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

// the pair's rotation angles and 1/r from two reciprocal square roots (each warp of a group
// computes them for its lanes' pairs, so they stay off the divide and square-root sequences)
__device__ __forceinline__ TcPairGeo tc_pair_geo(double dx, double dy, double dz) {
  TcPairGeo g;
  const double rxy2 = dx * dx + dy * dy;
  g.rinv = rsqrt(rxy2 + dz * dz);
  const double q = rxy2 > 0 ? rsqrt(rxy2) : 0.0;  // 1 / rxy
  const double rxy = rxy2 * q;
  g.ex1 = mk(dz * g.rinv, -rxy * g.rinv);
  g.ez1 = rxy2 > 0 ? mk(dy * q, dx * q) : mk(1, 0);
  return g;
}

// forward half for degree D of an order-Q M2L: scaled, rotated into the pair frame, unscaled
// -> smem.  QUIRK: Q is the expansion order itself, so the (Q, +-Q) entries vanish as in the
// reference.
template <int Q, int D, bool QUIRK>
__device__ __forceinline__ void tc_m2l_fwd(const double* __restrict__ Ms, cd ez1, cd ex1, double* buf, int lane) {
  double v[2 * D + 1], o[2 * D + 1];
#pragma unroll
  for (int k = 0; k < 2 * D + 1; k++) v[k] = __ldg(Ms + D * D + k) * c_fc[D * D + k];
  if (QUIRK && D == Q) {
    v[0] = 0.0;
    v[2 * D] = 0.0;
  }
  // rotate about z, swap, rotate about x, swap: one copy of the swap code, run twice
#pragma unroll 1
  for (int rep = 0; rep < 2; rep++) {
    tc_rot_fwd<D>(v, rep ? ex1 : ez1);
    TcSwapDeg<D>::apply(v, o);
#pragma unroll
    for (int k = 0; k < 2 * D + 1; k++) v[k] = o[k];
  }
#pragma unroll
  for (int k = 0; k < 2 * D + 1; k++) buf[(D * D + k) * 32 + lane] = v[k] * c_fcinv[D * D + k];
}

// translation along z to output degree N, then rotation back; accumulate into the lane's
// column of the shared accumulator.  Factors (n+k)! / r^(n+k+1) are formed on the fly.
// Pair batches processed at once by one CTA (each batch by 4 warps); limited by shared memory.
// Lower orders need less shared memory and tensor memory per group, so they run more groups
// (warps) per SM to hide the latency of their shorter per-batch work: 6 groups at order <= 8,
// 5 at order <= 10 (the most the 512 tensor-memory columns allow), 4 up to 12, 2 above.
template <int P>
struct TcM2LGroups {
  static constexpr int G = (P >= 14) ? 2 : (P <= 8 ? 6 : (P <= 10 ? 5 : 4));
};

// ---------------------------------------------------------------------------------------
// Per-lane accumulators in tensor memory.  Warp w of group g accumulates the locals of the
// degrees it owns for its lane's pairs in TMEM lane 32 (w % 4) + lane (the lane quarter the
// warp may access), columns g * CW + offset of the degree; a double takes two 32-bit columns.
// The allocation base is column-aligned, CW and every degree offset are multiples of 16.
// Shared memory then only holds the translation exchange buffer, which lets more groups
// (warps) share an SM.
// ---------------------------------------------------------------------------------------
template <int Q>
struct TcM2LTmem {
  using S = TcDegSets<Q>;
  // each degree's block starts on a multiple of 16 columns, so the 16/8/4/2-column chunks of
  // tc_tm_ld / tc_tm_st each start on a multiple of their own width
  static constexpr int cols_before(int w, int i) {
    int c = 0;
    for (int k = 0; k < i; k++)
      if (S::d[w][k] >= 0) c += (2 * (2 * S::d[w][k] + 1) + 15) / 16 * 16;
    return c;
  }
  static constexpr int cols_of(int w) { return cols_before(w, S::L); }
  static constexpr int cw_raw() {
    int m = 0;
    for (int w = 0; w < 4; w++) m = cols_of(w) > m ? cols_of(w) : m;
    return m;
  }
  static constexpr int CW = (cw_raw() + 15) / 16 * 16;  // columns per warp, multiple of 16
  static constexpr int TOTAL = CW * TcM2LGroups<Q>::G;
  static constexpr int ALLOC = TOTAL <= 32 ? 32 : TOTAL <= 64 ? 64 : TOTAL <= 128 ? 128 : TOTAL <= 256 ? 256 : 512;
  static_assert(TOTAL <= 512, "M2L accumulators exceed tensor memory");
};

#define TC_TM_R2(i) "=r"(r[(i)]), "=r"(r[(i) + 1])
#define TC_TM_W2(i) "r"(r[(i)]), "r"(r[(i) + 1])
template <int N>
__device__ __forceinline__ void tc_tm_ld_chunk(uint32_t ta, uint32_t* r);
template <int N>
__device__ __forceinline__ void tc_tm_st_chunk(uint32_t ta, const uint32_t* r);
template <>
__device__ __forceinline__ void tc_tm_ld_chunk<2>(uint32_t ta, uint32_t* r) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0,%1}, [%2];" : TC_TM_R2(0) : "r"(ta));
}
template <>
__device__ __forceinline__ void tc_tm_ld_chunk<4>(uint32_t ta, uint32_t* r) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];" : TC_TM_R2(0), TC_TM_R2(2) : "r"(ta));
}
template <>
__device__ __forceinline__ void tc_tm_ld_chunk<8>(uint32_t ta, uint32_t* r) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : TC_TM_R2(0), TC_TM_R2(2), TC_TM_R2(4), TC_TM_R2(6)
               : "r"(ta));
}
template <>
__device__ __forceinline__ void tc_tm_ld_chunk<16>(uint32_t ta, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : TC_TM_R2(0), TC_TM_R2(2), TC_TM_R2(4), TC_TM_R2(6), TC_TM_R2(8), TC_TM_R2(10), TC_TM_R2(12), TC_TM_R2(14)
      : "r"(ta));
}
template <>
__device__ __forceinline__ void tc_tm_st_chunk<2>(uint32_t ta, const uint32_t* r) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1,%2};" ::"r"(ta), TC_TM_W2(0) : "memory");
}
template <>
__device__ __forceinline__ void tc_tm_st_chunk<4>(uint32_t ta, const uint32_t* r) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1,%2,%3,%4};" ::"r"(ta), TC_TM_W2(0), TC_TM_W2(2)
               : "memory");
}
template <>
__device__ __forceinline__ void tc_tm_st_chunk<8>(uint32_t ta, const uint32_t* r) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(ta), TC_TM_W2(0),
               TC_TM_W2(2), TC_TM_W2(4), TC_TM_W2(6)
               : "memory");
}
template <>
__device__ __forceinline__ void tc_tm_st_chunk<16>(uint32_t ta, const uint32_t* r) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
          ta),
      TC_TM_W2(0), TC_TM_W2(2), TC_TM_W2(4), TC_TM_W2(6), TC_TM_W2(8), TC_TM_W2(10), TC_TM_W2(12), TC_TM_W2(14)
      : "memory");
}
#undef TC_TM_R2
#undef TC_TM_W2

// C (even) consecutive columns, as chunks of 16, 8, 4, 2; loads complete at tc_tm_wait_ld
template <int C, int OFF = 0>
__device__ __forceinline__ void tc_tm_ld(uint32_t ta, uint32_t* r) {
  if constexpr (C >= 16) {
    tc_tm_ld_chunk<16>(ta + OFF, r + OFF);
    tc_tm_ld<C - 16, OFF + 16>(ta, r);
  } else if constexpr (C >= 8) {
    tc_tm_ld_chunk<8>(ta + OFF, r + OFF);
    tc_tm_ld<C - 8, OFF + 8>(ta, r);
  } else if constexpr (C >= 4) {
    tc_tm_ld_chunk<4>(ta + OFF, r + OFF);
    tc_tm_ld<C - 4, OFF + 4>(ta, r);
  } else if constexpr (C >= 2) {
    tc_tm_ld_chunk<2>(ta + OFF, r + OFF);
  }
}
template <int C, int OFF = 0>
__device__ __forceinline__ void tc_tm_st(uint32_t ta, const uint32_t* r) {
  if constexpr (C >= 16) {
    tc_tm_st_chunk<16>(ta + OFF, r + OFF);
    tc_tm_st<C - 16, OFF + 16>(ta, r);
  } else if constexpr (C >= 8) {
    tc_tm_st_chunk<8>(ta + OFF, r + OFF);
    tc_tm_st<C - 8, OFF + 8>(ta, r);
  } else if constexpr (C >= 4) {
    tc_tm_st_chunk<4>(ta + OFF, r + OFF);
    tc_tm_st<C - 4, OFF + 4>(ta, r);
  } else if constexpr (C >= 2) {
    tc_tm_st_chunk<2>(ta + OFF, r + OFF);
  }
}
__device__ __forceinline__ void tc_tm_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_tm_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// the 2 K columns of K doubles -> registers (after tc_tm_ld and tc_tm_wait_ld)
template <int K>
__device__ __forceinline__ void tc_tm_to_f64(uint32_t* r, double* v) {
#pragma unroll
  for (int k = 0; k < K; k++) {
    asm volatile("" : "+r"(r[2 * k]), "+r"(r[2 * k + 1]));  // every use stays after the wait
    v[k] = __hiloint2double((int)r[2 * k + 1], (int)r[2 * k]);
  }
}

// qb (<= P): the batch's expansion order -- translation terms with n + k > qb are left out, as an
// order-qb M2L does (the caller skips output degrees N > qb)
template <int P, int N>
__device__ __forceinline__ void tc_m2l_back(const double* buf, double rinv, int lane, cd ez1, cd ex1,
                                            uint32_t tacc, bool valid, int qb) {
  double l[2 * N + 1], o[2 * N + 1];
#pragma unroll
  for (int k = 0; k < 2 * N + 1; k++) l[k] = 0.0;
  double pn = rinv;
#pragma unroll
  for (int j = 0; j < N; j++) pn *= rinv;  // rinv^(N+1)
  // the k loops stay rolled: the translation is a quarter of the unrolled code otherwise
  {
    double s = 0.0, pr = pn;
#pragma unroll 1
    for (int k = 0; k <= qb - N; k++) {
      s += buf[(k * k + k) * 32 + lane] * (c_fact[N + k] * pr);
      pr *= rinv;
    }
    l[N] = s;
  }
  constexpr int MMAX = N < P - N ? N : P - N;
  double pm = rinv;
#pragma unroll
  for (int m = 1; m <= MMAX; m++) {
    double sn = 0.0, sp = 0.0, pr = pn * pm;
#pragma unroll 1
    for (int k = m; k <= qb - N; k++) {
      const double f = c_fact[N + k] * pr;
      const int b = (k * k + k) * 32 + lane;
      sn += buf[b - m * 32] * f;
      sp += buf[b + m * 32] * f;
      pr *= rinv;
    }
    const double sg = (m & 1) ? -1.0 : 1.0;
    l[N - m] = sg * sn;
    l[N + m] = sg * sp;
    pm *= rinv;
  }
  // swap, rotate back about x, swap, rotate back about z: one copy of the swap code, run twice
#pragma unroll 1
  for (int rep = 0; rep < 2; rep++) {
    TcSwapDeg<N>::apply(l, o);
    tc_rot_inv<N>(o, rep ? ez1 : ex1);
#pragma unroll
    for (int k = 0; k < 2 * N + 1; k++) l[k] = o[k];
  }
  // read-modify-write of this lane's accumulator columns (every lane takes part)
  uint32_t r[2 * (2 * N + 1)];
  double a[2 * N + 1];
  tc_tm_ld<2 * (2 * N + 1)>(tacc, r);
  tc_tm_wait_ld();
  tc_tm_to_f64<2 * N + 1>(r, a);
#pragma unroll
  for (int k = 0; k < 2 * N + 1; k++) {
    const double v = a[k] + (valid ? l[k] : 0.0);
    r[2 * k] = (uint32_t)__double2loint(v);
    r[2 * k + 1] = (uint32_t)__double2hiint(v);
  }
  tc_tm_st<2 * (2 * N + 1)>(tacc, r);
}

// shared-memory layout of one M2L CTA (doubles): buf[G groups]; after the last batch the same
// space holds the accumulators of all 32 G lanes for the ordered final sum
template <int P>
struct TcM2LSmem {
  static constexpr int NT = (P + 1) * (P + 1);
  static constexpr int G = TcM2LGroups<P>::G;
  static constexpr int BUF = 0;
  static constexpr int TOTAL = G * NT * 32;
};

// Warp w of each 4-warp group owns the degrees TcDegSets<P>::d[w][*] (balanced by a
// per-degree cost model) for the group's 32 pairs; warps w and w + 4 run the same degree code,
// which keeps each SM sub-partition's instruction working set to one degree set.
template <int Q, bool QUIRK, int W, int I>
struct TcDegSeq {
  static constexpr int D = TcDegSets<Q>::d[W][I];
  static __device__ __forceinline__ void fwd(const double* Ms, cd ez1, cd ex1, double* buf, int lane, int qb) {
    if constexpr (D >= 0) {
      if (D <= qb) tc_m2l_fwd<Q, D, QUIRK>(Ms, ez1, ex1, buf, lane);
      TcDegSeq<Q, QUIRK, W, I + 1>::fwd(Ms, ez1, ex1, buf, lane, qb);
    }
  }
  static constexpr int COL = TcM2LTmem<Q>::cols_before(W, I);
  static __device__ __forceinline__ void back(const double* buf, double rinv, int lane, cd ez1, cd ex1,
                                              uint32_t twarp, bool valid, int qb) {
    if constexpr (D >= 0) {
      if (D <= qb) tc_m2l_back<Q, D>(buf, rinv, lane, ez1, ex1, twarp + COL, valid, qb);
      TcDegSeq<Q, QUIRK, W, I + 1>::back(buf, rinv, lane, ez1, ex1, twarp, valid, qb);
    }
  }
  // zero this warp's accumulator columns
  static __device__ __forceinline__ void zero(uint32_t twarp) {
    if constexpr (D >= 0) {
      uint32_t z[2 * (2 * D + 1)];
#pragma unroll
      for (int k = 0; k < 2 * (2 * D + 1); k++) z[k] = 0u;
      tc_tm_st<2 * (2 * D + 1)>(twarp + COL, z);
      TcDegSeq<Q, QUIRK, W, I + 1>::zero(twarp);
    }
  }
  // accumulators -> shared memory, row (coefficient) major with 32 G columns
  static __device__ __forceinline__ void readout(uint32_t twarp, double* sc, int acol) {
    if constexpr (D >= 0) {
      uint32_t r[2 * (2 * D + 1)];
      double a[2 * D + 1];
      tc_tm_ld<2 * (2 * D + 1)>(twarp + COL, r);
      tc_tm_wait_ld();
      tc_tm_to_f64<2 * D + 1>(r, a);
#pragma unroll
      for (int k = 0; k < 2 * D + 1; k++) sc[(D * D + k) * (32 * TcM2LGroups<Q>::G) + acol] = a[k];
      TcDegSeq<Q, QUIRK, W, I + 1>::readout(twarp, sc, acol);
    }
  }
};

template <int Q, bool QUIRK>
__device__ __forceinline__ void tc_m2l_fwd_warp(int w, const double* Ms, cd ez1, cd ex1, double* buf, int lane,
                                                int qb) {
  if (w == 0) TcDegSeq<Q, QUIRK, 0, 0>::fwd(Ms, ez1, ex1, buf, lane, qb);
  else if (w == 1) TcDegSeq<Q, QUIRK, 1, 0>::fwd(Ms, ez1, ex1, buf, lane, qb);
  else if (w == 2) TcDegSeq<Q, QUIRK, 2, 0>::fwd(Ms, ez1, ex1, buf, lane, qb);
  else TcDegSeq<Q, QUIRK, 3, 0>::fwd(Ms, ez1, ex1, buf, lane, qb);
}
template <int Q, bool QUIRK>
__device__ __forceinline__ void tc_m2l_back_warp(int w, const double* buf, double rinv, int lane, cd ez1, cd ex1,
                                                 uint32_t twarp, bool valid, int qb) {
  tc_tm_wait_st();  // the previous batch's accumulator stores
  if (w == 0) TcDegSeq<Q, QUIRK, 0, 0>::back(buf, rinv, lane, ez1, ex1, twarp, valid, qb);
  else if (w == 1) TcDegSeq<Q, QUIRK, 1, 0>::back(buf, rinv, lane, ez1, ex1, twarp, valid, qb);
  else if (w == 2) TcDegSeq<Q, QUIRK, 2, 0>::back(buf, rinv, lane, ez1, ex1, twarp, valid, qb);
  else TcDegSeq<Q, QUIRK, 3, 0>::back(buf, rinv, lane, ez1, ex1, twarp, valid, qb);
}
template <int Q, bool QUIRK>
__device__ __forceinline__ void tc_m2l_zero_warp(int w, uint32_t twarp) {
  if (w == 0) TcDegSeq<Q, QUIRK, 0, 0>::zero(twarp);
  else if (w == 1) TcDegSeq<Q, QUIRK, 1, 0>::zero(twarp);
  else if (w == 2) TcDegSeq<Q, QUIRK, 2, 0>::zero(twarp);
  else TcDegSeq<Q, QUIRK, 3, 0>::zero(twarp);
}
template <int Q, bool QUIRK>
__device__ __forceinline__ void tc_m2l_readout_warp(int w, uint32_t twarp, double* sc, int acol) {
  tc_tm_wait_st();
  if (w == 0) TcDegSeq<Q, QUIRK, 0, 0>::readout(twarp, sc, acol);
  else if (w == 1) TcDegSeq<Q, QUIRK, 1, 0>::readout(twarp, sc, acol);
  else if (w == 2) TcDegSeq<Q, QUIRK, 2, 0>::readout(twarp, sc, acol);
  else TcDegSeq<Q, QUIRK, 3, 0>::readout(twarp, sc, acol);
}

__device__ __forceinline__ void tc_bar_group(int grp) {
  asm volatile("bar.sync %0, 128;" ::"r"(2 + grp) : "memory");
}

template <int Q>
constexpr int tc_m2l_threads() { return 128 * TcM2LGroups<Q>::G; }

// M2L of order Q <= P over a per-target list (or, with `tend`, one order class's range of it);
// expansions are stored with order P.  Adds into L (zeroed before the first M2L launch of an
// evaluation).  One CTA per SM (shared
// memory), which owns the tensor memory it allocates.  One target per CTA, or, with `next`
// (a counter zeroed before the launch), a persistent grid whose CTAs take targets in turn.
template <int P, int Q, bool JERK>
__global__ void __launch_bounds__(tc_m2l_threads<Q>(), 1) k_m2l(const int* __restrict__ tlist, int ntl,
                                                               const int* __restrict__ tstart,
                                                               const int* __restrict__ src, TcCells c,
                                                               const unsigned* ntldev = nullptr,
                                                               unsigned* next = nullptr,
                                                               const int* __restrict__ tend = nullptr) {
  using SM = TcM2LSmem<Q>;
  using TM = TcM2LTmem<Q>;
  constexpr int NTQ = SM::NT, NTP = (P + 1) * (P + 1);
  constexpr int G = SM::G;
  constexpr bool QUIRK = Q == P;
  extern __shared__ double tc_m2l_smem[];
  __shared__ uint32_t s_tmem;
  __shared__ int s_ti;
  int ti = blockIdx.x;
  if (ntldev) ntl = (int)*ntldev;  // device-sized launch (graph)
  if (next) {
    if (threadIdx.x == 0) s_ti = (int)atomicAdd(next, 1u);
    __syncthreads();
    ti = s_ti;
  }
  if (ti >= ntl) return;
  if (!next && !c.has_sink[tlist[ti]]) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = warp >> 2, w = warp & 3, acol = grp * 32 + lane;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(&s_tmem)),
                 "r"(TM::ALLOC)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  tc_bar_cta();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  // this warp's columns in its lane quarter
  const uint32_t twarp = s_tmem + ((uint32_t)(32 * w) << 16) + (uint32_t)(grp * TM::CW);
  double* buf = tc_m2l_smem + SM::BUF + grp * NTQ * 32;
  for (;;) {
  const int t = tlist[ti];
  // the target's sources: [tstart[t], tstart[t + 1]), or one order class's range of them
  const int s_beg = tstart[t], s_end = tend ? tend[t] : tstart[t + 1];
  const double Xt = c.X[t], Yt = c.Y[t], Zt = c.Z[t];
  for (int arr = 0; arr < (c.has_sink[t] && s_end > s_beg ? (JERK ? 2 : 1) : 0); arr++) {
    const double* Mbase = arr ? c.Md : c.M;
    tc_m2l_zero_warp<Q, QUIRK>(w, twarp);
    for (int b0 = s_beg + grp * 32; b0 < s_end; b0 += 32 * G) {
      int idx = b0 + lane;
      bool valid = idx < s_end;
      // a source entry carries its pair's order below Q in its top bits (tc_m2l_src_order); the
      // batch runs at the largest order of its pairs, a lower order never applied to a pair
      const int sv = src[valid ? idx : s_beg];
      const int s = sv & kM2LSrcMask;
      const int qb = Q - (int)__reduce_min_sync(0xffffffffu, valid ? (unsigned)sv >> kM2LOrderShift : 31u);
      TcPairGeo pg = tc_pair_geo(Xt - c.X[s], Yt - c.Y[s], Zt - c.Z[s]);
      tc_m2l_fwd_warp<Q, QUIRK>(w, Mbase + (size_t)s * NTP, pg.ez1, pg.ex1, buf, lane, qb);
      tc_bar_group(grp);
      tc_m2l_back_warp<Q, QUIRK>(w, buf, pg.rinv, lane, pg.ez1, pg.ex1, twarp, valid, qb);
      tc_bar_group(grp);
    }
    tc_bar_cta();  // every group is done with its buffer
    double* sc = tc_m2l_smem;  // NT x 32 G accumulators
    tc_m2l_readout_warp<Q, QUIRK>(w, twarp, sc, acol);
    tc_bar_cta();
    // ordered sum over the 32 G lanes of each coefficient: warp per coefficient, lane j adds
    // columns j, j + 32, ... in order, then a fixed butterfly over the lanes
    double* Lt = (arr ? c.Ld : c.L) + (size_t)t * NTP;
    for (int r = warp; r < NTQ; r += 4 * G) {
      double v = 0.0;
#pragma unroll
      for (int q = 0; q < G; q++) v += sc[r * (32 * G) + 32 * q + lane];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) Lt[r] += v;
    }
    tc_bar_cta();
  }
  if (!next) break;
  if (threadIdx.x == 0) s_ti = (int)atomicAdd(next, 1u);
  tc_bar_cta();
  ti = s_ti;
  tc_bar_cta();
  if (ti >= ntl) break;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  tc_bar_cta();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s_tmem), "r"(TM::ALLOC) : "memory");
}

}  // namespace tc
