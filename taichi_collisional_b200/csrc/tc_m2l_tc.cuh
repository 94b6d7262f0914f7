// Tensor-core rotation M2L: the constant contractions on tcgen05 (TF32 pieces, FP32
// accumulation in tensor memory), the per-pair phase rotations on the CUDA cores in FP32.
//
// Same algorithm as tc_m2l_mixed.cuh (orthonormal scaling w = M F / r^n, rotate about z,
// swap x<->z, rotate about x, swap, translate along z, and back), restating M2L_rotate
// (taichi_with_jerks/kernel_fast_lean.h:1130-1371).  A tile of 128 (target, source) pairs
// is one 128-row matrix, one row per thread:
//   * the four swaps and the translation are products with constant block-diagonal
//     16 x 16 bins (plan in m2l_tc_plan.h): a swap "super-bin" holds two complete degrees,
//     real parts in one 16-column half and imaginary parts in the other (the swap never
//     mixes them), the second degree stored from the far end so that the order m of a
//     position is i, 15 - i or 0 in every super-bin -- one compact loop body serves them
//     all; each half is one tcgen05.mma.kind::tf32, M = 128, N = 16, two K steps of 8;
//   * FP32 accuracy from TF32 operands: a row value x = hi + mid + lo (three TF32 pieces,
//     33 significant bits) and a matrix entry b = hi + lo;
//       x b ~ lo b_hi + mid b_hi + hi b_lo + hi b_hi,
//     every dropped term is below 2^-30 of x b;
//   * hi and mid rows live in shared memory (canonical K-major layout, no swizzle: 8-row x
//     16-byte core matrices), lo rows in tensor memory (the A-from-tensor-memory form of
//     the MMA), the products in tensor memory, lane = pair row; each thread reads its row
//     back with tcgen05.ld one super-bin (32 columns) at a time, rotates it and writes the
//     next row; per-tile tables (phases e^{i m a}, r^-n, (r/r_ref)^-(n+1)) sit in spare
//     tensor-memory columns;
//   * per target, the rows are summed in FP64 (a warp butterfly and a 4-warp pass); each
//     row is scaled relative to the tile's largest 1/r first, so that the r^-(n+1)
//     factors stay inside the FP32 range.
// One persistent CTA of 128 threads per SM takes whole targets from a counter, so every
// target's sum is formed in a fixed order (results do not depend on scheduling).
#pragma once
#include "tc_m2l_mixed.cuh"
#include "m2l_tc_plan.h"

namespace tc {

// ---------------------------------------------------------------------------------------
// PTX wrappers (tcgen05, mbarrier, TF32 rounding)
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t tc_smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, no swizzle: start, leading (K-direction core matrix)
// byte offset, stride (8-row group) byte offset, descriptor version 1
__device__ __forceinline__ unsigned long long tc_umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  unsigned long long d = (unsigned long long)((saddr >> 4) & 0x3FFFu);
  d |= (unsigned long long)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (unsigned long long)((sbo >> 4) & 0x3FFFu) << 32;
  d |= 1ull << 46;
  return d;
}

// instruction descriptor: D f32, A and B tf32, both K-major, N = 16, M = 128
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void tc_mma_tf32(uint32_t dtmem, unsigned long long ad, unsigned long long bd,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
      "l"(ad), "l"(bd), "r"(kTcIdesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void tc_mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void tc_mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

// default limit of a bounded wait: ~2 s of device clock
constexpr long long kTcWaitLimit = 4000000000ll;

// bounded wait for the phase with the given parity; false after `limit` cycles of device clock
__device__ __forceinline__ bool tc_mbar_wait(uint32_t mbar, uint32_t parity, long long limit = kTcWaitLimit) {
  long long t0 = clock64();
  for (;;) {
    if (clock64() - t0 > limit) return false;  // checked first: a limit of a few cycles always runs out
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
}

__device__ __forceinline__ void tc_fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ float tc_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// NCOL (multiple of 16) consecutive tensor-memory columns of this thread's lane
template <int NCOL>
__device__ __forceinline__ void tc_tmem_ld(uint32_t taddr, float* d) {
  uint32_t r[NCOL];
#pragma unroll
  for (int b = 0; b < NCOL / 16; b++) {
    uint32_t* q = r + 16 * b;
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(q[0]), "=r"(q[1]), "=r"(q[2]), "=r"(q[3]), "=r"(q[4]), "=r"(q[5]), "=r"(q[6]), "=r"(q[7]),
          "=r"(q[8]), "=r"(q[9]), "=r"(q[10]), "=r"(q[11]), "=r"(q[12]), "=r"(q[13]), "=r"(q[14]), "=r"(q[15])
        : "r"(taddr + 16u * b));
  }
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < NCOL; i++) {
    asm volatile("" : "+r"(r[i]));  // keeps every use after the wait
    d[i] = __uint_as_float(r[i]);
  }
}

// ---------------------------------------------------------------------------------------
// more PTX wrappers: the A-from-tensor-memory MMA, tensor-memory stores and small loads
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void tc_mma_tf32_ts(uint32_t dtmem, uint32_t atmem, unsigned long long bd,
                                               uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(dtmem),
      "r"(atmem), "l"(bd), "r"(kTcIdesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void tc_tmem_st16(uint32_t taddr, const float* v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
          taddr),
      "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]), "f"(v[8]), "f"(v[9]),
      "f"(v[10]), "f"(v[11]), "f"(v[12]), "f"(v[13]), "f"(v[14]), "f"(v[15])
      : "memory");
}
__device__ __forceinline__ void tc_tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// one column (issue only; the value is valid after tc_tmem_wait_ld)
__device__ __forceinline__ uint32_t tc_tmem_ld1_issue(uint32_t taddr) {
  uint32_t r;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr));
  return r;
}
__device__ __forceinline__ void tc_tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---------------------------------------------------------------------------------------
// layout: shared memory and tensor-memory columns
// ---------------------------------------------------------------------------------------
template <int Q>
struct TcTcSmem {
  using PL = TcTcPlan<Q>;
  static constexpr int SBO_A = (PL::AW / 4) * 128;  // bytes between 8-row groups of A
  static constexpr int A_BYTES = 16 * SBO_A;        // 128 rows, one TF32 piece
  static constexpr int BIN_BYTES = 16 * 16 * 4;     // one 16 x 16 bin matrix
  static constexpr int NBIN = PL::NH + PL::NTB;
  static constexpr int B_BYTES = NBIN * BIN_BYTES;  // all bins, hi or lo
  static constexpr int OFF_AHI = 0, OFF_AMID = A_BYTES, OFF_BHI = 2 * A_BYTES, OFF_BLO = OFF_BHI + B_BYTES;
  static constexpr int OFF_MISC = OFF_BLO + B_BYTES;  // mbarrier, tmem base, next target, warp maxima
  // at least ~116 KB, so that a second CTA (and its tensor-memory allocation) never shares the SM
  static constexpr int TOTAL = (OFF_MISC + 128) > 120000 ? (OFF_MISC + 128) : 120000;
  static_assert(4 * PL::AW * 8 <= A_BYTES, "per-warp row sums reuse the hi rows");
  static_assert(PL::TW <= PL::AW, "translation columns inside the row");
};
// tensor-memory columns (512 allocated): products | lo rows | phases | r^-n (FP64) | q^(n+1)
constexpr uint32_t kTcColD = 0, kTcColLo = 192, kTcColPh = 384, kTcColRn = 448, kTcColQn = 480, kTcCols = 512;

// the bin matrices (hi bins then lo bins) in the canonical layout: element (n, k) of a bin
// (n = output column, k = input column) at float (n/8)*128 + (k/4)*32 + (n%8)*4 + k%4
__host__ __device__ inline int tc_tc_bin_index(int n, int k) {
  return (n >> 3) * 128 + (k >> 2) * 32 + (n & 7) * 4 + (k & 3);
}

// ---------------------------------------------------------------------------------------
// row pieces
// ---------------------------------------------------------------------------------------
// 16 values -> columns [col, col + 16) of this thread's row: hi and mid pieces to shared
// memory (ah, am point at the row's first chunk), lo piece to tensor memory (tl = lane base)
__device__ __forceinline__ void tc_tc_put16(char* ah, char* am, uint32_t tl, int col, const float* x) {
  float lo[16];
#pragma unroll
  for (int c = 0; c < 4; c++) {
    float h[4], m[4];
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const float v = x[4 * c + e];
      h[e] = tc_tf32(v);
      const float r = v - h[e];
      m[e] = tc_tf32(r);
      lo[4 * c + e] = tc_tf32(r - m[e]);
    }
    const int off = ((col >> 2) + c) * 128;
    *reinterpret_cast<float4*>(ah + off) = make_float4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<float4*>(am + off) = make_float4(m[0], m[1], m[2], m[3]);
  }
  tc_tmem_st16(tl + kTcColLo + (uint32_t)col, lo);
}

// phase of position i in a super-bin (D1, D2): order i (first degree), 15 - i (second) or 0
__device__ __forceinline__ void tc_tc_phase(int i, int d1, int d2, const float* pc, const float* ps, float& c,
                                            float& s) {
  const bool a = i <= d1, b = i >= 15 - d2;
  c = a ? pc[i] : (b ? pc[15 - i] : 1.f);
  s = a ? ps[i] : (b ? ps[15 - i] : 0.f);
}

// rotate the super-bin's (Im, Re) pairs by its positions' phases (INV: the inverse)
template <bool INV>
__device__ __forceinline__ void tc_tc_rot16(float* xr, float* xi, int d1, int d2, const float* pc, const float* ps) {
#pragma unroll
  for (int i = 0; i < 16; i++) {
    float c, s;
    tc_tc_phase(i, d1, d2, pc, ps, c, s);
    if (INV) s = -s;
    const float im = xi[i], re = xr[i];
    xi[i] = c * im + s * re;
    xr[i] = c * re - s * im;
  }
}

// the 16 phases (cos, sin of m a, m = 0..15) of one angle from tensor memory
__device__ __forceinline__ void tc_tc_phases(uint32_t tl, int angle, float* pc, float* ps) {
  float t[32];
  tc_tmem_ld<32>(tl + kTcColPh + 32u * angle, t);
#pragma unroll
  for (int i = 0; i < 16; i++) {
    pc[i] = t[i];
    ps[i] = t[16 + i];
  }
}

__device__ __forceinline__ void tc_tc_seq() { asm volatile("" ::: "memory"); }

// sum of x[i] over the warp's 32 lanes, for every i; lane l receives the sum of x[l]
__device__ __forceinline__ float tc_tc_butterfly32(float* x, int lane) {
#pragma unroll
  for (int s = 0; s < 5; s++) {
    const int bit = 16 >> s;
    const bool up = (lane & bit) != 0;
#pragma unroll
    for (int j = 0; j < bit; j++) {
      const float send = up ? x[j] : x[j + bit];
      const float keep = up ? x[j + bit] : x[j];
      x[j] = keep + __shfl_xor_sync(0xffffffffu, send, bit);
    }
  }
  return x[0];
}

// the same in FP64 (the per-tile sums over 128 pairs cancel strongly; FP32 would cost
// accuracy there)
__device__ __forceinline__ double tc_tc_butterfly32d(double* x, int lane) {
#pragma unroll
  for (int s = 0; s < 5; s++) {
    const int bit = 16 >> s;
    const bool up = (lane & bit) != 0;
#pragma unroll
    for (int j = 0; j < bit; j++) {
      const double send = up ? x[j] : x[j + bit];
      const double keep = up ? x[j + bit] : x[j];
      x[j] = keep + __shfl_xor_sync(0xffffffffu, send, bit);
    }
  }
  return x[0];
}

// ---------------------------------------------------------------------------------------
// pipeline stages (one thread = one row)
// ---------------------------------------------------------------------------------------
// multipoles (FP64, global) -> w = M F r^-n in FP32 -> rotate about z -> row
template <int Q>
__device__ __forceinline__ void tc_tc_f0(const double* Ms, bool valid, bool quirk, uint32_t tl, char* ah, char* am) {
  using PL = TcTcPlan<Q>;
  float pc[16], ps[16];
  tc_tc_phases(tl, 0, pc, ps);
#pragma unroll 1
  for (int s = 0; s < PL::NSB; s++) {
    const int d1 = PL::sb_d1(s), d2 = PL::sb_d2(s), z = PL::sb_zero(s);
    const int dd2 = d2 > 0 ? d2 : 0;
    uint32_t r1a = tc_tmem_ld1_issue(tl + kTcColRn + 2 * d1), r1b = tc_tmem_ld1_issue(tl + kTcColRn + 2 * d1 + 1);
    uint32_t r2a = tc_tmem_ld1_issue(tl + kTcColRn + 2 * dd2), r2b = tc_tmem_ld1_issue(tl + kTcColRn + 2 * dd2 + 1);
    tc_tmem_wait_ld();
    asm volatile("" : "+r"(r1a), "+r"(r1b), "+r"(r2a), "+r"(r2b));
    const double rn1 = __hiloint2double((int)r1b, (int)r1a), rn2 = __hiloint2double((int)r2b, (int)r2a);
    // every position's coefficient index, branch-free, so that all 32 loads are in flight
    // together (empty positions read coefficient 0 and are zeroed below)
    double vr[16], vi[16];
#pragma unroll
    for (int i = 0; i < 16; i++) {
      const bool a = i <= d1, b = i >= 15 - d2;
      const int n = a ? d1 : (b ? d2 : 0);
      const int m = a ? i : (b ? 15 - i : 0);
      const int k = n * n + n + m;
      vr[i] = Ms[k];
      vi[i] = Ms[k - 2 * m];
    }
    float xr[16], xi[16];
#pragma unroll
    for (int i = 0; i < 16; i++) {
      const bool a = i <= d1, b = i >= 15 - d2, c0 = z && i == d1 + 1;
      const int n = a ? d1 : (b ? d2 : 0);
      const int m = a ? i : (b ? 15 - i : 0);
      const int k = n * n + n + m;
      const double rn = a ? rn1 : (b ? rn2 : 1.0);
      const bool live = valid && (a || b || c0);
      xr[i] = live ? (float)((vr[i] * c_mF[k]) * rn) : 0.f;
      xi[i] = (live && m > 0) ? (float)((vi[i] * c_mF[k - 2 * m]) * rn) : 0.f;
    }
    if (quirk && d1 == Q) {  // the (Q, +-Q) multipole entries vanish as in the reference
      xr[Q] = 0.f;
      xi[Q] = 0.f;
    }
    tc_tc_rot16<false>(xr, xi, d1, d2, pc, ps);
    tc_tc_put16(ah, am, tl, 32 * s, xr);
    tc_tc_put16(ah, am, tl, 32 * s + 16, xi);
    tc_tc_seq();
  }
}

// products -> rotate (angle 0: z, 1: x) -> row
template <int Q, bool INV>
__device__ __forceinline__ void tc_tc_rot_stage(int angle, uint32_t tl, char* ah, char* am) {
  using PL = TcTcPlan<Q>;
  float pc[16], ps[16];
  tc_tc_phases(tl, angle, pc, ps);
#pragma unroll 1
  for (int s = 0; s < PL::NSB; s++) {
    const int d1 = PL::sb_d1(s), d2 = PL::sb_d2(s);
    float x[32];
    tc_tmem_ld<32>(tl + kTcColD + 32u * s, x);
    tc_tc_rot16<INV>(x, x + 16, d1, d2, pc, ps);
    tc_tc_put16(ah, am, tl, 32 * s, x);
    tc_tc_put16(ah, am, tl, 32 * s + 16, x + 16);
    tc_tc_seq();
  }
}

// swap products -> translation row (gather by column)
template <int Q>
__device__ __forceinline__ void tc_tc_f2(uint32_t tl, char* ah, char* am) {
  using PL = TcTcPlan<Q>;
#pragma unroll 1
  for (int h = 0; h < PL::TW / 16; h++) {
    uint32_t r[16];
#pragma unroll
    for (int j = 0; j < 16; j++) {
      const int k = PL::t_nat(16 * h + j);
      r[j] = tc_tmem_ld1_issue(tl + kTcColD + PL::d_col(k >= 0 ? k : 0));
    }
    tc_tmem_wait_ld();
    float x[16];
#pragma unroll
    for (int j = 0; j < 16; j++) {
      asm volatile("" : "+r"(r[j]));
      x[j] = PL::t_nat(16 * h + j) >= 0 ? __uint_as_float(r[j]) : 0.f;
    }
    tc_tc_put16(ah, am, tl, 16 * h, x);
    tc_tc_seq();
  }
}

// translation products -> swap row (gather by column; |m| > min(n, Q - n) stays zero)
template <int Q>
__device__ __forceinline__ void tc_tc_b0(uint32_t tl, char* ah, char* am) {
  using PL = TcTcPlan<Q>;
#pragma unroll 1
  for (int h = 0; h < PL::NH; h++) {
    uint32_t r[16];
#pragma unroll
    for (int j = 0; j < 16; j++) {
      const int k = PL::d_nat(16 * h + j);
      const int c = k >= 0 ? PL::t_col(k) : -1;
      r[j] = tc_tmem_ld1_issue(tl + kTcColD + (c >= 0 ? c : 0));
    }
    tc_tmem_wait_ld();
    float x[16];
#pragma unroll
    for (int j = 0; j < 16; j++) {
      asm volatile("" : "+r"(r[j]));
      const int k = PL::d_nat(16 * h + j);
      x[j] = (k >= 0 && PL::t_col(k) >= 0) ? __uint_as_float(r[j]) : 0.f;
    }
    tc_tc_put16(ah, am, tl, 16 * h, x);
    tc_tc_seq();
  }
}

// products -> rotate back about z -> scale by (r / r_ref)^-(n+1) -> per-warp column sums
template <int Q>
__device__ __forceinline__ void tc_tc_b2(uint32_t tl, double* red, int lane) {
  using PL = TcTcPlan<Q>;
  float pc[16], ps[16];
  tc_tc_phases(tl, 0, pc, ps);
#pragma unroll 1
  for (int s = 0; s < PL::NSB; s++) {
    const int d1 = PL::sb_d1(s), d2 = PL::sb_d2(s), z = PL::sb_zero(s);
    uint32_t q1 = tc_tmem_ld1_issue(tl + kTcColQn + d1), q2 = tc_tmem_ld1_issue(tl + kTcColQn + (d2 > 0 ? d2 : 0)),
             q0 = tc_tmem_ld1_issue(tl + kTcColQn);
    float x[32];
    tc_tmem_ld<32>(tl + kTcColD + 32u * s, x);  // its wait covers the three loads above
    asm volatile("" : "+r"(q1), "+r"(q2), "+r"(q0));
    const float qn1 = __uint_as_float(q1), qn2 = __uint_as_float(q2), qn0 = __uint_as_float(q0);
    tc_tc_rot16<true>(x, x + 16, d1, d2, pc, ps);
    double xd[32];
#pragma unroll
    for (int i = 0; i < 16; i++) {
      const float f = i <= d1 ? qn1 : (i >= 15 - d2 ? qn2 : ((z && i == d1 + 1) ? qn0 : 0.f));
      xd[i] = (double)(x[i] * f);
      xd[16 + i] = (double)(x[16 + i] * f);
    }
    red[32 * s + lane] = tc_tc_butterfly32d(xd, lane);
    tc_tc_seq();
  }
}

// ---------------------------------------------------------------------------------------
// MMA issue (one thread)
// ---------------------------------------------------------------------------------------
// lo B_hi + mid B_hi + hi B_lo + hi B_hi into the 128 x 16 product at tensor column dcol;
// row columns [acol, acol + 16), bin matrix `bin`
template <int Q>
__device__ __forceinline__ void tc_tc_mma_half(uint32_t tmem, uint32_t ahi, uint32_t amid, uint32_t bhi,
                                               uint32_t blo, int acol, int bin, int dcol) {
  using SM = TcTcSmem<Q>;
#pragma unroll
  for (int j = 0; j < 2; j++) {
    const uint32_t ao = (uint32_t)((acol >> 2) + 2 * j) * 128u;
    const uint32_t bo = (uint32_t)bin * SM::BIN_BYTES + 256u * j;
    const unsigned long long a_h = tc_umma_desc(ahi + ao, 128, SM::SBO_A);
    const unsigned long long a_m = tc_umma_desc(amid + ao, 128, SM::SBO_A);
    const unsigned long long b_h = tc_umma_desc(bhi + bo, 128, 512);
    const unsigned long long b_l = tc_umma_desc(blo + bo, 128, 512);
    const uint32_t d = tmem + kTcColD + (uint32_t)dcol;
    tc_mma_tf32_ts(d, tmem + kTcColLo + (uint32_t)(acol + 8 * j), b_h, j);
    tc_mma_tf32(d, a_m, b_h, 1u);
    tc_mma_tf32(d, a_h, b_l, 1u);
    tc_mma_tf32(d, a_h, b_h, 1u);
  }
}

// CTA barrier after every thread wrote its row, then one thread issues the products.  The
// barrier also makes `ok` CTA-uniform: once any thread's wait gave up, nothing more is issued
// (`issued` counts the commits, the same on every thread).
template <int Q, bool TRANS>
__device__ __forceinline__ void tc_tc_issue(char* smem, uint32_t tmem, uint32_t mbar, bool& ok, int& issued) {
  using SM = TcTcSmem<Q>;
  using PL = TcTcPlan<Q>;
  tc_tmem_wait_st();
  tc_fence_async_smem();
  tc_fence_before_sync();
  ok = __syncthreads_and(ok) != 0;
  if (!ok) return;
  issued++;
  if (threadIdx.x == 0) {
    tc_fence_after_sync();
    const uint32_t ahi = tc_smem_u32(smem + SM::OFF_AHI), amid = tc_smem_u32(smem + SM::OFF_AMID);
    const uint32_t bhi = tc_smem_u32(smem + SM::OFF_BHI), blo = tc_smem_u32(smem + SM::OFF_BLO);
    if (TRANS) {
      for (int h = 0; h < PL::TW / 16; h++) tc_tc_mma_half<Q>(tmem, ahi, amid, bhi, blo, 16 * h, PL::NH + (h >> 1), 16 * h);
    } else {
      for (int h = 0; h < PL::NH; h++) tc_tc_mma_half<Q>(tmem, ahi, amid, bhi, blo, 16 * h, h, 16 * h);
    }
    tc_mma_commit(mbar);
  }
}

template <int P, int Q, bool JERK>
__global__ void __launch_bounds__(128, 1) k_m2l_tc(const int* __restrict__ tlist, int ntl,
                                                   const int* __restrict__ tstart, const int* __restrict__ src,
                                                   TcCells c, const float* __restrict__ bins,
                                                   unsigned int* __restrict__ counter, unsigned int* __restrict__ err,
                                                   long long wait_limit = kTcWaitLimit) {
  using PL = TcTcPlan<Q>;
  using SM = TcTcSmem<Q>;
  constexpr int NTP = (P + 1) * (P + 1);  // storage stride of M and L (order P)
  extern __shared__ __align__(128) char smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double* red = reinterpret_cast<double*>(smem + SM::OFF_AHI);  // [4][AW], used after the last product
  unsigned long long* mbar_p = reinterpret_cast<unsigned long long*>(smem + SM::OFF_MISC);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + SM::OFF_MISC + 8);
  int* next_slot = reinterpret_cast<int*>(smem + SM::OFF_MISC + 12);
  double* wmax = reinterpret_cast<double*>(smem + SM::OFF_MISC + 16);  // [4]
  const uint32_t mbar = tc_smem_u32(mbar_p);
  char* ah = smem + SM::OFF_AHI + (tid >> 3) * SM::SBO_A + (tid & 7) * 16;
  char* am = smem + SM::OFF_AMID + (tid >> 3) * SM::SBO_A + (tid & 7) * 16;

  // constant bin matrices -> shared memory
  {
    const float4* s4 = reinterpret_cast<const float4*>(bins);
    float4* d4 = reinterpret_cast<float4*>(smem + SM::OFF_BHI);
    for (int i = tid; i < 2 * SM::B_BYTES / 16; i += blockDim.x) d4[i] = s4[i];
  }
  if (tid == 0) {
    tc_mbar_init(mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_u32(tmem_slot)),
                 "r"(kTcCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_async_smem();
  tc_fence_before_sync();
  __syncthreads();
  tc_fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  const uint32_t tl = tmem + ((uint32_t)(32 * warp) << 16);  // this warp's lane quarter
  uint32_t phase = 0;
  bool ok = true;
  int issued = 0;  // commits issued (CTA-uniform)

  for (;;) {
    if (tid == 0) *next_slot = (int)atomicAdd(counter, 1u);
    __syncthreads();
    const int ti = *next_slot;
    __syncthreads();
    if (ti >= ntl) break;
    const int t = tlist[ti];
    if (!c.has_sink[t]) continue;
    const int s_beg = tstart[t], s_end = tstart[t + 1];
    const double Xt = c.X[t], Yt = c.Y[t], Zt = c.Z[t];
    // FP64 accumulators of row columns tid and tid + 128, for L (a*) and Ld (j*)
    double a0 = 0.0, a1 = 0.0, j0 = 0.0, j1 = 0.0;
    for (int b0 = s_beg; b0 < s_end && ok; b0 += 128) {
      const int idx = b0 + tid;
      const bool valid = idx < s_end;
      const int s = src[valid ? idx : s_beg];
      const TcPairGeo pg = tc_pair_geo(Xt - c.X[s], Yt - c.Y[s], Zt - c.Z[s]);
      const double rinv = valid ? pg.rinv : 0.0;
      // per-pair tables in tensor memory: phases of both angles (m = 0..15), r^-n (FP64)
      {
        float t[64];
        cd ez = mk(1, 0), ex = mk(1, 0);
#pragma unroll
        for (int m = 0; m < 16; m++) {
          t[m] = (float)ez.x;
          t[16 + m] = (float)ez.y;
          t[32 + m] = (float)ex.x;
          t[48 + m] = (float)ex.y;
          ez = ez * pg.ez1;
          ex = ex * pg.ex1;
        }
#pragma unroll
        for (int h = 0; h < 4; h++) tc_tmem_st16(tl + kTcColPh + 16u * h, t + 16 * h);
        float rv[32];
        double rn = 1.0;
#pragma unroll
        for (int n = 0; n < 16; n++) {
          rv[2 * n] = __int_as_float(__double2loint(rn));
          rv[2 * n + 1] = __int_as_float(__double2hiint(rn));
          rn *= pg.rinv;
        }
        tc_tmem_st16(tl + kTcColRn, rv);
        tc_tmem_st16(tl + kTcColRn + 16, rv + 16);
        tc_tmem_wait_st();
      }
      // the tile's largest 1/r: reference scale of the r^-(n+1) factors
      double mx = rinv;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      if (lane == 0) wmax[warp] = mx;
      double rref = 0.0;
#pragma unroll 1
      for (int arr = 0; arr < (JERK ? 2 : 1); arr++) {
        const double* Ms = (arr ? c.Md : c.M) + (size_t)s * NTP;
        // ---- scale, rotate about z, swap
        tc_tc_f0<Q>(Ms, valid, Q == P, tl, ah, am);
        tc_tc_issue<Q, false>(smem, tmem, mbar, ok, issued);
        if (arr == 0) {
          rref = fmax(fmax(wmax[0], wmax[1]), fmax(wmax[2], wmax[3]));
          const float q = rref > 0.0 ? (float)(rinv / rref) : 0.f;
          float qv[16];
          qv[0] = valid ? q : 0.f;
#pragma unroll
          for (int n = 1; n < 16; n++) qv[n] = qv[n - 1] * q;
          tc_tmem_st16(tl + kTcColQn, qv);
          tc_tmem_wait_st();
        }
        // ---- rotate about x, swap
        ok = ok && tc_mbar_wait(mbar, phase, wait_limit);
        phase ^= 1u;
        tc_fence_after_sync();
        tc_tc_rot_stage<Q, false>(1, tl, ah, am);
        tc_tc_issue<Q, false>(smem, tmem, mbar, ok, issued);
        // ---- translate along z
        ok = ok && tc_mbar_wait(mbar, phase, wait_limit);
        phase ^= 1u;
        tc_fence_after_sync();
        tc_tc_f2<Q>(tl, ah, am);
        tc_tc_issue<Q, true>(smem, tmem, mbar, ok, issued);
        // ---- back: swap
        ok = ok && tc_mbar_wait(mbar, phase, wait_limit);
        phase ^= 1u;
        tc_fence_after_sync();
        tc_tc_b0<Q>(tl, ah, am);
        tc_tc_issue<Q, false>(smem, tmem, mbar, ok, issued);
        // ---- rotate back about x, swap
        ok = ok && tc_mbar_wait(mbar, phase, wait_limit);
        phase ^= 1u;
        tc_fence_after_sync();
        tc_tc_rot_stage<Q, true>(1, tl, ah, am);
        tc_tc_issue<Q, false>(smem, tmem, mbar, ok, issued);
        // ---- rotate back about z, scale relative to the tile's 1/r, sum the tile's rows
        ok = ok && tc_mbar_wait(mbar, phase, wait_limit);
        phase ^= 1u;
        tc_fence_after_sync();
        tc_tc_b2<Q>(tl, red + warp * PL::AW, lane);
        tc_fence_before_sync();
        __syncthreads();
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int j = tid + 128 * h;
          if (j < PL::AW) {
            const int k = PL::d_nat(j);
            if (k >= 0) {
              const double sk = red[j] + red[PL::AW + j] + red[2 * PL::AW + j] + red[3 * PL::AW + j];
              int n = 0;
              while ((n + 1) * (n + 1) <= k) n++;
              double rp = rref;
              for (int i = 0; i < n; i++) rp *= rref;
              const double add = sk * (c_mDoF[k] * rp);
              if (arr == 0) {
                if (h == 0) a0 += add; else a1 += add;
              } else {
                if (h == 0) j0 += add; else j1 += add;
              }
            }
          }
        }
        ok = __syncthreads_and(ok);  // red (in the hi rows) is overwritten by the next rows
      }
    }
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int j = tid + 128 * h;
      if (j < PL::AW) {
        const int k = PL::d_nat(j);
        if (k >= 0) {
          c.L[(size_t)t * NTP + k] += h ? a1 : a0;
          if (JERK) c.Ld[(size_t)t * NTP + k] += h ? j1 : j0;
        }
      }
    }
    if (!ok) break;
  }
  ok = __syncthreads_and(ok) != 0;
  if (!ok) {
    // a wait gave up: nothing was issued after it, so at most the last commit is outstanding;
    // wait for it with the default limit before the tensor memory it writes is freed
    if (issued > 0) tc_mbar_wait(mbar, (uint32_t)((issued - 1) & 1), kTcWaitLimit);
    if (tid == 0) atomicOr(err, TC_EBIT_TIMEOUT);
  }
  tc_fence_before_sync();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols) : "memory");
}

}  // namespace tc
