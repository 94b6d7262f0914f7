// System diagnostics and the compensated drift of the reference's integrator.
//
//   k_sys_diag_part / k_sys_diag_final
//     system_kinetic_energy (integrator.h:887-895), system_potential_energy (:897-904) and
//     system_center_of_mass (:906-925): sums over all bodies of m |v|^2 / 2, m pot / 2, m, m x
//     and m v.  The reference accumulates in long double (64-bit mantissa); here every sum is a
//     double-double (about 106 bits) so the result is the correctly rounded sum up to the
//     per-term rounding, and it does not depend on the launch shape: each thread folds a fixed
//     grid-stride sequence, blocks reduce in a fixed tree order, one block folds the partials.
//     The per-term values follow the reference's expressions in FP64 without contraction:
//     m * (vx*vx + vy*vy + vz*vz) / 2 and m * pot / 2 (G = 1 as exafmm.h:97); the centre-of-mass
//     products m x and m v enter exactly (two-product), as the reference forms them in long
//     double.  HBM-bound: 64 bytes read per body (m, x, y, z, vx, vy, vz, pot).
//
//   k_drift_compsum
//     drift (integrator.h:642-656) with COMPSUM (integrator.h:42): per axis
//       a = s;  e += dt * v;  s = a + e;  e += a - s
//     with the reference's pos_e carried by the caller between calls.  The e += dt * v term is a
//     single fused multiply-add, as the reference's expression contracts when it is compiled for
//     an FMA-capable x86 target (its Makefile builds with -march=native).
#pragma once

namespace tc {

constexpr int kDiagQ = 9;         // kinetic, potential, mass, m x (3), m v (3)
constexpr int kDiagThreads = 256;

struct TcDD {
  double hi, lo;
};

// a + b for a normalised double-double a and a double b (two-sum, then fast renormalisation)
__device__ __forceinline__ TcDD tc_dd_add(TcDD a, double b) {
  const double s = __dadd_rn(a.hi, b);
  const double bb = __dadd_rn(s, -a.hi);
  const double e = __dadd_rn(__dadd_rn(a.hi, -__dadd_rn(s, -bb)), __dadd_rn(b, -bb));
  const double t = __dadd_rn(e, a.lo);
  const double h = __dadd_rn(s, t);
  return {h, __dadd_rn(t, -__dadd_rn(h, -s))};
}

__device__ __forceinline__ TcDD tc_dd_add(TcDD a, TcDD b) {
  const double s = __dadd_rn(a.hi, b.hi);
  const double bb = __dadd_rn(s, -a.hi);
  const double e = __dadd_rn(__dadd_rn(a.hi, -__dadd_rn(s, -bb)), __dadd_rn(b.hi, -bb));
  const double t = __dadd_rn(e, __dadd_rn(a.lo, b.lo));
  const double h = __dadd_rn(s, t);
  return {h, __dadd_rn(t, -__dadd_rn(h, -s))};
}

// the exact product a * b as a double-double
__device__ __forceinline__ TcDD tc_dd_prod(double a, double b) {
  const double p = __dmul_rn(a, b);
  return {p, __fma_rn(a, b, -p)};
}

// block-wide fixed-order tree reduction of kDiagQ double-doubles; the result is in sh[0..]
__device__ __forceinline__ void tc_diag_block_reduce(TcDD (*sh)[kDiagThreads], TcDD* acc) {
  const int t = threadIdx.x;
#pragma unroll
  for (int q = 0; q < kDiagQ; q++) sh[q][t] = acc[q];
  __syncthreads();
  for (int s = kDiagThreads / 2; s > 0; s >>= 1) {
    if (t < s) {
#pragma unroll
      for (int q = 0; q < kDiagQ; q++) sh[q][t] = tc_dd_add(sh[q][t], sh[q][t + s]);
    }
    __syncthreads();
  }
}

// One double-double partial per block and quantity: part[(block * kDiagQ + q) * 2 + {0, 1}].
__global__ void __launch_bounds__(kDiagThreads, 3) k_sys_diag_part(
    int n, const double* __restrict__ m, const double* __restrict__ x, const double* __restrict__ y,
    const double* __restrict__ z, const double* __restrict__ vx, const double* __restrict__ vy,
    const double* __restrict__ vz, const double* __restrict__ pot, double* __restrict__ part) {
  __shared__ TcDD sh[kDiagQ][kDiagThreads];
  TcDD acc[kDiagQ];
#pragma unroll
  for (int q = 0; q < kDiagQ; q++) acc[q] = {0.0, 0.0};
  // 64-bit indices: i + stride must not wrap for n within one grid stride of INT_MAX
  const long long stride = (long long)gridDim.x * kDiagThreads;
  // software-pipelined: the next body's eight values are loaded before this body is folded, so
  // each thread keeps two bodies' loads in flight (same order of the sums as a plain loop)
  long long i = (long long)blockIdx.x * kDiagThreads + threadIdx.x;
  double cm = 0, cx = 0, cy = 0, cz = 0, cu = 0, cv = 0, cw = 0, cp = 0;
  if (i < n) { cm = m[i]; cx = x[i]; cy = y[i]; cz = z[i]; cu = vx[i]; cv = vy[i]; cw = vz[i]; cp = pot[i]; }
  for (; i < n; i += stride) {
    const double mi = cm, px = cx, py = cy, pz = cz, ux = cu, uy = cv, uz = cw, pi = cp;
    const long long j = i + stride;
    if (j < n) { cm = m[j]; cx = x[j]; cy = y[j]; cz = z[j]; cu = vx[j]; cv = vy[j]; cw = vz[j]; cp = pot[j]; }
    const double v2 = __dadd_rn(__dadd_rn(__dmul_rn(ux, ux), __dmul_rn(uy, uy)), __dmul_rn(uz, uz));
    acc[0] = tc_dd_add(acc[0], __dmul_rn(__dmul_rn(mi, v2), 0.5));
    acc[1] = tc_dd_add(acc[1], __dmul_rn(__dmul_rn(mi, pi), 0.5));
    acc[2] = tc_dd_add(acc[2], mi);
    acc[3] = tc_dd_add(acc[3], tc_dd_prod(mi, px));
    acc[4] = tc_dd_add(acc[4], tc_dd_prod(mi, py));
    acc[5] = tc_dd_add(acc[5], tc_dd_prod(mi, pz));
    acc[6] = tc_dd_add(acc[6], tc_dd_prod(mi, ux));
    acc[7] = tc_dd_add(acc[7], tc_dd_prod(mi, uy));
    acc[8] = tc_dd_add(acc[8], tc_dd_prod(mi, uz));
  }
  tc_diag_block_reduce(sh, acc);
  if (threadIdx.x < kDiagQ) {
    const TcDD r = sh[threadIdx.x][0];
    part[(blockIdx.x * kDiagQ + threadIdx.x) * 2] = r.hi;
    part[(blockIdx.x * kDiagQ + threadIdx.x) * 2 + 1] = r.lo;
  }
}

// (a.hi + a.lo) / (b.hi + b.lo) rounded to a double (one Newton correction of the quotient)
__device__ __forceinline__ double tc_dd_div(TcDD a, TcDD b) {
  const double q = a.hi / b.hi;
  const double r = __dadd_rn(__dadd_rn(__fma_rn(-q, b.hi, a.hi), a.lo), -__dmul_rn(q, b.lo));
  return __dadd_rn(q, r / b.hi);
}

// Folds nblk block partials (one block, fixed order) and writes
// out[0..8] = kinetic, potential, mass, centre of mass x y z, centre-of-mass velocity x y z.
__global__ void __launch_bounds__(kDiagThreads) k_sys_diag_final(int nblk, const double* __restrict__ part,
                                                                 double* __restrict__ out) {
  __shared__ TcDD sh[kDiagQ][kDiagThreads];
  TcDD acc[kDiagQ];
#pragma unroll
  for (int q = 0; q < kDiagQ; q++) acc[q] = {0.0, 0.0};
  for (int b = threadIdx.x; b < nblk; b += kDiagThreads) {
#pragma unroll
    for (int q = 0; q < kDiagQ; q++)
      acc[q] = tc_dd_add(acc[q], TcDD{part[(b * kDiagQ + q) * 2], part[(b * kDiagQ + q) * 2 + 1]});
  }
  tc_diag_block_reduce(sh, acc);
  if (threadIdx.x == 0) {
    out[0] = sh[0][0].hi;
    out[1] = sh[1][0].hi;
    out[2] = sh[2][0].hi;
    for (int d = 0; d < 3; d++) {
      out[3 + d] = tc_dd_div(sh[3 + d][0], sh[2][0]);
      out[6 + d] = tc_dd_div(sh[6 + d][0], sh[2][0]);
    }
  }
}

__global__ void k_drift_compsum(int n, double* __restrict__ x, double* __restrict__ y, double* __restrict__ z,
                                double* __restrict__ ex, double* __restrict__ ey, double* __restrict__ ez,
                                const double* __restrict__ vx, const double* __restrict__ vy,
                                const double* __restrict__ vz, double dt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double* const S[3] = {x, y, z};
  double* const E[3] = {ex, ey, ez};
  const double* const V[3] = {vx, vy, vz};
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double a = S[d][i];
    double e = __fma_rn(dt, V[d][i], E[d][i]);
    const double s = __dadd_rn(a, e);
    e = __dadd_rn(e, __dadd_rn(a, -s));
    S[d][i] = s;
    E[d][i] = e;
  }
}

}  // namespace tc
