// The error-controlled MAC (tc_set_error_mac): the low-order pre-pass that the reference runs
// before it (top tree integrator.h:476-493; jerks tree taichi_with_jerks/integrator.h:326-360)
// and the per-cell inputs of the MAC.  The top tree's pre-pass is described first; the jerks
// tree's differs in its near field and output (k_low_p2p_jerks below).
//
// Pre-pass (traverse_eager.h:36-52, :220-258, :306-322; kernel_fast_lean.h:1358-1647): an
// order-2 FMM on the geometric cells (centre and radius of the octree, before any enclosing
// ball), opening criterion |d|^2 > 3 (Ri + Rj)^2, whose output is a per-body estimate of the
// acceleration magnitude, acc_old:
//   acc_old = sum over its low-order P2P source cells of q_last / r^2  (only the LAST body of
//             each source cell counts: the reference's P2P_low assigns rather than adds in
//             its loop over sources, kernel_fast_lean.h:1509-1534; a coincident body gives 0)
//           + |grad phi| of the order-2 local expansion at the body (L2P_low, :1610-1646).
// Then every cell's min_acc is the least acc_old of its bodies (P2M, kernel_fast_lean.h:757)
// or of its children (M2M, :799-839), and Pn[n] = sqrt(sum_m M[n,m]^2 (n+m)!(n-m)!)
// (integrator.h:527-539) with the reference's factorial table, whose (2P)! entry is zero.
// Everything is FP64 with one thread per cell, body or target cell; sums over interaction
// lists run in the lists' sorted order (deterministic).
#pragma once
#include "tc_harmonics.cuh"

namespace tc {

constexpr int kLowNT = 9;  // order 2: (2 + 1)^2 terms

// regular solid harmonics to order 2 at d, complex full storage (index n*n+n+m)
__device__ __forceinline__ void tc_low_gnm(double dx, double dy, double dz, cd* G) {
  const double r2 = dx * dx + dy * dy + dz * dz;
  // columns m = 0, 1, 2 by the recurrence of make_Gnm (kernel_fast_lean.h:235-266)
  const cd g00 = mk(1, 0);
  const cd g11 = g00 * mk(dx / 2, dy / 2);
  const cd g22 = g11 * mk(dx / 4, dy / 4);
  const cd g10 = dz * g00;
  const cd g21 = dz * g11;
  const cd g20 = ((2 * 2 - 1.) / 4.0 * dz) * g10 - (r2 / 4.0) * g00;
  G[0] = g00;
  G[2] = g10;
  G[3] = g11;
  G[1] = mk(-g11.x, g11.y);  // (-1)^1 conj
  G[6] = g20;
  G[7] = g21;
  G[8] = g22;
  G[5] = mk(-g21.x, g21.y);
  G[4] = mk(g22.x, -g22.y);
}

// singular harmonics to order 2 (make_Tnm, kernel_fast_lean.h:193-233)
__device__ __forceinline__ void tc_low_tnm(double dx, double dy, double dz, cd* T) {
  const double r2 = dx * dx + dy * dy + dz * dz, invr2 = 1 / r2;
  T[0] = mk(sqrt(invr2), 0);
  // n = 1
  T[3] = T[0] * mk(dx * 1 * invr2, dy * 1 * invr2);
  T[2] = (invr2 * 1. * dz) * T[0];
  T[1] = mk(-T[3].x, T[3].y);  // conj(T[3] * -1)
  // n = 2
  T[8] = T[3] * mk(dx * 3 * invr2, dy * 3 * invr2);
  T[6] = (invr2 * 3. * dz) * T[2] - (invr2 * (1 - 0)) * T[0];
  T[7] = (invr2 * 3. * dz) * T[3];
  T[5] = mk(-T[7].x, T[7].y);  // conj(T[7] * -1)
  T[4] = mk(T[8].x, -T[8].y);  // conj(T[8] * 1)
}

// reference real storage -> complex full storage (real_2_complex, kernel_fast_lean.h:162-177)
__device__ __forceinline__ void tc_low_r2c(const double* r, cd* c) {
  for (int n = 0; n <= 2; n++) {
    const int is = n * n + n;
    c[is] = mk(r[is], 0);
    double s = -1;
    for (int m = 1; m <= n; m++) {
      c[is - m] = mk(r[is + m] * s, -r[is - m] * s);
      c[is + m] = mk(r[is + m], r[is - m]);
      s *= -1;
    }
  }
}

// complex (m >= 0 entries) -> real storage added to dst (complex_2_real then +=)
__device__ __forceinline__ void tc_low_c2r_add(const cd* c, double* dst) {
  for (int n = 0; n <= 2; n++) {
    const int is = n * n + n;
    dst[is] += c[is].x;
    for (int m = 1; m <= n; m++) {
      dst[is - m] += c[is + m].y;
      dst[is + m] += c[is + m].x;
    }
  }
}

// geometric radius of every cell: R0 / 2^level (build_tree.h:274)
__global__ void k_low_rgeo(int ncell, const int* __restrict__ level, const TcRootInfo* root, double* rgeo) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x)
    rgeo[c] = tc_level_radius(root->R0, level[c]);
}

// P2M_low of every leaf (kernel_fast_lean.h:1358-1374): M9 of the geometric centre
__global__ void k_low_p2m(int ncell, const TcBodies b, const TcCells c, double* __restrict__ M9) {
  for (int ci = blockIdx.x * blockDim.x + threadIdx.x; ci < ncell; ci += gridDim.x * blockDim.x) {
    double* M = M9 + (size_t)ci * kLowNT;
    for (int k = 0; k < kLowNT; k++) M[k] = 0.0;
    if (c.nchild[ci] != 0) continue;
    cd acc[kLowNT];
    for (int k = 0; k < kLowNT; k++) acc[k] = mk(0, 0);
    for (int i = c.begin[ci]; i < c.begin[ci] + c.nbody[ci]; i++) {
      cd G[kLowNT];
      tc_low_gnm(b.x[i] - c.gx[ci], b.y[i] - c.gy[ci], b.z[i] - c.gz[ci], G);
      for (int k = 0; k < kLowNT; k++) acc[k] += b.m[i] * G[k];
    }
    tc_low_c2r_add(acc, M);
  }
}

// M2M_low into the inner cells of level l (kernel_fast_lean.h:1376-1424)
__global__ void k_low_m2m(int l, const TcCells c, const int* __restrict__ lv_start, const int* __restrict__ lv_count,
                          double* __restrict__ M9) {
  const int cnt = lv_count[l], st = lv_start[l];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x) {
    const int ci = st + k;
    if (c.nchild[ci] == 0) continue;
    cd acc[kLowNT];
    for (int q = 0; q < kLowNT; q++) acc[q] = mk(0, 0);
    for (int cj = c.child[ci]; cj < c.child[ci] + c.nchild[ci]; cj++) {
      cd cm[kLowNT], G[kLowNT];
      tc_low_r2c(M9 + (size_t)cj * kLowNT, cm);
      tc_low_gnm(c.gx[cj] - c.gx[ci], c.gy[cj] - c.gy[ci], c.gz[cj] - c.gz[ci], G);
      for (int n = 0; n <= 2; n++)
        for (int m = 0; m <= n; m++) {
          const int ind = n * n + n + m;
          for (int kk = 0; kk <= n; kk++)
            for (int ll = max(-kk, m - n + kk); ll <= min(kk, m + n - kk); ll++)
              acc[ind] += cm[(n - kk) * (n - kk) + (n - kk) + (m - ll)] * G[kk * kk + kk + ll];
        }
    }
    tc_low_c2r_add(acc, M9 + (size_t)ci * kLowNT);
  }
}

// M2L_low into every target of the low-order M2L list, sources in list order
// (kernel_fast_lean.h:1426-1477); L9 is zero before
__global__ void k_low_m2l(int ncell, const TcCells c, const int* __restrict__ start, const int* __restrict__ src,
                          const double* __restrict__ M9, double* __restrict__ L9) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ncell; t += gridDim.x * blockDim.x) {
    for (int q = start[t]; q < start[t + 1]; q++) {
      const int s = src[q];
      double Mm[kLowNT];
      for (int k = 0; k < kLowNT; k++) Mm[k] = M9[(size_t)s * kLowNT + k];
      for (int n = 0; n <= 2; n++)
        for (int m = 1; m <= n; m++) Mm[n * n + n - m] *= -1;
      cd cm[kLowNT], T[kLowNT], o[kLowNT];
      tc_low_r2c(Mm, cm);
      tc_low_tnm(c.gx[t] - c.gx[s], c.gy[t] - c.gy[s], c.gz[t] - c.gz[s], T);
      for (int k = 0; k < kLowNT; k++) o[k] = mk(0, 0);
      for (int n = 0; n <= 2; n++)
        for (int m = 0; m <= n; m++) {
          const int ind = n * n + n + m;
          for (int kk = 0; kk <= 2 - n; kk++)
            for (int ll = -kk; ll <= kk; ll++)
              o[ind] += cm[kk * kk + kk + ll] * T[(n + kk) * (n + kk) + (n + kk) + (m + ll)];
        }
      tc_low_c2r_add(o, L9 + (size_t)t * kLowNT);
    }
  }
}

// P2P_low: acc_old[i] = sum over the low-order P2P source cells of the target cell of the
// last source body's q / r^2 (0 if it coincides with i), in list order
__global__ void k_low_p2p(int n, const TcBodies b, const TcCells c, const int* __restrict__ cell_of,
                          const int* __restrict__ start, const int* __restrict__ src, double* __restrict__ acc_old) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int t = cell_of[i];
    double a = 0.0;
    for (int q = start[t]; q < start[t + 1]; q++) {
      const int s = src[q];
      const int j = c.begin[s] + c.nbody[s] - 1;
      const double dx = b.x[i] - b.x[j], dy = b.y[i] - b.y[j], dz = b.z[i] - b.z[j];
      const double r2 = dx * dx + dy * dy + dz * dz;
      const double mj = r2 > 0 ? b.m[j] : 0.0;
      a += mj / (r2 > 0 ? r2 : HUGE_VAL);
    }
    acc_old[i] = a;
  }
}

// leaf of every body
__global__ void k_low_cell_of(int ncell, const TcCells c, int* __restrict__ cell_of) {
  for (int ci = blockIdx.x * blockDim.x + threadIdx.x; ci < ncell; ci += gridDim.x * blockDim.x)
    if (c.nchild[ci] == 0)
      for (int i = c.begin[ci]; i < c.begin[ci] + c.nbody[ci]; i++) cell_of[i] = ci;
}

// L2L_low from the inner cells of level l to their children (kernel_fast_lean.h:1558-1608)
__global__ void k_low_l2l(int l, const TcCells c, const int* __restrict__ lv_start, const int* __restrict__ lv_count,
                          double* __restrict__ L9) {
  const int cnt = lv_count[l], st = lv_start[l];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x) {
    const int ci = st + k;
    if (c.nchild[ci] == 0) continue;
    cd cl[kLowNT];
    tc_low_r2c(L9 + (size_t)ci * kLowNT, cl);
    for (int cj = c.child[ci]; cj < c.child[ci] + c.nchild[ci]; cj++) {
      cd G[kLowNT], o[kLowNT];
      tc_low_gnm(c.gx[ci] - c.gx[cj], c.gy[ci] - c.gy[cj], c.gz[ci] - c.gz[cj], G);
      for (int q = 0; q < kLowNT; q++) {
        G[q] = conj(G[q]);
        o[q] = mk(0, 0);
      }
      for (int n = 0; n <= 2; n++)
        for (int m = 0; m <= n; m++) {
          const int ind = n * n + n + m;
          for (int kk = 0; kk <= 2 - n; kk++)
            for (int ll = -kk; ll <= kk; ll++)
              o[ind] += cl[(n + kk) * (n + kk) + (n + kk) + (m + ll)] * G[kk * kk + kk + ll];
        }
      tc_low_c2r_add(o, L9 + (size_t)cj * kLowNT);
    }
  }
}

// L2P_low (kernel_fast_lean.h:1610-1646): acc_old += |grad phi| of every leaf body
__global__ void k_low_l2p(int n, const TcBodies b, const TcCells c, const int* __restrict__ cell_of,
                          const double* __restrict__ L9, double* __restrict__ acc_old) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int ci = cell_of[i];
    cd cl[kLowNT], G[kLowNT], Phi[4];
    tc_low_r2c(L9 + (size_t)ci * kLowNT, cl);
    tc_low_gnm(c.gx[ci] - b.x[i], c.gy[ci] - b.y[i], c.gz[ci] - b.z[i], G);
    for (int q = 0; q < kLowNT; q++) G[q] = conj(G[q]);
    for (int q = 0; q < 4; q++) Phi[q] = mk(0, 0);
    for (int nn = 0; nn <= 1; nn++)
      for (int m = 0; m <= nn; m++) {
        const int ind = nn * nn + nn + m;
        for (int kk = 0; kk <= 2 - nn; kk++)
          for (int ll = -kk; ll <= kk; ll++)
            Phi[ind] += cl[(nn + kk) * (nn + kk) + (nn + kk) + (m + ll)] * G[kk * kk + kk + ll];
      }
    acc_old[i] += sqrt(Phi[3].x * Phi[3].x + Phi[3].y * Phi[3].y + Phi[2].x * Phi[2].x);
  }
}

// ---------------------------------------------------------------------------------------
// The jerks tree's pre-pass (taichi_with_jerks/integrator.h:326-360) differs from the top
// tree's in its near field and its output: P2P_low (taichi_with_jerks/kernel_fast_lean.h:
// 1567-1688, the SIMD_P2P branch the reference is built with) sums the acceleration VECTOR of
// every source body of a low-order P2P source cell in FP32 (16 targets per SIMD vector, one
// FP32 sum per source cell, added to the body's FP64 F), L2P_low (:1742-1780) subtracts the
// order-2 local's gradient from F, and acc_old = |F| (integrator.h:350-356).  The FP32
// arithmetic follows the reference's x86-64-v4 build operation by operation: positions and
// masses rounded to FP32, dx = xj + (-xi), r2 = fma(dz, dz, fma(dy, dy, dx dx)), IEEE sqrt
// and division, f = ((m / r) / r) / r as three products, a = fma(dx, f, a).
// ---------------------------------------------------------------------------------------
__global__ void k_low_p2p_jerks(int n, const TcBodies b, const TcCells c, const int* __restrict__ cell_of,
                                const int* __restrict__ start, const int* __restrict__ src,
                                double* __restrict__ F) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int t = cell_of[i];
    const float xi = -(float)b.x[i], yi = -(float)b.y[i], zi = -(float)b.z[i];
    double Fx = 0.0, Fy = 0.0, Fz = 0.0;
    for (int q = start[t]; q < start[t + 1]; q++) {
      const int s = src[q];
      float ax = 0.f, ay = 0.f, az = 0.f;
      for (int j = c.begin[s]; j < c.begin[s] + c.nbody[s]; j++) {
        const float dx = __fadd_rn(xi, (float)b.x[j]);
        const float dy = __fadd_rn(yi, (float)b.y[j]);
        const float dz = __fadd_rn(zi, (float)b.z[j]);
        const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
        const float mj = r2 > 0.f ? (float)b.m[j] : 0.f;
        const float rr = r2 > 0.f ? r2 : __int_as_float(0x7f800000);
        const float inv = __fdiv_rn(1.f, __fsqrt_rn(rr));
        const float f = __fmul_rn(__fmul_rn(__fmul_rn(mj, inv), inv), inv);
        ax = __fmaf_rn(dx, f, ax);
        ay = __fmaf_rn(dy, f, ay);
        az = __fmaf_rn(dz, f, az);
      }
      Fx += (double)ax;
      Fy += (double)ay;
      Fz += (double)az;
    }
    F[i] = Fx;
    F[(size_t)n + i] = Fy;
    F[2 * (size_t)n + i] = Fz;
  }
}

// L2P_low of the jerks tree: F -= grad of the order-2 local at the body, acc_old = |F|
__global__ void k_low_l2p_jerks(int n, const TcBodies b, const TcCells c, const int* __restrict__ cell_of,
                                const double* __restrict__ L9, const double* __restrict__ F,
                                double* __restrict__ acc_old) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int ci = cell_of[i];
    cd cl[kLowNT], G[kLowNT], Phi[4];
    tc_low_r2c(L9 + (size_t)ci * kLowNT, cl);
    tc_low_gnm(c.gx[ci] - b.x[i], c.gy[ci] - b.y[i], c.gz[ci] - b.z[i], G);
    for (int q = 0; q < kLowNT; q++) G[q] = conj(G[q]);
    for (int q = 0; q < 4; q++) Phi[q] = mk(0, 0);
    for (int nn = 0; nn <= 1; nn++)
      for (int m = 0; m <= nn; m++) {
        const int ind = nn * nn + nn + m;
        for (int kk = 0; kk <= 2 - nn; kk++)
          for (int ll = -kk; ll <= kk; ll++)
            Phi[ind] += cl[(nn + kk) * (nn + kk) + (nn + kk) + (m + ll)] * G[kk * kk + kk + ll];
      }
    const double fx = F[i] - Phi[3].x, fy = F[(size_t)n + i] - Phi[3].y, fz = F[2 * (size_t)n + i] - Phi[2].x;
    acc_old[i] = sqrt(__fma_rn(fz, fz, __fma_rn(fx, fx, __dmul_rn(fy, fy))));
  }
}

// min_acc of the cells of level l: the least acc_old of a leaf's bodies, or of an inner cell's
// children (1e30 when empty)
__global__ void k_min_acc(int l, const TcCells c, const int* __restrict__ lv_start, const int* __restrict__ lv_count,
                          const double* __restrict__ acc_old, double* __restrict__ min_acc) {
  const int cnt = lv_count[l], st = lv_start[l];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x) {
    const int ci = st + k;
    double v = 1e30;
    if (c.nchild[ci] == 0) {
      for (int i = c.begin[ci]; i < c.begin[ci] + c.nbody[ci]; i++) v = fmin(acc_old[i], v);
    } else {
      for (int cj = c.child[ci]; cj < c.child[ci] + c.nchild[ci]; cj++) v = fmin(min_acc[cj], v);
    }
    min_acc[ci] = v;
  }
}

// Pn as integrator.h:527-539 computes it: factorials of the reference's table, (2P)! = 0
template <int P>
__global__ void k_cell_pn_ref(int ncell, const double* __restrict__ M, double* __restrict__ pn) {
  constexpr int NT = (P + 1) * (P + 1);
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
    const double* mc = M + (size_t)c * NT;
    for (int n = 0; n <= P; n++) {
      double s = 0.0;
      for (int m = -n; m <= n; m++) {
        const double fa = (n + m == 2 * P) ? 0.0 : c_fact[n + m];
        const double fb = (n - m == 2 * P) ? 0.0 : c_fact[n - m];
        const double v = mc[n * n + n + m];
        s += v * v * fa * fb;
      }
      pn[(size_t)c * (P + 1) + n] = sqrt(s);
    }
  }
}

}  // namespace tc
