// Near field: P2P over the (target cell, source cell) list, target-stationary.
// Restates P2P_simple (kernel_fast_lean.h:268-459; a = sum m d / r^3, p = sum m / r, r = 0
// skipped, no softening) and the jerk P2P (taichi_with_jerks/kernel_fast_lean.h:499-699;
// J = sum m [dv / r^3 - 3 (d.dv) d / r^5]).
//
// One warp per target cell.  A cell with nt <= 32 bodies uses groups of next_pow2(nt) lanes,
// each group taking every ng-th source body, so small leaves still fill the warp; the
// groups are combined with a fixed shuffle tree (deterministic sums).
#pragma once
#include "tc_down.cuh"

namespace tc {

template <bool JERK>
struct TcAcc {
  double pot, ax, ay, az, jx, jy, jz;
  __device__ __forceinline__ void zero() { pot = ax = ay = az = jx = jy = jz = 0.0; }
  __device__ __forceinline__ void add_xor(int o) {
    pot += __shfl_xor_sync(0xffffffffu, pot, o);
    ax += __shfl_xor_sync(0xffffffffu, ax, o);
    ay += __shfl_xor_sync(0xffffffffu, ay, o);
    az += __shfl_xor_sync(0xffffffffu, az, o);
    if (JERK) {
      jx += __shfl_xor_sync(0xffffffffu, jx, o);
      jy += __shfl_xor_sync(0xffffffffu, jy, o);
      jz += __shfl_xor_sync(0xffffffffu, jz, o);
    }
  }
};

template <bool JERK>
__device__ __forceinline__ void tc_p2p_one(double xi, double yi, double zi, double vxi, double vyi, double vzi,
                                           const TcBodies& b, int j, TcAcc<JERK>& a) {
  if (!(b.flags[j] & 2)) return;
  double dx = b.x[j] - xi, dy = b.y[j] - yi, dz = b.z[j] - zi;
  double r2 = dx * dx + dy * dy + dz * dz;
  if (!(r2 > 0.0)) return;
  double invr = rsqrt(r2), invr2 = invr * invr;
  double f = b.m[j] * invr;
  a.pot += f;
  f *= invr2;
  a.ax += dx * f;
  a.ay += dy * f;
  a.az += dz * f;
  if (JERK) {
    double dvx = b.vx[j] - vxi, dvy = b.vy[j] - vyi, dvz = b.vz[j] - vzi;
    double vr = 3.0 * (dx * dvx + dy * dvy + dz * dvz);
    a.jx += dvx * f;
    a.jy += dvy * f;
    a.jz += dvz * f;
    f *= -invr2 * vr;
    a.jx += dx * f;
    a.jy += dy * f;
    a.jz += dz * f;
  }
}

constexpr int kP2PWarps = 4;

template <bool JERK>
__global__ void __launch_bounds__(kP2PWarps * 32) k_p2p(const int* __restrict__ tlist, int ntl,
                                                        const int* __restrict__ tstart, const int* __restrict__ src,
                                                        const TcBodies b, const TcCells c, TcOut out) {
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int k = blockIdx.x * kP2PWarps + w; k < ntl; k += gridDim.x * kP2PWarps) {
    int t = tlist[k];
    if (!c.has_sink[t]) continue;
    int tb = c.begin[t], nt = c.nbody[t];
    int sb = tstart[t], se = tstart[t + 1];
    int gsz = 32, ng = 1;
    if (nt <= 16) {
      gsz = 1;
      while (gsz < nt) gsz <<= 1;
      ng = 32 / gsz;
    }
    int grp = lane / gsz, ti = lane % gsz;
    for (int t0 = 0; t0 < nt; t0 += gsz) {
      int i = tb + t0 + ti;
      bool vi = (t0 + ti) < nt;
      double xi = 0, yi = 0, zi = 0, vxi = 0, vyi = 0, vzi = 0;
      if (vi) {
        xi = b.x[i]; yi = b.y[i]; zi = b.z[i];
        if (JERK) { vxi = b.vx[i]; vyi = b.vy[i]; vzi = b.vz[i]; }
      }
      TcAcc<JERK> a;
      a.zero();
      if (vi) {
        for (int q = sb; q < se; q++) {
          int s = src[q];
          int jb = c.begin[s], je = jb + c.nbody[s];
          for (int j = jb + grp; j < je; j += ng) tc_p2p_one<JERK>(xi, yi, zi, vxi, vyi, vzi, b, j, a);
        }
      }
      for (int o = gsz; o < 32; o <<= 1) a.add_xor(o);
      if (vi && grp == 0 && (b.flags[i] & 1)) {
        out.pot[i] += a.pot;
        out.ax[i] += a.ax;
        out.ay[i] += a.ay;
        out.az[i] += a.az;
        if (JERK) {
          out.jx[i] += a.jx;
          out.jy[i] += a.jy;
          out.jz[i] += a.jz;
        }
      }
    }
  }
}

// direct summation (N below the direct threshold): one warp per 32 targets
template <bool JERK>
__global__ void k_direct(int n, const TcBodies b, TcOut out) {
  int lane = threadIdx.x & 31;
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int nwarp = (gridDim.x * blockDim.x) >> 5;
  for (int t0 = warp * 32; t0 < n; t0 += nwarp * 32) {
    int i = t0 + lane;
    bool vi = i < n;
    TcAcc<JERK> a;
    a.zero();
    if (vi && (b.flags[i] & 1)) {
      double xi = b.x[i], yi = b.y[i], zi = b.z[i];
      double vxi = JERK ? b.vx[i] : 0, vyi = JERK ? b.vy[i] : 0, vzi = JERK ? b.vz[i] : 0;
      for (int j = 0; j < n; j++) tc_p2p_one<JERK>(xi, yi, zi, vxi, vyi, vzi, b, j, a);
    }
    if (vi) {
      out.pot[i] = a.pot; out.ax[i] = a.ax; out.ay[i] = a.ay; out.az[i] = a.az;
      if (JERK) { out.jx[i] = a.jx; out.jy[i] = a.jy; out.jz[i] = a.jz; }
    }
  }
}

// Morton order -> caller order
__global__ void k_scatter_out(int n, const int* __restrict__ perm, TcOut s, double* pot, double* ax, double* ay,
                              double* az, double* jx, double* jy, double* jz) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int j = perm[i];
  pot[j] = s.pot[i]; ax[j] = s.ax[i]; ay[j] = s.ay[i]; az[j] = s.az[i];
  if (jx) { jx[j] = s.jx ? s.jx[i] : 0.0; jy[j] = s.jy ? s.jy[i] : 0.0; jz[j] = s.jz ? s.jz[i] : 0.0; }
}

}  // namespace tc

namespace tc {

// ---------------------------------------------------------------------------------------
// Mixed-precision near field: FP32 interactions, compensated sums.
// Positions enter relative to the target cell centre as FP32 (hi, lo) pairs formed in FP64,
// so dx = (xj_hi - xi_hi) + (xj_lo - xi_lo) keeps ~1e-14 relative accuracy even for close
// pairs; each 32-source tile is summed in FP32 and folded into (hi, lo) accumulators with
// a two-sum; the final per-target sum is formed in FP64.
// ---------------------------------------------------------------------------------------
struct TcF2 {
  float hi, lo;
  __device__ __forceinline__ void add(float t) {  // two-sum
    float s = hi + t;
    float bp = s - hi;
    float e = (hi - (s - bp)) + (t - bp);
    hi = s;
    lo += e;
  }
  __device__ __forceinline__ double val() const { return (double)hi + (double)lo; }
};

template <bool JERK>
__global__ void __launch_bounds__(kP2PWarps * 32) k_p2p_mixed(const int* __restrict__ tlist, int ntl,
                                                              const int* __restrict__ tstart,
                                                              const int* __restrict__ src, const TcBodies b,
                                                              const TcCells c, TcOut out) {
  // per warp source tile: xh yh zh xl yl zl m vx vy vz
  __shared__ float tile[kP2PWarps][10][32];
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float(*T)[32] = tile[w];
  for (int k = blockIdx.x * kP2PWarps + w; k < ntl; k += gridDim.x * kP2PWarps) {
    int t = tlist[k];
    if (!c.has_sink[t]) continue;
    const double Xc = c.X[t], Yc = c.Y[t], Zc = c.Z[t];
    int tb = c.begin[t], nt = c.nbody[t];
    int sb = tstart[t], se = tstart[t + 1];
    int gsz = 32, ng = 1;
    if (nt <= 16) {
      gsz = 1;
      while (gsz < nt) gsz <<= 1;
      ng = 32 / gsz;
    }
    int grp = lane / gsz, ti = lane % gsz;
    for (int t0 = 0; t0 < nt; t0 += gsz) {
      int i = tb + t0 + ti;
      bool vi = (t0 + ti) < nt;
      float xh = 0, yh = 0, zh = 0, xl = 0, yl = 0, zl = 0, vxi = 0, vyi = 0, vzi = 0;
      if (vi) {
        double dx = b.x[i] - Xc, dy = b.y[i] - Yc, dz = b.z[i] - Zc;
        xh = (float)dx; xl = (float)(dx - (double)xh);
        yh = (float)dy; yl = (float)(dy - (double)yh);
        zh = (float)dz; zl = (float)(dz - (double)zh);
        if (JERK) { vxi = (float)b.vx[i]; vyi = (float)b.vy[i]; vzi = (float)b.vz[i]; }
      }
      TcF2 pot = {0, 0}, ax = {0, 0}, ay = {0, 0}, az = {0, 0}, jx = {0, 0}, jy = {0, 0}, jz = {0, 0};
      for (int q = sb; q < se; q++) {
        int s = src[q];
        int jb = c.begin[s], jn = c.nbody[s];
        for (int j0 = 0; j0 < jn; j0 += 32) {
          int cnt = min(32, jn - j0);
          __syncwarp();
          if (lane < cnt) {
            int j = jb + j0 + lane;
            double dx = b.x[j] - Xc, dy = b.y[j] - Yc, dz = b.z[j] - Zc;
            float h;
            h = (float)dx; T[0][lane] = h; T[3][lane] = (float)(dx - (double)h);
            h = (float)dy; T[1][lane] = h; T[4][lane] = (float)(dy - (double)h);
            h = (float)dz; T[2][lane] = h; T[5][lane] = (float)(dz - (double)h);
            T[6][lane] = (b.flags[j] & 2) ? (float)b.m[j] : 0.f;
            if (JERK) { T[7][lane] = (float)b.vx[j]; T[8][lane] = (float)b.vy[j]; T[9][lane] = (float)b.vz[j]; }
          }
          __syncwarp();
          float sp = 0, sx = 0, sy = 0, sz = 0, qx = 0, qy = 0, qz = 0;
          if (vi) {
            for (int jj = grp; jj < cnt; jj += ng) {
              float dx = (T[0][jj] - xh) + (T[3][jj] - xl);
              float dy = (T[1][jj] - yh) + (T[4][jj] - yl);
              float dz = (T[2][jj] - zh) + (T[5][jj] - zl);
              float r2 = dx * dx + dy * dy + dz * dz;
              float ri = r2 > 0.f ? rsqrtf(r2) : 0.f;
              float f = T[6][jj] * ri;
              sp += f;
              float ri2 = ri * ri;
              f *= ri2;
              sx += dx * f;
              sy += dy * f;
              sz += dz * f;
              if (JERK) {
                float dvx = T[7][jj] - vxi, dvy = T[8][jj] - vyi, dvz = T[9][jj] - vzi;
                float vr = 3.f * (dx * dvx + dy * dvy + dz * dvz);
                qx += dvx * f;
                qy += dvy * f;
                qz += dvz * f;
                float g = -f * ri2 * vr;
                qx += dx * g;
                qy += dy * g;
                qz += dz * g;
              }
            }
          }
          pot.add(sp); ax.add(sx); ay.add(sy); az.add(sz);
          if (JERK) { jx.add(qx); jy.add(qy); jz.add(qz); }
        }
      }
      TcAcc<JERK> a;
      a.pot = pot.val(); a.ax = ax.val(); a.ay = ay.val(); a.az = az.val();
      a.jx = jx.val(); a.jy = jy.val(); a.jz = jz.val();
      for (int o = gsz; o < 32; o <<= 1) a.add_xor(o);
      if (vi && grp == 0 && (b.flags[i] & 1)) {
        out.pot[i] += a.pot;
        out.ax[i] += a.ax;
        out.ay[i] += a.ay;
        out.az[i] += a.az;
        if (JERK) {
          out.jx[i] += a.jx;
          out.jy[i] += a.jy;
          out.jz[i] += a.jz;
        }
      }
    }
  }
}

}  // namespace tc
