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
