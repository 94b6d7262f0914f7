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
  // sum of the ng lane groups (group g = lanes [g gsz, (g + 1) gsz)) into group 0 by a fixed
  // tree: at step s, group g (a multiple of 2 s) adds group g + s
  __device__ __forceinline__ void add_groups(int gsz, int ng, int grp) {
    for (int st = 1; st < ng; st <<= 1) {
      const int off = st * gsz;
      const bool take = (grp % (2 * st)) == 0 && grp + st < ng;
      double v;
      v = __shfl_down_sync(0xffffffffu, pot, off); if (take) pot += v;
      v = __shfl_down_sync(0xffffffffu, ax, off); if (take) ax += v;
      v = __shfl_down_sync(0xffffffffu, ay, off); if (take) ay += v;
      v = __shfl_down_sync(0xffffffffu, az, off); if (take) az += v;
      if (JERK) {
        v = __shfl_down_sync(0xffffffffu, jx, off); if (take) jx += v;
        v = __shfl_down_sync(0xffffffffu, jy, off); if (take) jy += v;
        v = __shfl_down_sync(0xffffffffu, jz, off); if (take) jz += v;
      }
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
  double invr = rsqrt(r2 + b.eps2), invr2 = invr * invr;
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
                                                        const TcBodies b, const TcCells c, TcOut out,
                                                        const unsigned* ntldev = nullptr, int nsplit = 1,
                                                        double* __restrict__ part = nullptr, int pstride = 0) {
  // Work item k: target leaf k / nsplit, chunk k % nsplit of its source-cell list.  With
  // nsplit == 1 the item adds into out; otherwise it stores its partial sums in
  // part[(chunk * NC + component) * pstride + body] for k_p2p_join (few target leaves: more
  // warps than leaves, the chunks folded afterwards in a fixed order).
  if (ntldev) ntl = (int)*ntldev;  // device-sized launch (graph)
  constexpr int NC = JERK ? 7 : 4;
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long nitem = (long long)ntl * nsplit;
  for (long long k = (long long)blockIdx.x * kP2PWarps + w; k < nitem; k += (long long)gridDim.x * kP2PWarps) {
    const int kk = (int)(k / nsplit), chunk = (int)(k % nsplit);
    int t = tlist[kk];
    if (!c.has_sink[t]) continue;
    int tb = c.begin[t], nt = c.nbody[t];
    const int sb0 = tstart[t], len = tstart[t + 1] - sb0;
    const int sb = sb0 + (int)((long long)len * chunk / nsplit);
    const int se = sb0 + (int)((long long)len * (chunk + 1) / nsplit);
    for (int t0 = 0; t0 < nt; t0 += 32) {
      // up to 32 targets per pass; a last pass of r <= 16 targets runs floor(32 / r) lane
      // groups of r lanes, each over every ng-th source
      const int r = min(32, nt - t0);
      const int gsz = r > 16 ? 32 : r, ng = 32 / gsz;
      const int grp = lane / gsz, ti = lane % gsz;
      int i = tb + t0 + ti;
      bool vi = grp < ng && (t0 + ti) < nt;
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
      a.add_groups(gsz, ng, grp);
      if (vi && grp == 0) {
        if (nsplit > 1) {
          double* pp = part + (size_t)chunk * NC * pstride + i;
          pp[0] = a.pot;
          pp[(size_t)pstride] = a.ax;
          pp[2 * (size_t)pstride] = a.ay;
          pp[3 * (size_t)pstride] = a.az;
          if (JERK) {
            pp[4 * (size_t)pstride] = a.jx;
            pp[5 * (size_t)pstride] = a.jy;
            pp[6 * (size_t)pstride] = a.jz;
          }
        } else if (b.flags[i] & 1) {
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
}

// Folds the nsplit chunk partials of k_p2p (chunk 0 first) into the sink bodies of each target
// leaf: one warp per leaf, one lane per body.
template <bool JERK>
__global__ void __launch_bounds__(kP2PWarps * 32) k_p2p_join(const int* __restrict__ tlist, int ntl,
                                                             const TcBodies b, const TcCells c, TcOut out,
                                                             int nsplit, const double* __restrict__ part,
                                                             int pstride, const unsigned* ntldev = nullptr) {
  if (ntldev) ntl = (int)*ntldev;  // device-sized launch (graph)
  constexpr int NC = JERK ? 7 : 4;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int k = blockIdx.x * kP2PWarps + w; k < ntl; k += gridDim.x * kP2PWarps) {
    const int t = tlist[k];
    if (!c.has_sink[t]) continue;
    const int tb = c.begin[t], nt = c.nbody[t];
    for (int u = lane; u < nt; u += 32) {
      const int i = tb + u;
      if (!(b.flags[i] & 1)) continue;
      double v[NC];
#pragma unroll
      for (int q = 0; q < NC; q++) v[q] = 0.0;
      for (int ch = 0; ch < nsplit; ch++) {
        const double* pp = part + (size_t)ch * NC * pstride + i;
#pragma unroll
        for (int q = 0; q < NC; q++) v[q] += pp[(size_t)q * pstride];
      }
      out.pot[i] += v[0];
      out.ax[i] += v[1];
      out.ay[i] += v[2];
      out.az[i] += v[3];
      if (JERK) {
        out.jx[i] += v[4];
        out.jy[i] += v[5];
        out.jz[i] += v[6];
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

// FP64 direct sums at selected bodies: the judge of the selector, and tc_direct_sums.  Block
// (c, g) takes the source chunk c and up to 256 targets (one per thread, group g); sources pass
// through shared memory in tiles, so every body is read once per block.
// part[(k * nchunk + c) * 8 + q] = chunk c's (pot, ax, ay, az, jx, jy, jz) of target k.
constexpr int kJudgeTile = 256;
template <bool JERK>
__global__ void __launch_bounds__(kJudgeTile) k_direct_targets(int n, int nt, int nchunk, const int* __restrict__ tgt,
                                                               const TcBodies b, double* __restrict__ part) {
  __shared__ double sx[kJudgeTile], sy[kJudgeTile], sz[kJudgeTile], sm[kJudgeTile];
  __shared__ double su[JERK ? kJudgeTile : 1], sv[JERK ? kJudgeTile : 1], sw[JERK ? kJudgeTile : 1];
  const int c = blockIdx.x, k = blockIdx.y * kJudgeTile + threadIdx.x;
  const int chunk = (n + nchunk - 1) / nchunk;
  const int j0 = c * chunk, j1 = min(n, j0 + chunk);
  const int i = k < nt ? tgt[k] : 0;
  const double xi = b.x[i], yi = b.y[i], zi = b.z[i];
  const double ui = JERK ? b.vx[i] : 0.0, vi = JERK ? b.vy[i] : 0.0, wi = JERK ? b.vz[i] : 0.0;
  double pot = 0.0, ax = 0.0, ay = 0.0, az = 0.0, jx = 0.0, jy = 0.0, jz = 0.0;
  for (int t0 = j0; t0 < j1; t0 += kJudgeTile) {
    const int j = t0 + threadIdx.x;
    __syncthreads();
    if (j < j1) {
      sx[threadIdx.x] = b.x[j];
      sy[threadIdx.x] = b.y[j];
      sz[threadIdx.x] = b.z[j];
      sm[threadIdx.x] = (b.flags[j] & 2) ? b.m[j] : 0.0;
      if (JERK) {
        su[threadIdx.x] = b.vx[j];
        sv[threadIdx.x] = b.vy[j];
        sw[threadIdx.x] = b.vz[j];
      }
    }
    __syncthreads();
    const int cnt = min(kJudgeTile, j1 - t0);
    for (int q = 0; q < cnt; q++) {
      const double dx = sx[q] - xi, dy = sy[q] - yi, dz = sz[q] - zi;
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 > 0.0) {
        const double invr = rsqrt(r2 + b.eps2), invr2 = invr * invr;
        const double f = sm[q] * invr;
        pot += f;
        const double f3 = f * invr2;
        ax += dx * f3;
        ay += dy * f3;
        az += dz * f3;
        if (JERK) {
          const double du = su[q] - ui, dv = sv[q] - vi, dw = sw[q] - wi;
          const double g = -3.0 * f3 * invr2 * (dx * du + dy * dv + dz * dw);
          jx += du * f3 + dx * g;
          jy += dv * f3 + dy * g;
          jz += dw * f3 + dz * g;
        }
      }
    }
  }
  if (k < nt) {
    double* o = part + ((size_t)k * nchunk + c) * 8;
    o[0] = pot; o[1] = ax; o[2] = ay; o[3] = az; o[4] = jx; o[5] = jy; o[6] = jz;
  }
}

// judge: out[k] = {direct pot, ax, ay, az (chunks summed in order), evaluated ax, ay, az}
__global__ void k_direct_targets_sum(int nt, int nchunk, const int* __restrict__ tgt, const double* __restrict__ part,
                                     TcOut ev, double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nt) return;
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  for (int c = 0; c < nchunk; c++)
    for (int q = 0; q < 4; q++) v[q] += part[((size_t)k * nchunk + c) * 8 + q];
  const int i = tgt[k];
  double* o = out + 7 * (size_t)k;
  o[0] = v[0]; o[1] = v[1]; o[2] = v[2]; o[3] = v[3];
  o[4] = ev.ax[i]; o[5] = ev.ay[i]; o[6] = ev.az[i];
}

// tc_direct_sums: out[k] = direct (pot, ax, ay, az, jx, jy, jz), chunks summed in order
__global__ void k_direct_targets_out(int nt, int nchunk, const double* __restrict__ part, double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nt) return;
  double v[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int c = 0; c < nchunk; c++)
    for (int q = 0; q < 7; q++) v[q] += part[((size_t)k * nchunk + c) * 8 + q];
  for (int q = 0; q < 7; q++) out[7 * (size_t)k + q] = v[q];
}

// Time-step pass of the top-level tree (get_force_and_potential(bodies, true) on the theta
// path): P2P of kernel_fast_lean.h:462-548 (the SIMD / DOUBLE_P2P branch), in FP64.  For a
// target body and one source cell: pot and acc from the cell's sources as in P2P_simple, and
// the pairwise step
//   tau1 = dt/sqrt2 r sqrt(r/mi) / (1 - dtau1/2),  dtau1 = min(1, 3/2 tau1 (d.dv)/r^2)
//   tau2 = dt r/|dv|       / (1 - dtau2/2),  dtau2 = min(1, tau2 (d.dv)/r^2 (1 + mi/(v^2 r)))
// minimised over the cell's bodies; the target's step sum gains 1/min^4.  As in the
// reference, mi starts at the target's mass and accumulates every body of the cell met so far
// (sources or not, self excluded) in the cell's body order, so each lane (one target) walks
// each source cell's bodies in order.  One warp per target cell.
__global__ void __launch_bounds__(kP2PWarps * 32) k_p2p_steps(const int* __restrict__ tlist, int ntl,
                                                              const int* __restrict__ tstart,
                                                              const int* __restrict__ src, const TcBodies b,
                                                              const TcCells c, TcOut out, double dtp,
                                                              double* __restrict__ tsum, int nsplit = 1,
                                                              double* __restrict__ part = nullptr,
                                                              int pstride = 0) {
  // work item k: target leaf k / nsplit, chunk k % nsplit of its source cells (whole cells, so
  // the per-cell time-step terms are unchanged); with nsplit > 1 the chunk's pot, acc and
  // 1/tau^4 sums go to part[(chunk * 5 + component) * pstride + body] for k_p2p_steps_join
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double dts = dtp / 1.41421356237309504880;  // dt_param / M_SQRT2
  const long long nitem = (long long)ntl * nsplit;
  for (long long kw = (long long)blockIdx.x * kP2PWarps + w; kw < nitem; kw += (long long)gridDim.x * kP2PWarps) {
    const int k = (int)(kw / nsplit), chunk = (int)(kw % nsplit);
    const int t = tlist[k];
    if (!c.has_sink[t]) continue;
    const int tb = c.begin[t], nt = c.nbody[t];
    const int sb0 = tstart[t], len = tstart[t + 1] - sb0;
    const int sb = sb0 + (int)((long long)len * chunk / nsplit);
    const int se = sb0 + (int)((long long)len * (chunk + 1) / nsplit);
    for (int t0 = 0; t0 < nt; t0 += 32) {
      const bool vi = t0 + lane < nt;
      const int i = tb + (vi ? t0 + lane : 0);
      const double xi = b.x[i], yi = b.y[i], zi = b.z[i], ui = b.vx[i], vvi = b.vy[i], wi = b.vz[i];
      const double m0 = b.m[i];
      double pot = 0.0, ax = 0.0, ay = 0.0, az = 0.0, ts = 0.0;
      for (int q = sb; q < se; q++) {
        const int sc = src[q];
        const int jb = c.begin[sc], jn = c.nbody[sc];
        double mi = m0, tmin = 1e38;
        for (int j = jb; j < jb + jn; j++) {
          double mj = b.m[j];
          const double dx = b.x[j] - xi, dy = b.y[j] - yi, dz = b.z[j] - zi;
          const double du = b.vx[j] - ui, dv = b.vy[j] - vvi, dw = b.vz[j] - wi;
          double r2 = dx * dx + dy * dy + dz * dz;
          const double v2 = du * du + dv * dv + dw * dw + 1e-20;
          if (!(r2 > 0.0)) {
            mj = 0.0;
            r2 = 1e38;
          }
          mi += mj;
          const double vdotdr2 = (dx * du + dy * dv + dz * dw) / r2;
          const double r = sqrt(r2), invr = 1.0 / r;
          double tau = dts * r * sqrt(r / mi);
          double dtau = 3.0 * tau * vdotdr2 / 2.0;
          if (!(dtau < 1.0)) dtau = 1.0;
          tau /= (1.0 - dtau / 2.0);
          tmin = tau < tmin ? tau : tmin;
          tau = dtp * r / sqrt(v2);
          dtau = tau * vdotdr2 * (1.0 + mi / (v2 * r));
          if (!(dtau < 1.0)) dtau = 1.0;
          tau /= (1.0 - dtau / 2.0);
          tmin = tau < tmin ? tau : tmin;
          mj *= invr;
          if (b.flags[j] & 2) {
            pot += mj;
            const double f = mj * (invr * invr);
            ax += dx * f;
            ay += dy * f;
            az += dz * f;
          }
        }
        tmin *= tmin;
        tmin *= tmin;
        ts += 1.0 / tmin;
      }
      if (vi && nsplit > 1) {
        double* pp = part + (size_t)chunk * 5 * pstride + i;
        pp[0] = pot;
        pp[(size_t)pstride] = ax;
        pp[2 * (size_t)pstride] = ay;
        pp[3 * (size_t)pstride] = az;
        pp[4 * (size_t)pstride] = ts;
      } else if (vi && (b.flags[i] & 1)) {
        out.pot[i] += pot;
        out.ax[i] += ax;
        out.ay[i] += ay;
        out.az[i] += az;
        tsum[i] += ts;
      }
    }
  }
}

// Folds the chunks of k_p2p_steps (chunk 0 first) into the sink bodies of each target leaf.
__global__ void __launch_bounds__(kP2PWarps * 32) k_p2p_steps_join(const int* __restrict__ tlist, int ntl,
                                                                   const TcBodies b, const TcCells c, TcOut out,
                                                                   double* __restrict__ tsum, int nsplit,
                                                                   const double* __restrict__ part, int pstride) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int k = blockIdx.x * kP2PWarps + w; k < ntl; k += gridDim.x * kP2PWarps) {
    const int t = tlist[k];
    if (!c.has_sink[t]) continue;
    const int tb = c.begin[t], nt = c.nbody[t];
    for (int u = lane; u < nt; u += 32) {
      const int i = tb + u;
      if (!(b.flags[i] & 1)) continue;
      double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
      for (int ch = 0; ch < nsplit; ch++) {
        const double* pp = part + (size_t)ch * 5 * pstride + i;
#pragma unroll
        for (int q = 0; q < 5; q++) v[q] += pp[(size_t)q * pstride];
      }
      out.pot[i] += v[0];
      out.ax[i] += v[1];
      out.ay[i] += v[2];
      out.az[i] += v[3];
      tsum[i] += v[4];
    }
  }
}

// one array, Morton order -> caller order
__global__ void k_scatter_one(int n, const int* __restrict__ perm, const double* __restrict__ s,
                              double* __restrict__ d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) d[perm[i]] = s[i];
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
// k_p2p_mixed: the mixed-precision near field.
//
// One warp per target leaf, one target per lane; a last pass of r <= 16 targets runs
// floor(32 / r) lane groups, each over every ng-th source pair of each tile (so small leaves
// still fill the warp).  A tile takes the next 32 bodies of the target's source cells read as
// one sequence, so small source leaves still fill it.
//
// Arithmetic.  Sources are staged per 32-source tile as FP32 (hi, lo) pairs of positions and of
// masses, formed in FP64 once per evaluation (k_body_f32), so dx = (xj_hi - xi_hi) + (xj_lo -
// xi_lo) carries one rounding even for close pairs (the hi parts of neighbours subtract exactly).  Each lane evaluates two
// sources at once with the packed FP32x2 instructions of sm_100 (FADD2/FMUL2/FFMA2: one issue
// for two pairs); the tile stores the two sources' fields side by side so one 16-byte
// broadcast load feeds both halves.  1/r is the hardware estimate refined by one Newton
// step; each tile's FP32 sums are folded into (hi, lo) accumulators by a two-sum; the final
// sums are FP64.
//
// Accuracy.  The FP32 pair terms carry a few units of 2^-24 each, and so does their per-tile
// FP32 sum -- relative to the largest term in the sum.  A term far larger than the target's
// acceleration would leave an error far larger than the FMM's own.  So every pair whose
// strength m / r^2 exceeds tau = excl_frac |a_far| (the target's far-field acceleration,
// which the downward pass has already written into out) is left out of the FP32 sums and
// recorded; after the loop the recorded pairs are added in FP64.  A lane with more than kP2PRec
// strong pairs (a zero far field makes every pair strong) goes over its sources a second time,
// in the same tiles and lane groups, and adds every strong pair in FP64 (the same FP32 test
// decides).
// ---------------------------------------------------------------------------------------
constexpr int kP2PRec = 16;
// strong-pair threshold: pairs with m / r^2 above this fraction of the far-field acceleration
// are summed in FP64
constexpr float kP2PExclFrac = 1e-2f;

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

// FP32 (hi, lo) split of x - c
__device__ __forceinline__ void tc_split(double x, double c, float& h, float& l) {
  double d = x - c;
  h = (float)d;
  l = (float)(d - (double)h);
}

__device__ __forceinline__ float2 tc_f2(float a) { return make_float2(a, a); }

// the hardware 1/sqrt estimate (inputs here are never subnormal: r2 + eps2 of a pair that is
// kept, or 0 for a pair that is dropped)
__device__ __forceinline__ float tc_rsqrt_est(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// A tile: 32 sources as 16 pairs (2p, 2p + 1); field group g of pair p is one float4 holding
// both sources' values of two fields: g0 (xh, yh), g1 (zh, xl), g2 (yl, zl), g3 (mh, ml),
// g4 (vx, vy), g5 (vz, -), each as (source 2p, source 2p + 1).
constexpr int kP2PGroups = 6;
struct TcTile {
  float4 g[kP2PGroups][16];
};

// one target's FP32 state; the target's fields are negated and duplicated into both halves
template <bool JERK>
struct TcMixP {
  float2 nxh, nyh, nzh, nxl, nyl, nzl, nvx, nvy, nvz, eps2;
  float tau;
  float2 sp, sx, sy, sz, qx, qy, qz;  // this tile's sums, one per half
  TcF2 pot, ax, ay, az, jx, jy, jz;   // compensated totals
};

// The FP32 splits of every body, once per evaluation: positions as (hi, lo) pairs of the
// coordinates themselves (the difference (xj_hi - xi_hi) + (xj_lo - xi_lo) of two bodies keeps
// one rounding, the hi parts of neighbours subtracting exactly), the source mass likewise (0 for
// a non-source), velocities rounded.  Each tile then reads three 16-byte words per source.
template <bool JERK>
__global__ void k_body_f32(int n, const TcBodies b) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  float xh, yh, zh, xl, yl, zl, mh, ml;
  tc_split(b.x[j], 0.0, xh, xl);
  tc_split(b.y[j], 0.0, yh, yl);
  tc_split(b.z[j], 0.0, zh, zl);
  tc_split((b.flags[j] & 2) ? b.m[j] : 0.0, 0.0, mh, ml);
  b.f32[3 * (size_t)j] = make_float4(xh, yh, zh, mh);
  b.f32[3 * (size_t)j + 1] = make_float4(xl, yl, zl, ml);
  b.f32[3 * (size_t)j + 2] =
      JERK ? make_float4((float)b.vx[j], (float)b.vy[j], (float)b.vz[j], 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
}

// stage source j (or a zero-mass source at the origin when j < 0) at tile slot l
template <bool JERK>
__device__ __forceinline__ void tc_tile_put(TcTile& T, int l, const TcBodies& b, int j, double, double, double) {
  float xh = 0.f, yh = 0.f, zh = 0.f, xl = 0.f, yl = 0.f, zl = 0.f, mh = 0.f, ml = 0.f, vx = 0.f, vy = 0.f, vz = 0.f;
  if (j >= 0) {
    const float4 h = b.f32[3 * (size_t)j], lo = b.f32[3 * (size_t)j + 1];
    xh = h.x; yh = h.y; zh = h.z; mh = h.w;
    xl = lo.x; yl = lo.y; zl = lo.z; ml = lo.w;
    if (JERK) {
      const float4 v = b.f32[3 * (size_t)j + 2];
      vx = v.x; vy = v.y; vz = v.z;
    }
  }
  const int p = l >> 1, h = l & 1;
  float* g0 = reinterpret_cast<float*>(&T.g[0][p]);
  float* g1 = reinterpret_cast<float*>(&T.g[1][p]);
  float* g2 = reinterpret_cast<float*>(&T.g[2][p]);
  float* g3 = reinterpret_cast<float*>(&T.g[3][p]);
  g0[h] = xh; g0[2 + h] = yh;
  g1[h] = zh; g1[2 + h] = xl;
  g2[h] = yl; g2[2 + h] = zl;
  g3[h] = mh; g3[2 + h] = ml;
  if (JERK) {
    float* g4 = reinterpret_cast<float*>(&T.g[4][p]);
    float* g5 = reinterpret_cast<float*>(&T.g[5][p]);
    g4[h] = vx; g4[2 + h] = vy;
    g5[h] = vz;
  }
}

// The FP32 geometry of source pair p: differences, 1/r, m/r, and whether each half's m/r^2
// exceeds the target's threshold.  The only definition of "strong": the main loop and the
// overflow pass both call it.
template <bool JERK>
__device__ __forceinline__ void tc_mixp_geom(const TcMixP<JERK>& T, const TcTile& S, int p, float2& dx, float2& dy,
                                             float2& dz, float2& ri, float2& f0, bool& sa, bool& sb) {
  const float4 g0 = S.g[0][p], g1 = S.g[1][p], g2 = S.g[2][p], g3 = S.g[3][p];
  dx = __fadd2_rn(__fadd2_rn(make_float2(g0.x, g0.y), T.nxh), __fadd2_rn(make_float2(g1.z, g1.w), T.nxl));
  dy = __fadd2_rn(__fadd2_rn(make_float2(g0.z, g0.w), T.nyh), __fadd2_rn(make_float2(g2.x, g2.y), T.nyl));
  dz = __fadd2_rn(__fadd2_rn(make_float2(g1.x, g1.y), T.nzh), __fadd2_rn(make_float2(g2.z, g2.w), T.nzl));
  const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
  const float2 rs = __fadd2_rn(r2, T.eps2);  // softened (eps2 = 0: unchanged)
  const float2 y = make_float2(tc_rsqrt_est(rs.x), tc_rsqrt_est(rs.y));
  // one Newton step: ri = y + (y / 2) (1 - rs y^2), written as y - (y / 2) (rs y^2 - 1)
  const float2 e = __ffma2_rn(__fmul2_rn(rs, y), y, tc_f2(-1.f));
  ri = __ffma2_rn(__fmul2_rn(y, tc_f2(-0.5f)), e, y);
  ri.x = r2.x > 0.f ? ri.x : 0.f;  // coincident bodies (and the target itself) add nothing
  ri.y = r2.y > 0.f ? ri.y : 0.f;
  f0 = __ffma2_rn(make_float2(g3.z, g3.w), ri, __fmul2_rn(make_float2(g3.x, g3.y), ri));
  const float2 st = __fmul2_rn(f0, ri);
  sa = st.x > T.tau;
  sb = st.y > T.tau;
}

template <bool JERK>
__device__ __forceinline__ void tc_mixp_pair(TcMixP<JERK>& T, const TcTile& S, int p, bool& sa, bool& sb) {
  float2 dx, dy, dz, ri, f0;
  tc_mixp_geom<JERK>(T, S, p, dx, dy, dz, ri, f0, sa, sb);
  if (sa) f0.x = 0.f;  // strong: summed in FP64 instead
  if (sb) f0.y = 0.f;
  const float2 ri2 = __fmul2_rn(ri, ri);
  const float2 f = __fmul2_rn(f0, ri2);
  T.sp = __fadd2_rn(T.sp, f0);
  T.sx = __ffma2_rn(dx, f, T.sx);
  T.sy = __ffma2_rn(dy, f, T.sy);
  T.sz = __ffma2_rn(dz, f, T.sz);
  if (JERK) {
    const float4 g4 = S.g[4][p];
    const float2 g5 = *reinterpret_cast<const float2*>(&S.g[5][p]);
    const float2 dvx = __fadd2_rn(make_float2(g4.x, g4.y), T.nvx);
    const float2 dvy = __fadd2_rn(make_float2(g4.z, g4.w), T.nvy);
    const float2 dvz = __fadd2_rn(g5, T.nvz);
    // g = -f / r^2 * 3 (d . dv)
    const float2 vrn = __fmul2_rn(tc_f2(-3.f), __ffma2_rn(dx, dvx, __ffma2_rn(dy, dvy, __fmul2_rn(dz, dvz))));
    const float2 g = __fmul2_rn(__fmul2_rn(f, ri2), vrn);
    T.qx = __ffma2_rn(dx, g, __ffma2_rn(dvx, f, T.qx));
    T.qy = __ffma2_rn(dy, g, __ffma2_rn(dvy, f, T.qy));
    T.qz = __ffma2_rn(dz, g, __ffma2_rn(dvz, f, T.qz));
  }
}

template <bool JERK>
__device__ __forceinline__ void tc_mixp_fold(TcMixP<JERK>& T) {
  T.pot.add(__fadd_rn(T.sp.x, T.sp.y));
  T.ax.add(__fadd_rn(T.sx.x, T.sx.y));
  T.ay.add(__fadd_rn(T.sy.x, T.sy.y));
  T.az.add(__fadd_rn(T.sz.x, T.sz.y));
  if (JERK) {
    T.jx.add(__fadd_rn(T.qx.x, T.qx.y));
    T.jy.add(__fadd_rn(T.qy.x, T.qy.y));
    T.jz.add(__fadd_rn(T.qz.x, T.qz.y));
  }
  T.sp = T.sx = T.sy = T.sz = T.qx = T.qy = T.qz = tc_f2(0.f);
}

template <bool JERK>
__device__ __forceinline__ void tc_mixp_init(TcMixP<JERK>& T, const TcBodies& b, const TcOut& out, int i, bool v,
                                             double Xc, double Yc, double Zc, float excl_frac) {
  float xh = 0.f, yh = 0.f, zh = 0.f, xl = 0.f, yl = 0.f, zl = 0.f, vx = 0.f, vy = 0.f, vz = 0.f;
  T.tau = 0.f;
  if (v) {
    const float4 h = b.f32[3 * (size_t)i], lo = b.f32[3 * (size_t)i + 1];
    xh = h.x; yh = h.y; zh = h.z;
    xl = lo.x; yl = lo.y; zl = lo.z;
    if (JERK) {
      const float4 w = b.f32[3 * (size_t)i + 2];
      vx = w.x; vy = w.y; vz = w.z;
    }
    const double a = sqrt(out.ax[i] * out.ax[i] + out.ay[i] * out.ay[i] + out.az[i] * out.az[i]);
    T.tau = (float)(excl_frac * a);
  }
  T.nxh = tc_f2(-xh); T.nyh = tc_f2(-yh); T.nzh = tc_f2(-zh);
  T.nxl = tc_f2(-xl); T.nyl = tc_f2(-yl); T.nzl = tc_f2(-zl);
  T.nvx = tc_f2(-vx); T.nvy = tc_f2(-vy); T.nvz = tc_f2(-vz);
  T.eps2 = tc_f2((float)b.eps2);
  T.sp = T.sx = T.sy = T.sz = T.qx = T.qy = T.qz = tc_f2(0.f);
  T.pot = T.ax = T.ay = T.az = T.jx = T.jy = T.jz = TcF2{0.f, 0.f};
}

template <bool JERK>
__device__ __forceinline__ TcAcc<JERK> tc_mixp_total(const TcMixP<JERK>& T) {
  TcAcc<JERK> a;
  a.pot = T.pot.val(); a.ax = T.ax.val(); a.ay = T.ay.val(); a.az = T.az.val();
  a.jx = T.jx.val(); a.jy = T.jy.val(); a.jz = T.jz.val();
  return a;
}

// The next tile of a target's sources, taken as one sequence of bodies (its source cells'
// bodies one after the other), so a tile holds 32 sources even where the source leaves are
// small.  (q, off) is the warp-uniform cursor: the next source cell and the next body in it.
// The first body and body count of cells q0 + l are held by lane l (cjb, cjn), reloaded 32 cells
// at a time.  Returns the tile's count; lane l gets the body index of slot l (-1 past the count).
__device__ __forceinline__ void tc_src_cells(const int* __restrict__ src, const TcCells& c, int q0, int se, int lane,
                                             int& cjb, int& cjn) {
  cjb = 0;
  cjn = 0;
  if (q0 + lane < se) {
    const int s = src[q0 + lane];
    cjb = c.begin[s];
    cjn = c.nbody[s];
  }
}
__device__ __forceinline__ int tc_next_tile(const int* __restrict__ src, const TcCells& c, int se, int& q, int& off,
                                            int& q0, int& cjb, int& cjn, int lane, int& myj) {
  int fill = 0;
  myj = -1;
  while (fill < 32 && q < se) {
    if (q >= q0 + 32) {
      q0 = q;
      tc_src_cells(src, c, q0, se, lane, cjb, cjn);
    }
    const int jb = __shfl_sync(0xffffffffu, cjb, q - q0), jn = __shfl_sync(0xffffffffu, cjn, q - q0);
    const int take = min(32 - fill, jn - off);
    if (lane >= fill && lane < fill + take) myj = jb + off + lane - fill;
    fill += take;
    off += take;
    if (off >= jn) {
      q++;
      off = 0;
    }
  }
  return fill;
}

// Seven CTAs (28 warps) per SM: the register cap (73) spills a few words per thread, and the
// occupancy still wins at N = 4M (79.6 ms against 84.2 ms at five CTAs, 81.2 at six; the compensated
// totals kept in shared memory instead of registers measured no better).
template <bool JERK>
__global__ void __launch_bounds__(kP2PWarps * 32, 7) k_p2p_mixed(const int* __restrict__ tlist, int ntl,
                                                                 const int* __restrict__ tstart,
                                                                 const int* __restrict__ src, const TcBodies b,
                                                                 const TcCells c, TcOut out, float excl_frac,
                                                                 const unsigned* ntldev = nullptr) {
  if (ntldev) ntl = (int)*ntldev;  // device-sized launch (graph)
  // per warp: the source tile and each lane's recorded strong pairs
  __shared__ TcTile tile[kP2PWarps];
  __shared__ int tj[kP2PWarps][32];  // body index of each tile slot
  __shared__ int rec[kP2PWarps][kP2PRec][32];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  TcTile& TL = tile[w];
  for (int k = blockIdx.x * kP2PWarps + w; k < ntl; k += gridDim.x * kP2PWarps) {
    const int t = tlist[k];
    if (!c.has_sink[t]) continue;
    const double Xc = c.X[t], Yc = c.Y[t], Zc = c.Z[t];
    const int tb = c.begin[t], nt = c.nbody[t];
    const int sb = tstart[t], se = tstart[t + 1];
    for (int t0 = 0; t0 < nt; t0 += 32) {
      // up to 32 targets per pass; a last pass of r <= 16 targets runs floor(32 / r) lane
      // groups of r lanes, each over every ng-th source pair
      const int r = min(32, nt - t0);
      const int gsz = r > 16 ? 32 : r, ng = 32 / gsz;
      const int grp = lane / gsz, ti = lane % gsz;
      const bool act = grp < ng && ti < r;
      const int i = tb + t0 + ti;
      int nrl = 0;  // strong pairs this lane met
      TcMixP<JERK> A;
      tc_mixp_init<JERK>(A, b, out, i, act, Xc, Yc, Zc, excl_frac);
      int q0 = sb, cjb, cjn;
      tc_src_cells(src, c, q0, se, lane, cjb, cjn);
      for (int q = sb, off = 0; q < se;) {
        int myj;
        const int cnt = tc_next_tile(src, c, se, q, off, q0, cjb, cjn, lane, myj), np = (cnt + 1) >> 1;
        __syncwarp();
        if (lane < 2 * np) tc_tile_put<JERK>(TL, lane, b, myj, Xc, Yc, Zc);
        tj[w][lane] = myj;
        __syncwarp();
        if (act) {
          for (int p = grp; p < np; p += ng) {
            bool sa, sbb;
            tc_mixp_pair<JERK>(A, TL, p, sa, sbb);
            if (sa | sbb) {
              if (sa) {
                if (nrl < kP2PRec) rec[w][nrl][lane] = tj[w][2 * p];
                nrl++;
              }
              if (sbb) {
                if (nrl < kP2PRec) rec[w][nrl][lane] = tj[w][2 * p + 1];
                nrl++;
              }
            }
          }
        }
        tc_mixp_fold<JERK>(A);
      }
      TcAcc<JERK> a = tc_mixp_total<JERK>(A);
      const bool ovf = act && nrl > kP2PRec;
      if (__any_sync(0xffffffffu, ovf)) {
        // a lane whose list overflowed goes over its own sources again (the same tiles, the same
        // lane groups) and adds every strong pair in FP64; the other lanes only stage the tiles
        const double xi = ovf ? b.x[i] : 0.0, yi = ovf ? b.y[i] : 0.0, zi = ovf ? b.z[i] : 0.0;
        const double vxi = (JERK && ovf) ? b.vx[i] : 0.0, vyi = (JERK && ovf) ? b.vy[i] : 0.0,
                     vzi = (JERK && ovf) ? b.vz[i] : 0.0;
        q0 = sb;
        tc_src_cells(src, c, q0, se, lane, cjb, cjn);
        for (int q = sb, off = 0; q < se;) {
          int myj;
          const int cnt = tc_next_tile(src, c, se, q, off, q0, cjb, cjn, lane, myj), np = (cnt + 1) >> 1;
          __syncwarp();
          if (lane < 2 * np) tc_tile_put<JERK>(TL, lane, b, myj, Xc, Yc, Zc);
          tj[w][lane] = myj;
          __syncwarp();
          if (ovf) {
            for (int p = grp; p < np; p += ng) {
              float2 dx, dy, dz, ri, f0;
              bool sa, sbb;
              tc_mixp_geom<JERK>(A, TL, p, dx, dy, dz, ri, f0, sa, sbb);
              if (sa) tc_p2p_one<JERK>(xi, yi, zi, vxi, vyi, vzi, b, tj[w][2 * p], a);
              if (sbb) tc_p2p_one<JERK>(xi, yi, zi, vxi, vyi, vzi, b, tj[w][2 * p + 1], a);
            }
          }
        }
      }
      // each lane adds its own recorded strong pairs in FP64
      if (act && !ovf && nrl > 0) {
        const double xi = b.x[i], yi = b.y[i], zi = b.z[i];
        const double vxi = JERK ? b.vx[i] : 0.0, vyi = JERK ? b.vy[i] : 0.0, vzi = JERK ? b.vz[i] : 0.0;
        for (int e = 0; e < nrl; e++) tc_p2p_one<JERK>(xi, yi, zi, vxi, vyi, vzi, b, rec[w][e][lane], a);
      }
      a.add_groups(gsz, ng, grp);
      if (act && grp == 0 && (b.flags[i] & 1)) {
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
