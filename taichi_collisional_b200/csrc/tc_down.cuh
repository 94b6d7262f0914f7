// Downward pass on the device: L2L one level at a time (parents first), then L2P per leaf.
// Restates downwardPass (traverse_eager.h:326-346), L2L (kernel_fast_lean.h:941-987; Ldot
// taichi_with_jerks/kernel_fast_lean.h:1001-1058) and L2P (kernel_fast_lean.h:989-1032;
// jerk :1060-1128): only degrees n <= 1 of the shifted local are evaluated,
//   p += Re Phi[0,0];  F -= (Re Phi[1,1], Im Phi[1,1], Re Phi[1,0])
//   J -= (Re Phidot[1,1], Im Phidot[1,1], Re Phidot[1,0]),  Phidot = L conj(Gdot) + Ldot conj(G)
#pragma once
#include "tc_upward.cuh"

namespace tc {

// L2L into cell ci (level >= 1) from its parent; one warp per cell.  The parent's local (and
// Ldot) is staged in shared memory as complex full storage.
template <int P, bool JERK>
__global__ void __launch_bounds__(TcTransW<P>::W * 32) k_l2l_level(int l, TcCells c,
                                                                   const int* __restrict__ lv_start,
                                                                   const int* __restrict__ lv_count) {
  constexpr int W = TcTransW<P>::W;
  constexpr int NT = (P + 1) * (P + 1);
  constexpr int NOUT = (P + 1) * (P + 2) / 2;
  constexpr int PER = (NOUT + 31) / 32;
  __shared__ cd sG[W][NT];
  __shared__ cd sL[W][NT];
  __shared__ cd sLd[W][JERK ? NT : 1];
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int cnt = lv_count[l], st = lv_start[l];
  for (int k = blockIdx.x * W + w; k < cnt; k += gridDim.x * W) {
    int ci = st + k;
    if (!c.has_sink[ci]) continue;
    int pa = c.parent[ci];
    cd* G = sG[w];
    cd* SL = sL[w];
    cd* SLd = sLd[w];
    const double* Lp = c.L + (size_t)pa * NT;
    const double* Ldp = JERK ? c.Ld + (size_t)pa * NT : nullptr;
    for (int i = lane; i < NT; i += 32) {
      int n = 0;
      while ((n + 1) * (n + 1) <= i) n++;
      SL[i] = tc_r2c(Lp, n, i - n * n - n);
      if (JERK) SLd[i] = tc_r2c(Ldp, n, i - n * n - n);
    }
    tc_warp_gnm_smem<P>(c.X[pa] - c.X[ci], c.Y[pa] - c.Y[ci], c.Z[pa] - c.Z[ci], G);  // ends with __syncwarp
    double* Lc = c.L + (size_t)ci * NT;
    double* Ldc = JERK ? c.Ld + (size_t)ci * NT : nullptr;
#pragma unroll
    for (int q = 0; q < PER; q++) {
      int o = lane + 32 * q;
      if (o >= NOUT) break;
      int n = 0;
      while ((n + 1) * (n + 2) / 2 <= o) n++;
      int m = o - n * (n + 1) / 2;
      cd s = mk(0, 0), sd = mk(0, 0);
      for (int kk = 0; kk <= P - n; kk++) {
        const int nn = n + kk, base = nn * nn + nn + m;  // local (n + kk, m + ll)
        for (int ll = -kk; ll <= kk; ll++) {
          cd g = conj(G[kk * kk + kk + ll]);
          s += SL[base + ll] * g;
          if (JERK) sd += SLd[base + ll] * g;
        }
      }
      int is = n * n + n;
      Lc[is + m] += s.x;
      if (m > 0) Lc[is - m] += s.y;
      if (JERK) {
        Ldc[is + m] += sd.x;
        if (m > 0) Ldc[is - m] += sd.y;
      }
    }
    __syncwarp();
  }
}

struct TcOut {
  double *pot, *ax, *ay, *az, *jx, *jy, *jz;  // Morton order
};

// acceleration of one body from a local expansion held as complex full storage `sl`
// (dX = cell centre - body), the non-jerk part of the L2P below
template <int P>
__device__ __forceinline__ void tc_l2p_acc(const cd* sl, double dx, double dy, double dz, double* a) {
  double r2 = dx * dx + dy * dy + dz * dz;
  cd p10 = mk(0, 0), p11 = mk(0, 0);
  for (int m = 0; m <= P; m++) {
    double sgn = (m & 1) ? -1.0 : 1.0;
    cd d0 = mk(1, 0);
    for (int j = 1; j <= m; j++) d0 = d0 * mk(dx / (2 * j), dy / (2 * j));
    TcCol col;
    col.init(m, d0);
#pragma unroll
    for (int n = 0; n <= P; n++) {
      cd gb = col.step(n, dz, r2);
      if (n >= m && n <= P - 1) {
        cd cgp = conj(gb), cgn = sgn * gb;
        int k1 = (n + 1) * (n + 1) + (n + 1);
        p10 += sl[k1 + m] * cgp;
        p11 += sl[k1 + 1 + m] * cgp;
        if (m > 0) {
          p10 += sl[k1 - m] * cgn;
          p11 += sl[k1 + 1 - m] * cgn;
        }
      }
    }
  }
  a[0] = -p11.x;
  a[1] = -p11.y;
  a[2] = -p10.x;
}

// L2P for every leaf; one warp per leaf, one lane per body.  The solid-harmonic columns use the
// tabulated recurrence of the P2M (TcColTab, tc_col_next).
template <int P, bool JERK>
__global__ void __launch_bounds__(kUpWarps * 32) k_l2p(const int* __restrict__ leaves, int nleaf, const TcBodies b,
                                                       const TcCells c, TcOut out,
                                                       const unsigned* nldev = nullptr) {
  constexpr int NT = (P + 1) * (P + 1);
  __shared__ cd sL[kUpWarps][NT];
  __shared__ cd sLd[kUpWarps][JERK ? NT : 1];
  __shared__ TcColTab<P> tab;
  tab.fill();
  __syncthreads();
  if (nldev) nleaf = (int)*nldev;  // device-sized launch (graph)
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int k = blockIdx.x * kUpWarps + w; k < nleaf; k += gridDim.x * kUpWarps) {
    int ci = leaves[k];
    if (!c.has_sink[ci]) continue;
    const double* L = c.L + (size_t)ci * NT;
    const double* Ld = JERK ? c.Ld + (size_t)ci * NT : nullptr;
    for (int i = lane; i < NT; i += 32) {
      int n = 0;
      while ((n + 1) * (n + 1) <= i) n++;
      int m = i - n * n - n;
      sL[w][i] = tc_r2c(L, n, m);
      if (JERK) sLd[w][i] = tc_r2c(Ld, n, m);
    }
    __syncwarp();
    const cd* sl = sL[w];
    const cd* sld = sLd[w];
    double X = c.X[ci], Y = c.Y[ci], Z = c.Z[ci];
    int beg = c.begin[ci], nb = c.nbody[ci];
    for (int i = beg + lane; i < beg + nb; i += 32) {
      if (!(b.flags[i] & 1)) continue;
      double dx = X - b.x[i], dy = Y - b.y[i], dz = Z - b.z[i];
      double r2 = dx * dx + dy * dy + dz * dz;
      cd p00 = mk(0, 0), p10 = mk(0, 0), p11 = mk(0, 0);
      cd q10 = mk(0, 0), q11 = mk(0, 0);
      cd etad, zd, ksid;
      if (JERK) {
        double vx = -b.vx[i], vy = -b.vy[i], vz = -b.vz[i];
        etad = mk(-vx * 0.5, vy * 0.5);
        zd = mk(vz, 0);
        ksid = mk(vx * 0.5, vy * 0.5);
      }
      // diagonal G[j][j] at j = m - 1, m, m + 1, advanced with the order m
      cd Dm1 = mk(0, 0), D0 = mk(1, 0), Dp1 = mk(dx * tab.H[1], dy * tab.H[1]);
      for (int m = 0; m <= P; m++) {
        const double sgn = (m & 1) ? -1.0 : 1.0;
        const int ca = m > 0 ? m - 1 : 1, cc = m + 1;  // column -1 is -conj(column 1)
        cd A1 = mk(0, 0), A2 = mk(0, 0), B1 = mk(0, 0), B2 = mk(0, 0), C1 = mk(0, 0), C2 = mk(0, 0);
#pragma unroll
        for (int n = 0; n <= P; n++) {
          cd pa, pb, pc;  // G[n-1][m-1], G[n-1][m], G[n-1][m+1]
          if (JERK) {
            pa = m > 0 ? A1 : mk(-C1.x, C1.y);
            pb = B1;
            pc = C1;
            tc_col_next(n == cc, Dp1, C1, C2, tab.A[n][cc], tab.B[n][cc], dz, r2);
            if (m > 0) tc_col_next(n == ca, Dm1, A1, A2, tab.A[n][ca], tab.B[n][ca], dz, r2);
          }
          const cd gb = tc_col_next(n == m, D0, B1, B2, tab.A[n][m], tab.B[n][m], dz, r2);
          if (n >= m) {
            // l = +m and l = -m terms of sum_k,l L[n'+k, m'+l] conj(G[k,l]) at k = n
            cd cgp = conj(gb), cgn = sgn * gb;
            int kk = n * n + n;
            p00 += sl[kk + m] * cgp;
            if (m > 0) p00 += sl[kk - m] * cgn;
            if (n <= P - 1) {
              int k1 = (n + 1) * (n + 1) + (n + 1);
              p10 += sl[k1 + m] * cgp;
              p11 += sl[k1 + 1 + m] * cgp;
              if (m > 0) {
                p10 += sl[k1 - m] * cgn;
                p11 += sl[k1 + 1 - m] * cgn;
              }
            }
            if (JERK && n <= P - 1) {
              cd gd = mk(0, 0);
              if (n >= 1) {
                if (m <= n - 2) gd += pc * etad;
                if (m <= n - 1) gd += pb * zd;
                gd += pa * ksid;
              }
              cd cdp = conj(gd), cdn = sgn * gd;
              int k1 = (n + 1) * (n + 1) + (n + 1);
              q10 += sl[k1 + m] * cdp + sld[k1 + m] * cgp;
              q11 += sl[k1 + 1 + m] * cdp + sld[k1 + 1 + m] * cgp;
              if (m > 0) {
                q10 += sl[k1 - m] * cdn + sld[k1 - m] * cgn;
                q11 += sl[k1 + 1 - m] * cdn + sld[k1 + 1 - m] * cgn;
              }
            }
          }
        }
        Dm1 = D0;
        D0 = Dp1;
        Dp1 = Dp1 * mk(dx * tab.H[m + 2], dy * tab.H[m + 2]);
      }
      out.pot[i] += p00.x;
      out.ax[i] -= p11.x;
      out.ay[i] -= p11.y;
      out.az[i] -= p10.x;
      if (JERK) {
        out.jx[i] -= q11.x;
        out.jy[i] -= q11.y;
        out.jz[i] -= q10.x;
      }
    }
    __syncwarp();
  }
}

}  // namespace tc
