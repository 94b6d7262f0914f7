// Upward pass on the device: the balls of every leaf (one launch), P2M of every leaf (one
// launch), then one launch per tree level (deepest first) for the inner cells, one warp per
// cell.  Restates upwardPass (traverse_eager.h:9-34) with MINIBALL: each cell's expansion centre
// and radius are the smallest ball enclosing its bodies (leaf, kernel_fast_lean.h:707-737)
// or, for an inner cell, the bodies of its leaf children plus 64 t-design points around
// every grandchild (:833-892); R = r_ball + 1e-6.  Then P2M (:745-781) for leaves and M2M
// (:900-938) for inner cells; with jerks also Mdot (taichi_with_jerks/kernel_fast_lean.h:
// 769-817, :950-998).
#pragma once
#include "tc_harmonics.cuh"

namespace tc {

// ---------------------------------------------------------------------------------------
// smallest enclosing ball: pivoting (farthest point, warp-parallel) + exact small solver
// ---------------------------------------------------------------------------------------
struct TcPointSet {
  // children of an inner cell: leaf children give bodies, inner children give 64 points
  // per grandchild.  For a leaf cell: its own bodies.
  int leaf, nseg;
  int seg_start[9];   // prefix of point counts
  int seg_kind[8];    // 0 = bodies [seg_a, seg_a + count), 1 = t-design around cells [seg_a ..)
  int seg_a[8];
  int total;
};

__device__ __forceinline__ double tc_d2(const double* a, const double* b) {
  double x = a[0] - b[0], y = a[1] - b[1], z = a[2] - b[2];
  return x * x + y * y + z * z;
}

// ball through q[0..k-1] with centre in their affine hull; false if degenerate
__device__ bool tc_circumsphere(int k, const double (*q)[3], double* c, double* r2) {
  if (k == 1) {
    c[0] = q[0][0]; c[1] = q[0][1]; c[2] = q[0][2];
    *r2 = 0;
    return true;
  }
  double v[3][3], A[3][3], bb[3], lam[3];
  int d = k - 1;
  for (int i = 0; i < d; i++)
    for (int j = 0; j < 3; j++) v[i][j] = q[i + 1][j] - q[0][j];
  for (int i = 0; i < d; i++) {
    for (int j = 0; j < d; j++) A[i][j] = 2 * (v[i][0] * v[j][0] + v[i][1] * v[j][1] + v[i][2] * v[j][2]);
    bb[i] = v[i][0] * v[i][0] + v[i][1] * v[i][1] + v[i][2] * v[i][2];
  }
  double scale = 0;
  for (int i = 0; i < d; i++) scale = fmax(scale, fabs(A[i][i]));
  for (int col = 0; col < d; col++) {
    int piv = col;
    for (int r = col + 1; r < d; r++)
      if (fabs(A[r][col]) > fabs(A[piv][col])) piv = r;
    if (fabs(A[piv][col]) <= 1e-13 * scale) return false;
    if (piv != col) {
      for (int j = 0; j < d; j++) { double t = A[col][j]; A[col][j] = A[piv][j]; A[piv][j] = t; }
      double t = bb[col]; bb[col] = bb[piv]; bb[piv] = t;
    }
    for (int r = col + 1; r < d; r++) {
      double f = A[r][col] / A[col][col];
      for (int j = col; j < d; j++) A[r][j] -= f * A[col][j];
      bb[r] -= f * bb[col];
    }
  }
  for (int i = d - 1; i >= 0; i--) {
    double s = bb[i];
    for (int j = i + 1; j < d; j++) s -= A[i][j] * lam[j];
    lam[i] = s / A[i][i];
  }
  double off[3] = {0, 0, 0};
  for (int i = 0; i < d; i++)
    for (int j = 0; j < 3; j++) off[j] += lam[i] * v[i][j];
  for (int j = 0; j < 3; j++) c[j] = q[0][j] + off[j];
  *r2 = off[0] * off[0] + off[1] * off[1] + off[2] * off[2];
  return true;
}

// Smallest ball with q on its boundary enclosing the support set s; updates s.  Every subset
// of s (at most 3 points, with q) is one lane's candidate; the warp keeps the valid candidate
// of least radius, ties to the lowest subset index -- the subset a loop over the subsets in
// index order keeps -- and every lane ends with the same result.
__device__ bool tc_mb_small(double (*s)[3], int& ns, const double* q, double* c, double* r2) {
  const int lane = threadIdx.x & 31;
  const int mask = lane;
  double rr = INFINITY, cc[3] = {0, 0, 0};
  bool ok = false;
  if (mask < (1 << ns) && __popc(mask) <= 3) {
    double pts[4][3];
    int k = 0;
    pts[k][0] = q[0]; pts[k][1] = q[1]; pts[k][2] = q[2]; k++;
    for (int i = 0; i < ns; i++)
      if (mask & (1 << i)) { pts[k][0] = s[i][0]; pts[k][1] = s[i][1]; pts[k][2] = s[i][2]; k++; }
    if (tc_circumsphere(k, pts, cc, &rr)) {
      ok = true;
      for (int i = 0; i < ns && ok; i++)
        if (!(mask & (1 << i)) && tc_d2(s[i], cc) > rr * (1 + 1e-13) + 1e-300) ok = false;
    }
  }
  double krr = ok ? rr : INFINITY;
  int km = ok ? mask : 0x7fffffff;
  for (int o = 16; o > 0; o >>= 1) {
    const double orr = __shfl_xor_sync(0xffffffffu, krr, o);
    const int om = __shfl_xor_sync(0xffffffffu, km, o);
    if (orr < krr || (orr == krr && om < km)) { krr = orr; km = om; }
  }
  if (km == 0x7fffffff) return false;
  const int best = km;
  const double bc0 = __shfl_sync(0xffffffffu, cc[0], best), bc1 = __shfl_sync(0xffffffffu, cc[1], best),
               bc2 = __shfl_sync(0xffffffffu, cc[2], best);
  double nsv[4][3];
  int k = 0;
  nsv[k][0] = q[0]; nsv[k][1] = q[1]; nsv[k][2] = q[2]; k++;
  for (int i = 0; i < ns; i++)
    if (best & (1 << i)) { nsv[k][0] = s[i][0]; nsv[k][1] = s[i][1]; nsv[k][2] = s[i][2]; k++; }
  for (int i = 0; i < k; i++) { s[i][0] = nsv[i][0]; s[i][1] = nsv[i][1]; s[i][2] = nsv[i][2]; }
  ns = k;
  c[0] = bc0; c[1] = bc1; c[2] = bc2;
  *r2 = krr;
  return true;
}

// Farthest point from c (largest excess e = |p - c|^2 - r2; ties -> lowest point index).
// Items are bodies or t-design groups (64 points around one grandchild); a group whose
// bounding sphere cannot beat the best excess found so far is skipped.
__device__ __forceinline__ void tc_mb_farthest(const TcPointSet& ps, const TcBodies& b, const TcCells& cl,
                                               const double* td, const double* c, double r2, double& best_e,
                                               int& best_i) {
  int lane = threadIdx.x & 31;
  best_e = 0;
  best_i = 0x7fffffff;
  if (ps.leaf) {
    for (int i = lane; i < ps.total; i += 32) {
      int bi = ps.seg_a[0] + i;
      double p[3] = {b.x[bi], b.y[bi], b.z[bi]};
      double e = tc_d2(p, c) - r2;
      if (e > best_e) { best_e = e; best_i = i; }
    }
  } else {
    for (int s = 0; s < ps.nseg; s++) {
      int cnt = ps.seg_kind[s] == 0 ? ps.seg_start[s + 1] - ps.seg_start[s] : (ps.seg_start[s + 1] - ps.seg_start[s]) >> 6;
      for (int it = lane; it < cnt; it += 32) {
        if (ps.seg_kind[s] == 0) {
          int bi = ps.seg_a[s] + it;
          double p[3] = {b.x[bi], b.y[bi], b.z[bi]};
          double e = tc_d2(p, c) - r2;
          if (e > best_e) { best_e = e; best_i = ps.seg_start[s] + it; }
        } else {
          int g = ps.seg_a[s] + it;
          double X = cl.X[g], Y = cl.Y[g], Z = cl.Z[g], R = cl.R[g];
          double q[3] = {X, Y, Z};
          double dc = sqrt(tc_d2(q, c)) + R * td[192];  // td[192] = largest |t_k| of the table
          if (dc * dc * (1.0 + 1e-12) - r2 < best_e) continue;
          int base = ps.seg_start[s] + (it << 6);
          for (int k = 0; k < 64; k++) {
            double p[3] = {X + R * td[3 * k], Y + R * td[3 * k + 1], Z + R * td[3 * k + 2]};
            double e = tc_d2(p, c) - r2;
            if (e > best_e) { best_e = e; best_i = base + k; }
          }
        }
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    double oe = __shfl_xor_sync(0xffffffffu, best_e, o);
    int oi = __shfl_xor_sync(0xffffffffu, best_i, o);
    if (oe > best_e || (oe == best_e && oi < best_i)) { best_e = oe; best_i = oi; }
  }
}

__device__ __forceinline__ void tc_point_td(const TcPointSet& ps, int idx, const TcBodies& b, const TcCells& c,
                                            const double* td, double* p) {
  if (ps.leaf) {
    int i = ps.seg_a[0] + idx;
    p[0] = b.x[i]; p[1] = b.y[i]; p[2] = b.z[i];
    return;
  }
  int s = 0;
  while (idx >= ps.seg_start[s + 1]) s++;
  int loc = idx - ps.seg_start[s];
  if (ps.seg_kind[s] == 0) {
    int i = ps.seg_a[s] + loc;
    p[0] = b.x[i]; p[1] = b.y[i]; p[2] = b.z[i];
  } else {
    int g = ps.seg_a[s] + (loc >> 6), k = loc & 63;
    double R = c.R[g];
    p[0] = c.X[g] + R * td[3 * k];
    p[1] = c.Y[g] + R * td[3 * k + 1];
    p[2] = c.Z[g] + R * td[3 * k + 2];
  }
}

// every lane of the warp ends with the same (c, r2)
__device__ void tc_warp_miniball(const TcPointSet& ps, const TcBodies& b, const TcCells& cl, const double* td,
                                 double* c, double* r2, unsigned int* err) {
  int lane = threadIdx.x & 31;
  double s[4][3];
  int ns = 1;
  tc_point_td(ps, 0, b, cl, td, s[0]);
  c[0] = s[0][0]; c[1] = s[0][1]; c[2] = s[0][2];
  *r2 = 0;
  for (int it = 0; it < 512; it++) {
    double best_e;
    int best_i;
    tc_mb_farthest(ps, b, cl, td, c, *r2, best_e, best_i);
    if (best_i == 0x7fffffff || best_e <= *r2 * 1e-15) return;
    double q[3];
    tc_point_td(ps, best_i, b, cl, td, q);
    double old = *r2;
    if (!tc_mb_small(s, ns, q, c, r2)) break;
    if (!(*r2 > old)) return;  // no growth: the ball is final (the reference's stop rule)
  }
  // not converged: grow the ball to enclose every point and flag it
  double mx = 0;
  for (int i = lane; i < ps.total; i += 32) {
    double p[3];
    tc_point_td(ps, i, b, cl, td, p);
    mx = fmax(mx, tc_d2(p, c));
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  *r2 = fmax(*r2, mx);
  if (lane == 0) tc_set_err(err, TC_EBIT_MINIBALL);
}

// ---------------------------------------------------------------------------------------
// P2M of every leaf (kernel_fast_lean.h:745-781; with jerks the Mdot of
// taichi_with_jerks/kernel_fast_lean.h:769-817): M[n][m] = sum_b q_b G[n][m](x_b - X) and
// Mdot[n][m] = sum_b q_b Gdot[n][m](x_b - X, v_b).
//
// One warp per leaf, LW lanes per body (lane a = order m), 32 / LW bodies per pass.  The
// column recurrence in n uses tabulated coefficients (no divisions):
//   G[n][c] = (A[n][c] dz) G[n-1][c] - (B[n][c] r^2) G[n-2][c],
//   A = (2n-1) / (n^2 - c^2), B = 1 / (n^2 - c^2) for n > c, A = B = 0 for n <= c,
// so a column is zero below its diagonal, and G[c][c] is picked from the running diagonal
// d_n = d_{n-1} (x + i y) / (2n), shared by every column of the body.  At n = c + 1 the
// recurrence is exactly dz G[c][c] (A = 1, G[c-1][c] = 0).
// ---------------------------------------------------------------------------------------
template <int P>
struct TcColTab {
  double A[P + 1][P + 2], B[P + 1][P + 2];
  double H[P + 3];  // 1 / (2j): the diagonal step G[j][j] = G[j-1][j-1] (x + i y) / (2j)
  __device__ void fill() {
    for (int i = threadIdx.x; i < (P + 1) * (P + 2); i += blockDim.x) {
      int n = i / (P + 2), c = i % (P + 2);
      double m2 = (double)(n * n - c * c);
      A[n][c] = n > c ? (2 * n - 1.) / m2 : 0.0;
      B[n][c] = n > c ? 1.0 / m2 : 0.0;
    }
    for (int j = threadIdx.x; j < P + 3; j += blockDim.x) H[j] = j > 0 ? 0.5 / j : 0.0;
  }
};

// G[n][c] from G[n-1][c] (g1), G[n-2][c] (g2); on the diagonal it is d; shifts g1, g2
__device__ __forceinline__ cd tc_col_next(bool on_diag, cd d, cd& g1, cd& g2, double ta, double tb, double dz,
                                          double r2) {
  double u = ta * dz, v = tb * r2;
  cd g = mk(u * g1.x - v * g2.x, u * g1.y - v * g2.y);
  if (on_diag) g = d;
  g2 = g1;
  g1 = g;
  return g;
}

constexpr int kP2MWarps = 4;
#ifndef TC_P2M_JERK_BLOCKS
#define TC_P2M_JERK_BLOCKS 2  // resident blocks per SM asked of the compiler (2: no spills)
#endif

template <int P, bool JERK>
__global__ void __launch_bounds__(kP2MWarps * 32, JERK ? TC_P2M_JERK_BLOCKS : 4) k_p2m_leaves(int ncell, const TcBodies b, TcCells c,
                                                                                      const TcLevels* lvd = nullptr) {
  constexpr int NT = (P + 1) * (P + 1);
  constexpr int LW = (P + 1 <= 16) ? 16 : 32;  // lanes per body
  constexpr int NH = 32 / LW;                  // bodies per pass
  __shared__ TcColTab<P> tab;
  __shared__ double sbod[kP2MWarps][32][9];    // dx dy dz q vx vy vz (row padded to 9)
  tab.fill();
  __syncthreads();
  if (lvd) ncell = lvd->ncell;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int a = lane % LW, h = lane / LW;
  // columns a-1, a, a+1 (column -1 is -conj(column 1), so a = 0 runs column 1 twice)
  const int ca = a > 0 ? a - 1 : 1, cb = a <= P ? a : P, cc = a <= P ? a + 1 : P + 1;
  double(*S)[9] = sbod[w];
  for (int ci = blockIdx.x * kP2MWarps + w; ci < ncell; ci += gridDim.x * kP2MWarps) {
    if (c.nchild[ci] != 0) continue;
    const int beg = c.begin[ci], nb = c.nbody[ci];
    const double X = c.X[ci], Y = c.Y[ci], Z = c.Z[ci];
    cd acc[P + 1], accd[P + 1];
#pragma unroll
    for (int n = 0; n <= P; n++) { acc[n] = mk(0, 0); accd[n] = mk(0, 0); }
    for (int j0 = 0; j0 < nb; j0 += 32) {
      const int cnt = min(32, nb - j0);
      __syncwarp();
      if (lane < cnt) {
        const int i = beg + j0 + lane;
        S[lane][0] = b.x[i] - X;
        S[lane][1] = b.y[i] - Y;
        S[lane][2] = b.z[i] - Z;
        S[lane][3] = (b.flags[i] & 2) ? b.m[i] : 0.0;
        if (JERK) { S[lane][4] = b.vx[i]; S[lane][5] = b.vy[i]; S[lane][6] = b.vz[i]; }
      }
      __syncwarp();
      for (int jj = h; a <= P && jj < cnt; jj += NH) {
        const double dx = S[jj][0], dy = S[jj][1], dz = S[jj][2], q = S[jj][3];
        const double r2 = dx * dx + dy * dy + dz * dz;
        cd etad, zd, ksid;
        if (JERK) {
          const double vx = S[jj][4], vy = S[jj][5], vz = S[jj][6];
          etad = mk(-vx * 0.5, vy * 0.5);
          zd = mk(vz, 0);
          ksid = mk(vx * 0.5, vy * 0.5);
        }
        // column indices laundered per body: keeps the coefficient loads inside the body loop
        // (hoisted, the 6 (P + 1) table values would not fit in registers)
        int ka = ca, kb = cb, kc = cc;
        asm volatile("" : "+r"(ka), "+r"(kb), "+r"(kc));
        cd d = mk(1, 0);
        cd A1 = mk(0, 0), A2 = mk(0, 0), B1 = mk(0, 0), B2 = mk(0, 0), C1 = mk(0, 0), C2 = mk(0, 0);
#pragma unroll
        for (int n = 0; n <= P; n++) {
          if (JERK && n >= 1) {
            // Gdot[n][a] from G[n-1][a-1], G[n-1][a], G[n-1][a+1]
            const cd pa = a > 0 ? A1 : mk(-C1.x, C1.y);
            cd gd = mk(0, 0);
            if (a <= n - 2) gd += C1 * etad;
            if (a <= n - 1) gd += B1 * zd;
            if (n - 1 >= 1 || a >= 1) gd += pa * ksid;
            accd[n] += q * gd;
          }
          if (n >= 1) d = d * mk(dx * (0.5 / n), dy * (0.5 / n));
          if (JERK) {
            tc_col_next(n == kc, d, C1, C2, tab.A[n][kc], tab.B[n][kc], dz, r2);
            tc_col_next(n == ka, d, A1, A2, tab.A[n][ka], tab.B[n][ka], dz, r2);
          }
          const cd gb = tc_col_next(n == kb, d, B1, B2, tab.A[n][kb], tab.B[n][kb], dz, r2);
          acc[n] += q * gb;
        }
      }
    }
    if (NH == 2) {
#pragma unroll
      for (int n = 0; n <= P; n++) {
        acc[n].x += __shfl_down_sync(0xffffffffu, acc[n].x, 16);
        acc[n].y += __shfl_down_sync(0xffffffffu, acc[n].y, 16);
        if (JERK) {
          accd[n].x += __shfl_down_sync(0xffffffffu, accd[n].x, 16);
          accd[n].y += __shfl_down_sync(0xffffffffu, accd[n].y, 16);
        }
      }
    }
    if (h == 0 && a <= P) {
      double* M = c.M + (size_t)ci * NT;
      double* Md = JERK ? c.Md + (size_t)ci * NT : nullptr;
#pragma unroll
      for (int n = 0; n <= P; n++) {
        if (n < a) continue;
        const int is = n * n + n;
        M[is + a] = acc[n].x;
        if (a > 0) M[is - a] = acc[n].y;
        if (JERK) {
          Md[is + a] = accd[n].x;
          if (a > 0) Md[is - a] = accd[n].y;
        }
      }
    }
  }
}

// G(dX) into shared memory, complex full storage (negative m by symmetry)
template <int P>
__device__ __forceinline__ void tc_warp_gnm_smem(double dx, double dy, double dz, cd* G) {
  int lane = threadIdx.x & 31;
  double r2 = dx * dx + dy * dy + dz * dz;
  for (int m = lane; m <= P; m += 32) {
    cd d0 = mk(1, 0);
    for (int j = 1; j <= m; j++) d0 = d0 * mk(dx / (2 * j), dy / (2 * j));
    TcCol col;
    col.init(m, d0);
    double s = (m & 1) ? -1.0 : 1.0;
    for (int n = 0; n <= P; n++) {
      cd g = col.step(n, dz, r2);
      if (n < m) continue;
      G[n * n + n + m] = g;
      if (m > 0) G[n * n + n - m] = mk(s * g.x, -s * g.y);
    }
  }
  __syncwarp();
}

// M2M into cell ci from its children (O(p^4) complex translation, kernel_fast_lean.h:921-931).
// Each child's multipole (and Mdot) is staged in shared memory as complex full storage
// (negative orders by symmetry), so every term is two shared loads and a complex FMA.
template <int P, bool JERK>
__device__ void tc_m2m_warp(int ci, const TcCells& c, cd* G, cd* SM, cd* SMd) {
  constexpr int NT = (P + 1) * (P + 1);
  constexpr int NOUT = (P + 1) * (P + 2) / 2;
  constexpr int PER = (NOUT + 31) / 32;
  int lane = threadIdx.x & 31;
  cd acc[PER], accd[PER];
#pragma unroll
  for (int k = 0; k < PER; k++) { acc[k] = mk(0, 0); accd[k] = mk(0, 0); }
  int ch0 = c.child[ci], nch = c.nchild[ci];
  for (int ch = ch0; ch < ch0 + nch; ch++) {
    const double* Mc = c.M + (size_t)ch * NT;
    const double* Mdc = JERK ? c.Md + (size_t)ch * NT : nullptr;
    for (int i = lane; i < NT; i += 32) {
      int n = 0;
      while ((n + 1) * (n + 1) <= i) n++;
      SM[i] = tc_r2c(Mc, n, i - n * n - n);
      if (JERK) SMd[i] = tc_r2c(Mdc, n, i - n * n - n);
    }
    tc_warp_gnm_smem<P>(c.X[ch] - c.X[ci], c.Y[ch] - c.Y[ci], c.Z[ch] - c.Z[ci], G);  // ends with __syncwarp
#pragma unroll
    for (int k = 0; k < PER; k++) {
      int o = lane + 32 * k;
      if (o >= NOUT) break;
      int n = 0;
      while ((n + 1) * (n + 2) / 2 <= o) n++;
      int m = o - n * (n + 1) / 2;
      cd s = mk(0, 0), sd = mk(0, 0);
      for (int kk = 0; kk <= n; kk++) {
        const int lo = max(-kk, m - n + kk), hi = min(kk, m + n - kk);
        const int nn = n - kk, base = nn * nn + nn + m;  // source (n - kk, m - l)
        for (int l = lo; l <= hi; l++) {
          cd g = G[kk * kk + kk + l];
          s += SM[base - l] * g;
          if (JERK) sd += SMd[base - l] * g;
        }
      }
      acc[k] += s;
      if (JERK) accd[k] += sd;
    }
    __syncwarp();
  }
  double* M = c.M + (size_t)ci * NT;
  double* Md = JERK ? c.Md + (size_t)ci * NT : nullptr;
#pragma unroll
  for (int k = 0; k < PER; k++) {
    int o = lane + 32 * k;
    if (o >= NOUT) break;
    int n = 0;
    while ((n + 1) * (n + 2) / 2 <= o) n++;
    int m = o - n * (n + 1) / 2;
    int is = n * n + n;
    M[is + m] = acc[k].x;
    if (m > 0) M[is - m] = acc[k].y;
    if (JERK) {
      Md[is + m] = accd[k].x;
      if (m > 0) Md[is - m] = accd[k].y;
    }
  }
}

// warps per block of the M2M and L2L level kernels (three NT-complex arrays per warp in
// static shared memory, at most 48 KB)
template <int P>
struct TcTransW {
  static constexpr int W = P >= 14 ? 2 : 4;
};

constexpr int kUpWarps = 4;

// t-design table in shared memory; s_td[192] = the largest |t_k| (rows 36-47 of the
// reference's table are not unit vectors, |t| = 1.1968, so the pruning bound uses the norm)
__device__ __forceinline__ void tc_load_tdesign(double* s_td) {
  for (int i = threadIdx.x; i < 192; i += blockDim.x) s_td[i] = c_tdesign[i];
  if (threadIdx.x == 0) {
    double mx = 0;
    for (int k = 0; k < 64; k++)
      mx = fmax(mx, sqrt(c_tdesign[3 * k] * c_tdesign[3 * k] + c_tdesign[3 * k + 1] * c_tdesign[3 * k + 1] +
                         c_tdesign[3 * k + 2] * c_tdesign[3 * k + 2]));
    s_td[192] = mx * (1.0 + 1e-12);
  }
  __syncthreads();
}

// one warp: expansion centre, radius and has_sink of cell ci
__device__ void tc_cell_ball(int ci, const TcBodies& b, TcCells& c, const double* s_td, unsigned int* err) {
  int lane = threadIdx.x & 31;
  TcPointSet ps;
  int nch = c.nchild[ci];
  bool sink = false;
  if (nch == 0) {
    ps.leaf = 1;
    ps.seg_a[0] = c.begin[ci];
    ps.total = c.nbody[ci];
    for (int i = c.begin[ci] + lane; i < c.begin[ci] + c.nbody[ci]; i += 32) sink |= (b.flags[i] & 1) != 0;
  } else {
    ps.leaf = 0;
    ps.nseg = nch;
    int tot = 0;
    for (int s = 0; s < nch; s++) {
      int ch = c.child[ci] + s;
      ps.seg_start[s] = tot;
      sink |= c.has_sink[ch] != 0;
      if (c.nchild[ch] == 0) {
        ps.seg_kind[s] = 0;
        ps.seg_a[s] = c.begin[ch];
        tot += c.nbody[ch];
      } else {
        ps.seg_kind[s] = 1;
        ps.seg_a[s] = c.child[ch];
        tot += 64 * c.nchild[ch];
      }
    }
    ps.seg_start[nch] = tot;
    ps.total = tot;
  }
  sink = __any_sync(0xffffffffu, sink);
  double cc[3], r2;
  tc_warp_miniball(ps, b, c, s_td, cc, &r2, err);
  if (lane == 0) {
    c.X[ci] = cc[0]; c.Y[ci] = cc[1]; c.Z[ci] = cc[2];
    c.R[ci] = sqrt(r2) + 1e-6;
    c.has_sink[ci] = sink;
  }
  __syncwarp();
}

// balls of every leaf (they depend on the leaf's own bodies only)
__global__ void __launch_bounds__(kUpWarps * 32) k_leaf_balls(int ncell, const TcBodies b, TcCells c,
                                                              unsigned int* err, const TcLevels* lvd = nullptr) {
  __shared__ double s_td[193];
  tc_load_tdesign(s_td);
  if (lvd) ncell = lvd->ncell;  // device-sized launch (graph): the cell count of this tree
  int w = threadIdx.x >> 5;
  for (int ci = blockIdx.x * kUpWarps + w; ci < ncell; ci += gridDim.x * kUpWarps)
    if (c.nchild[ci] == 0) tc_cell_ball(ci, b, c, s_td, err);
}

// inner cells of level l: ball over the children's points, then M2M from the children
template <int P, bool JERK>
__global__ void __launch_bounds__(TcTransW<P>::W * 32) k_upward_level(int l, const TcBodies b, TcCells c,
                                                                      const int* __restrict__ lv_start,
                                                                      const int* __restrict__ lv_count,
                                                                      unsigned int* err) {
  constexpr int W = TcTransW<P>::W, NT = (P + 1) * (P + 1);
  __shared__ cd sG[W][NT];
  __shared__ cd sM[W][NT];
  __shared__ cd sMd[W][JERK ? NT : 1];
  __shared__ double s_td[193];
  tc_load_tdesign(s_td);
  int w = threadIdx.x >> 5;
  int cnt = lv_count[l], st = lv_start[l];
  for (int k = blockIdx.x * W + w; k < cnt; k += gridDim.x * W) {
    int ci = st + k;
    if (c.nchild[ci] == 0) continue;
    tc_cell_ball(ci, b, c, s_td, err);
    tc_m2m_warp<P, JERK>(ci, c, sG[w], sM[w], sMd[w]);
    __syncwarp();
  }
}

}  // namespace tc
