/* CPU oracle for the FMM gravity evaluation -- TEST INFRASTRUCTURE ONLY (see tc_oracle.h).
 *
 * Plain C99, FP64, single thread.  Each function names the reference code it restates;
 * paths are relative to the reference project (QirongZhu/taichi_collisional).
 */
#include "tc_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../taichi_collisional_b200/csrc/swap_tables.h"
#include "../taichi_collisional_b200/csrc/tdesign.h"

typedef double complex cplx;

#define PMAX_O TC_SWAP_PMAX
#define NT(p) (((p) + 1) * ((p) + 1))

/* ------------------------------------------------------------------------------------ */
/* Tables: initKernel, kernel_fast_lean.h:122-160.                                       */
/* factorial_table is filled for i < 2P only, so factorial_table[2P] == 0 (quirk: the   */
/* (P,+-P) entries of the scaled M2L multipole vanish).                                  */
/* ------------------------------------------------------------------------------------ */
static int g_p = -1;
static double g_fact[2 * PMAX_O + 2];
static double g_fc[NT(PMAX_O)], g_fcinv[NT(PMAX_O)];

void tco_init(int p) {
  if (p == g_p) return;
  g_p = p;
  memset(g_fact, 0, sizeof(g_fact));
  g_fact[0] = 1.0;
  for (int i = 1; i < 2 * p; i++) g_fact[i] = (double)i * g_fact[i - 1];
  for (int n = 0; n <= p; n++)
    for (int m = -n; m <= n; m++) {
      int am = m < 0 ? -m : m;
      double f = g_fact[n + am] * g_fact[n - am];
      g_fc[n * n + n + m] = f;
      g_fcinv[n * n + n + m] = f != 0.0 ? 1.0 / f : 0.0; /* the inf entry is never read */
    }
}

/* make_Gnm, kernel_fast_lean.h:235-266: regular solid harmonics, full storage with
 * G[n,-m] = (-1)^m conj(G[n,m]). */
static void make_gnm(const double* dX, cplx* G, int p) {
  double r2 = dX[0] * dX[0] + dX[1] * dX[1] + dX[2] * dX[2];
  G[0] = 1.0;
  for (int n = 1; n <= p; n++) {
    int n2 = n * n, ind = n2 + n + n, is = n2 - n, inew = n2 + n;
    G[ind] = G[n2 - 1] * CMPLX(dX[0] / (2 * n), dX[1] / (2 * n));
    for (int m = 0; m < n - 1; m++) {
      int m2 = n2 - m * m;
      G[inew + m] = (2 * n - 1.) / m2 * dX[2] * G[is + m] - r2 / m2 * G[n2 - 3 * n + 2 + m];
    }
    G[inew + n - 1] = dX[2] * G[is + n - 1];
    double s = -1;
    for (int m = 1; m <= n; m++) {
      G[inew - m] = conj(G[inew + m] * s);
      s = -s;
    }
  }
}

void tco_make_gnm(const double* dX, double* re, double* im, int p) {
  cplx G[NT(PMAX_O)];
  make_gnm(dX, G, p);
  for (int i = 0; i < NT(p); i++) { re[i] = creal(G[i]); im[i] = cimag(G[i]); }
}

/* make_Gnmdot, taichi_with_jerks/kernel_fast_lean.h:272-304: time derivative of G for a
 * displacement moving with velocity dV.  Terms that would read G at n<0 or at (0,-1) are
 * zero (the reference reads one element before its array there). */
static cplx gget(const cplx* G, int n, int m) {
  if (n < 0) return 0.0;
  int am = m < 0 ? -m : m;
  if (am > n) return 0.0;
  return G[n * n + n + m];
}
static void make_gnmdot(const double* dV, const cplx* G, cplx* Gd, int p) {
  cplx etad = CMPLX(-dV[0] * 0.5, dV[1] * 0.5), zd = dV[2], ksid = CMPLX(dV[0] * 0.5, dV[1] * 0.5);
  for (int n = 0; n <= p; n++) {
    int is = n * n + n;
    for (int m = 0; m <= n; m++) {
      cplx acc = 0.0;
      if (m <= n - 2) acc += gget(G, n - 1, m + 1) * etad;
      if (m <= n - 1) acc += gget(G, n - 1, m) * zd;
      acc += gget(G, n - 1, m - 1) * ksid;
      Gd[is + m] = acc;
    }
    double s = -1;
    for (int m = 1; m <= n; m++) {
      Gd[is - m] = conj(Gd[is + m] * s);
      s = -s;
    }
  }
}

/* real_2_complex / complex_2_real, kernel_fast_lean.h:162-191. */
static void r2c(const double* r, cplx* c, int p) {
  for (int n = 0; n <= p; n++) {
    int is = n * n + n;
    c[is] = r[is];
    double s = -1;
    for (int m = 1; m <= n; m++) {
      c[is - m] = CMPLX(r[is + m] * s, -r[is - m] * s);
      c[is + m] = CMPLX(r[is + m], r[is - m]);
      s = -s;
    }
  }
}
static void c2r_add(const cplx* c, double* r, int p) {
  for (int n = 0; n <= p; n++) {
    int is = n * n + n;
    r[is] += creal(c[is]);
    for (int m = 1; m <= n; m++) {
      r[is - m] += cimag(c[is + m]);
      r[is + m] += creal(c[is + m]);
    }
  }
}

/* swap_x_z, kernel_rotate.h:6-53 (tables derived in gen_swap_tables.py). */
void tco_swap_xz(double* v, int p) {
  double o[NT(PMAX_O)];
  for (int i = 0; i < NT(p); i++) {
    double s = 0;
    for (int k = tc_swap_rowptr[i]; k < tc_swap_rowptr[i + 1]; k++) s += tc_swap_val[k] * v[tc_swap_col[k]];
    o[i] = s;
  }
  memcpy(v, o, sizeof(double) * NT(p));
}

/* ------------------------------------------------------------------------------------ */
/* Single-cell kernels.                                                                   */
/* ------------------------------------------------------------------------------------ */

/* P2M, kernel_fast_lean.h:745-781 (+ Mdot, taichi_with_jerks/kernel_fast_lean.h:769-817). */
void tco_p2m(int p, int nb, const double* x, const double* y, const double* z, const double* vx,
             const double* vy, const double* vz, const double* m, const double* C, double* M,
             double* Md) {
  cplx cm[NT(PMAX_O)], cmd[NT(PMAX_O)], G[NT(PMAX_O)], Gd[NT(PMAX_O)];
  for (int i = 0; i < NT(p); i++) cm[i] = cmd[i] = 0;
  for (int b = 0; b < nb; b++) {
    double dX[3] = {x[b] - C[0], y[b] - C[1], z[b] - C[2]};
    make_gnm(dX, G, p);
    for (int i = 0; i < NT(p); i++) cm[i] += m[b] * G[i];
    if (Md) {
      double dV[3] = {vx[b], vy[b], vz[b]};
      make_gnmdot(dV, G, Gd, p);
      for (int i = 0; i < NT(p); i++) cmd[i] += m[b] * Gd[i];
    }
  }
  c2r_add(cm, M, p);
  if (Md) c2r_add(cmd, Md, p);
}

/* M2M translation, kernel_fast_lean.h:900-938 (Mdot: taichi_with_jerks :950-998).
 * dX = child centre - parent centre. */
void tco_m2m(int p, const double* Mc, const double* Mdc, const double* dX, double* Mp,
             double* Mdp) {
  cplx c[NT(PMAX_O)], cd[NT(PMAX_O)], G[NT(PMAX_O)], o[NT(PMAX_O)], od[NT(PMAX_O)];
  r2c(Mc, c, p);
  if (Mdc) r2c(Mdc, cd, p);
  make_gnm(dX, G, p);
  for (int i = 0; i < NT(p); i++) o[i] = od[i] = 0;
  for (int n = 0; n <= p; n++)
    for (int m = 0; m <= n; m++) {
      int idx = n * n + n + m;
      for (int k = 0; k <= n; k++) {
        int lo = -k > m - n + k ? -k : m - n + k, hi = k < m + n - k ? k : m + n - k;
        for (int l = lo; l <= hi; l++) {
          int a = (n - k) * (n - k) + (n - k) + (m - l), g = k * k + k + l;
          o[idx] += c[a] * G[g];
          if (Mdc) od[idx] += cd[a] * G[g];
        }
      }
    }
  c2r_add(o, Mp, p);
  if (Mdc) c2r_add(od, Mdp, p);
}

/* L2L, kernel_fast_lean.h:941-987 (Ldot: taichi_with_jerks :1001-1058).
 * dX = parent centre - child centre. */
void tco_l2l(int p, const double* Lp, const double* Ldp, const double* dX, double* Lc,
             double* Ldc) {
  cplx c[NT(PMAX_O)], cd[NT(PMAX_O)], G[NT(PMAX_O)], o[NT(PMAX_O)], od[NT(PMAX_O)];
  r2c(Lp, c, p);
  if (Ldp) r2c(Ldp, cd, p);
  make_gnm(dX, G, p);
  for (int i = 0; i < NT(p); i++) { G[i] = conj(G[i]); o[i] = od[i] = 0; }
  for (int n = 0; n <= p; n++)
    for (int m = 0; m <= n; m++) {
      int idx = n * n + n + m;
      for (int k = 0; k <= p - n; k++)
        for (int l = -k; l <= k; l++) {
          int a = (n + k) * (n + k) + (n + k) + (m + l), g = k * k + k + l;
          o[idx] += c[a] * G[g];
          if (Ldp) od[idx] += cd[a] * G[g];
        }
    }
  c2r_add(o, Lc, p);
  if (Ldp) c2r_add(od, Ldc, p);
}

/* L2P, kernel_fast_lean.h:989-1032 (jerk: taichi_with_jerks :1060-1128).
 * dX = cell centre - body position, v = body velocity (NULL: no jerk). */
void tco_l2p(int p, const double* L, const double* Ld, const double* dX, const double* v,
             double* out) {
  cplx c[NT(PMAX_O)], cd[NT(PMAX_O)], G[NT(PMAX_O)], Gd[NT(PMAX_O)];
  cplx Phi[4] = {0, 0, 0, 0}, Phid[4] = {0, 0, 0, 0};
  r2c(L, c, p);
  if (Ld) r2c(Ld, cd, p);
  make_gnm(dX, G, p);
  if (Ld) {
    double dV[3] = {-v[0], -v[1], -v[2]};
    make_gnmdot(dV, G, Gd, p);
  }
  for (int i = 0; i < NT(p); i++) { G[i] = conj(G[i]); if (Ld) Gd[i] = conj(Gd[i]); }
  for (int n = 0; n <= 1; n++)
    for (int m = 0; m <= n; m++) {
      int idx = n * n + n + m;
      for (int k = 0; k <= p - n; k++)
        for (int l = -k; l <= k; l++) {
          int a = (n + k) * (n + k) + (n + k) + (m + l), g = k * k + k + l;
          Phi[idx] += c[a] * G[g];
          if (Ld) {
            Phid[idx] += c[a] * Gd[g];
            Phid[idx] += cd[a] * G[g];
          }
        }
    }
  out[0] += creal(Phi[0]);
  out[1] -= creal(Phi[3]);
  out[2] -= cimag(Phi[3]);
  out[3] -= creal(Phi[2]);
  if (Ld) {
    out[4] -= creal(Phid[3]);
    out[5] -= cimag(Phid[3]);
    out[6] -= creal(Phid[2]);
  }
}

/* z-axis phase rotation of a real-stored vector by e^{i m a} (conj when inv). */
static void rotz(double* v, const double* er, const double* ei, int p, int inv) {
  for (int n = 1; n <= p; n++) {
    int is = n * n + n;
    for (int m = 1; m <= n; m++) {
      double im = v[is - m], re = v[is + m], a = er[m], b = ei[m];
      if (!inv) {
        v[is - m] = a * im + b * re;
        v[is + m] = a * re - b * im;
      } else {
        v[is - m] = a * im - b * re;
        v[is + m] = a * re + b * im;
      }
    }
  }
}

/* M2L_rotate, one-sided (taichi_with_jerks/kernel_fast_lean.h:1130-1371; the top-level
 * mutual form kernel_fast_lean.h:1034-1295 is two one-sided calls).  dX = Xt - Xs.
 * L and Ld are accumulated. */
void tco_m2l_rotate(int p, const double* M, const double* Md, const double* dX, double* L,
                    double* Ld) {
  tco_init(p);
  int nt = NT(p);
  double rxy2 = dX[0] * dX[0] + dX[1] * dX[1], rxy = sqrt(rxy2);
  double r2 = rxy2 + dX[2] * dX[2], r = sqrt(r2), rinv = 1.0 / r;
  double zr[PMAX_O + 1], zi[PMAX_O + 1], xr[PMAX_O + 1], xi[PMAX_O + 1];
  zr[0] = 1; zi[0] = 0; xr[0] = 1; xi[0] = 0;
  zr[1] = 1; zi[1] = 0;
  xr[1] = dX[2] * rinv; xi[1] = -rxy * rinv;
  if (rxy > 0) {
    double q = 1.0 / rxy;
    zr[1] = dX[1] * q;
    zi[1] = dX[0] * q;
  }
  for (int m = 1; m < p; m++) {
    zr[m + 1] = zr[m] * zr[1] - zi[m] * zi[1];
    zi[m + 1] = zr[m] * zi[1] + zi[m] * zr[1];
    xr[m + 1] = xr[m] * xr[1] - xi[m] * xi[1];
    xi[m + 1] = xr[m] * xi[1] + xi[m] * xr[1];
  }
  for (int arr = 0; arr < 2; arr++) {
    const double* src = arr ? Md : M;
    double* dst = arr ? Ld : L;
    if (!src) continue;
    double a[NT(PMAX_O)], l[NT(PMAX_O)];
    for (int i = 0; i < nt; i++) { a[i] = src[i] * g_fc[i]; l[i] = 0; }
    rotz(a, zr, zi, p, 0);
    tco_swap_xz(a, p);
    rotz(a, xr, xi, p, 0);
    tco_swap_xz(a, p);
    for (int i = 0; i < nt; i++) a[i] *= g_fcinv[i];
    /* translation along z, kernel_fast_lean.h:1161-1200 */
    double pn = rinv;
    for (int n = 0; n <= p; n++) {
      int is = n * (n + 1);
      double pr = pn;
      for (int k = 0; k <= p - n; k++) {
        l[is] += a[k * (k + 1)] * (g_fact[n + k] * pr);
        pr *= rinv;
      }
      double pm = rinv, s = -1;
      int mmax = n < p - n ? n : p - n;
      for (int m = 1; m <= mmax; m++) {
        pr = pn * pm;
        for (int k = m; k <= p - n; k++) {
          int ik = k * (k + 1);
          double f = g_fact[n + k] * pr * s;
          l[is - m] += a[ik - m] * f;
          l[is + m] += a[ik + m] * f;
          pr *= rinv;
        }
        s = -s;
        pm *= rinv;
      }
      pn *= rinv;
    }
    tco_swap_xz(l, p);
    rotz(l, xr, xi, p, 1);
    tco_swap_xz(l, p);
    rotz(l, zr, zi, p, 1);
    for (int i = 0; i < nt; i++) dst[i] += l[i];
  }
}

/* make_Tnm + textbook O(p^4) M2L, kernel_fast_lean.h:193-233, :1297-1350 (independent
 * check of the rotation form).  dX = Xt - Xs. */
void tco_m2l_direct(int p, const double* M, const double* dX, double* L) {
  int nt = NT(p);
  cplx T[NT(PMAX_O)], cM[NT(PMAX_O)], o[NT(PMAX_O)];
  double r2 = dX[0] * dX[0] + dX[1] * dX[1] + dX[2] * dX[2], invr2 = 1 / r2;
  T[0] = sqrt(invr2);
  for (int n = 1; n <= p; n++) {
    int n2 = n * n, ind = n2 + n + n;
    T[ind] = T[n2 - 1] * CMPLX(dX[0] * (2 * n - 1) * invr2, dX[1] * (2 * n - 1) * invr2);
    int is = n2 - n, inew = n2 + n;
    if (n > 1)
      for (int m = 0; m < n - 1; m++)
        T[inew + m] = invr2 * (2 * n - 1.) * dX[2] * T[is + m] -
                      invr2 * ((n - 1) * (n - 1) - m * m) * T[n2 - 3 * n + 2 + m];
    T[inew + n - 1] = invr2 * (2 * n - 1.) * dX[2] * T[is + n - 1];
    double s = -1;
    for (int m = 1; m <= n; m++) {
      T[n2 + n - m] = conj(T[n2 + n + m] * s);
      s = -s;
    }
  }
  double Mm[NT(PMAX_O)];
  memcpy(Mm, M, sizeof(double) * nt);
  for (int n = 1; n <= p; n++)
    for (int m = 1; m <= n; m++) Mm[n * n + n - m] *= -1;
  r2c(Mm, cM, p);
  for (int i = 0; i < nt; i++) o[i] = 0;
  for (int n = 0; n <= p; n++)
    for (int m = -n; m <= n; m++)
      for (int k = 0; k <= p - n; k++)
        for (int l = -k; l <= k; l++)
          o[n * n + n + m] += cM[k * k + k + l] * T[(n + k) * (n + k) + (n + k) + (m + l)];
  c2r_add(o, L, p);
}

/* ------------------------------------------------------------------------------------ */
/* Smallest enclosing ball (the reference calls Gaertner's Miniball, miniball.hpp, from  */
/* P2M kernel_fast_lean.h:707-737 and M2M :833-892).  Own implementation of the pivoting */
/* scheme: repeatedly take the farthest point (first in input order on ties) and solve  */
/* the small problem "smallest ball through q enclosing the support set" exactly.        */
/* ------------------------------------------------------------------------------------ */
static int circumsphere(int k, const double (*q)[3], double* c, double* r2) {
  /* ball through q[0..k-1] with centre in their affine hull */
  if (k == 1) { memcpy(c, q[0], 3 * sizeof(double)); *r2 = 0; return 1; }
  double v[3][3], A[3][3], b[3], lam[3];
  int d = k - 1;
  for (int i = 0; i < d; i++)
    for (int j = 0; j < 3; j++) v[i][j] = q[i + 1][j] - q[0][j];
  for (int i = 0; i < d; i++) {
    for (int j = 0; j < d; j++) A[i][j] = 2 * (v[i][0] * v[j][0] + v[i][1] * v[j][1] + v[i][2] * v[j][2]);
    b[i] = v[i][0] * v[i][0] + v[i][1] * v[i][1] + v[i][2] * v[i][2];
  }
  /* Gaussian elimination with partial pivoting */
  double scale = 0;
  for (int i = 0; i < d; i++) scale = fmax(scale, fabs(A[i][i]));
  for (int col = 0; col < d; col++) {
    int piv = col;
    for (int r = col + 1; r < d; r++) if (fabs(A[r][col]) > fabs(A[piv][col])) piv = r;
    if (fabs(A[piv][col]) <= 1e-13 * scale) return 0;
    if (piv != col) {
      for (int j = 0; j < d; j++) { double t = A[col][j]; A[col][j] = A[piv][j]; A[piv][j] = t; }
      double t = b[col]; b[col] = b[piv]; b[piv] = t;
    }
    for (int r = col + 1; r < d; r++) {
      double f = A[r][col] / A[col][col];
      for (int j = col; j < d; j++) A[r][j] -= f * A[col][j];
      b[r] -= f * b[col];
    }
  }
  for (int i = d - 1; i >= 0; i--) {
    double s = b[i];
    for (int j = i + 1; j < d; j++) s -= A[i][j] * lam[j];
    lam[i] = s / A[i][i];
  }
  double off[3] = {0, 0, 0};
  for (int i = 0; i < d; i++)
    for (int j = 0; j < 3; j++) off[j] += lam[i] * v[i][j];
  for (int j = 0; j < 3; j++) c[j] = q[0][j] + off[j];
  *r2 = off[0] * off[0] + off[1] * off[1] + off[2] * off[2];
  return 1;
}

static double d2(const double* a, const double* b) {
  double x = a[0] - b[0], y = a[1] - b[1], z = a[2] - b[2];
  return x * x + y * y + z * z;
}

/* smallest ball with q on the boundary enclosing support s[0..ns-1]; updates s */
static int mb_small(double (*s)[3], int* ns, const double* q, double* c, double* r2) {
  int n = *ns, best_mask = -1;
  double bc[3] = {0, 0, 0}, br2 = INFINITY;
  for (int mask = 0; mask < (1 << n); mask++) {
    if (__builtin_popcount((unsigned)mask) > 3) continue;
    double pts[4][3];
    int k = 0;
    memcpy(pts[k++], q, 3 * sizeof(double));
    for (int i = 0; i < n; i++)
      if (mask & (1 << i)) memcpy(pts[k++], s[i], 3 * sizeof(double));
    double cc[3], rr;
    if (!circumsphere(k, (const double(*)[3])pts, cc, &rr)) continue;
    if (rr >= br2) continue;
    int ok = 1;
    for (int i = 0; i < n && ok; i++)
      if (!(mask & (1 << i)) && d2(s[i], cc) > rr * (1 + 1e-13) + 1e-300) ok = 0;
    if (ok) { br2 = rr; memcpy(bc, cc, sizeof(bc)); best_mask = mask; }
  }
  if (best_mask < 0) return 0;
  double ns_[4][3];
  int k = 0;
  memcpy(ns_[k++], q, 3 * sizeof(double));
  for (int i = 0; i < n; i++)
    if (best_mask & (1 << i)) memcpy(ns_[k++], s[i], 3 * sizeof(double));
  memcpy(s, ns_, sizeof(double) * 3 * k);
  *ns = k;
  memcpy(c, bc, sizeof(bc));
  *r2 = br2;
  return 1;
}

int tco_miniball(int np, const double* pts, double* c, double* r2) {
  double s[4][3];
  int ns = 1;
  memcpy(s[0], pts, 3 * sizeof(double));
  memcpy(c, pts, 3 * sizeof(double));
  *r2 = 0;
  for (int it = 0; it < 1000; it++) {
    int piv = -1;
    double maxe = 0;
    for (int i = 0; i < np; i++) {
      double e = d2(pts + 3 * i, c) - *r2;
      if (e > maxe) { maxe = e; piv = i; }
    }
    if (piv < 0 || maxe <= *r2 * 1e-15) return 0;
    double old = *r2;
    if (!mb_small(s, &ns, pts + 3 * piv, c, r2)) return 2;
    if (!(*r2 > old)) return 0; /* no growth: final (pivot loop of miniball.hpp stops the same way) */
  }
  return 1;
}

/* ------------------------------------------------------------------------------------ */
/* Tree build: getBounds build_tree.h:239-260, Morton keys :443-454, Body::operator<     */
/* exafmm.h:31-40 (z most significant in each bit triple), buildCellsSorted :344-435.    */
/* ------------------------------------------------------------------------------------ */
typedef struct {
  int n, ncell, cap, p, variant;
  int* perm;
  double *x, *y, *z, *vx, *vy, *vz, *m;
  unsigned char *sink, *source;
  int *begin, *nbody, *nchild, *child, *level;
  double *gx, *R0c, *X, *R;
  unsigned char* has_sink;
  double *M, *Md, *L, *Ld;
  long long nm2l, np2p, m2l_cap, p2p_cap;
  int *m2l_t, *m2l_s, *p2p_t, *p2p_s;
  double theta;
  int ncrit, max_level;
} otree;

static otree T;

typedef struct { uint64_t hi; uint32_t lo; int idx; } okey;

static int okey_cmp(const void* a, const void* b) {
  const okey *u = (const okey*)a, *v = (const okey*)b;
  if (u->hi != v->hi) return u->hi < v->hi ? -1 : 1;
  if (u->lo != v->lo) return u->lo < v->lo ? -1 : 1;
  return u->idx < v->idx ? -1 : (u->idx > v->idx);
}

static void spread_key(uint32_t mx, uint32_t my, uint32_t mz, uint64_t* hi, uint32_t* lo) {
  /* 84-bit interleave, bit 3b+2 = z_b, 3b+1 = y_b, 3b = x_b; hi = bits 21..83, lo = 0..20 */
  uint64_t h = 0;
  uint32_t l = 0;
  for (int b = 27; b >= 0; b--) {
    for (int d = 2; d >= 0; d--) {
      uint32_t bit = ((d == 0 ? mx : d == 1 ? my : mz) >> b) & 1u;
      int pos = 3 * b + d;
      if (pos >= 21) h |= (uint64_t)bit << (pos - 21);
      else l |= bit << pos;
    }
  }
  *hi = h;
  *lo = l;
}

static int push_cell(void) {
  if (T.ncell == T.cap) {
    int nc = T.cap ? 2 * T.cap : 1024;
    T.begin = realloc(T.begin, nc * sizeof(int));
    T.nbody = realloc(T.nbody, nc * sizeof(int));
    T.nchild = realloc(T.nchild, nc * sizeof(int));
    T.child = realloc(T.child, nc * sizeof(int));
    T.level = realloc(T.level, nc * sizeof(int));
    T.gx = realloc(T.gx, 3 * nc * sizeof(double));
    T.R0c = realloc(T.R0c, nc * sizeof(double));
    T.cap = nc;
  }
  return T.ncell++;
}

static int octant_of(int i, const double* X) {
  return (T.x[i] >= X[0]) + ((T.y[i] >= X[1]) << 1) + ((T.z[i] >= X[2]) << 2);
}

static void build_cells(int c, int begin, int end, const double* X, double R, int level) {
  T.begin[c] = begin;
  T.nbody[c] = end - begin;
  T.nchild[c] = 0;
  T.child[c] = -1;
  T.level[c] = level;
  memcpy(T.gx + 3 * c, X, 3 * sizeof(double));
  T.R0c[c] = R / (1 << level);
  if (level > T.max_level) T.max_level = level;
  if (end - begin <= T.ncrit) return;
  int size[8] = {0}, off[8];
  if (end - begin <= 32) {
    for (int i = begin; i < end; i++) size[octant_of(i, X)]++;
    int o = begin;
    for (int i = 0; i < 8; i++) { off[i] = o; o += size[i]; }
  } else {
    off[0] = begin;
    for (int i = 1; i < 8; i++) {
      int left = begin, right = end;
      while (left < right - 1) {
        int mid = (left + right) / 2;
        if (octant_of(mid, X) >= i) right = mid; else left = mid;
      }
      off[i] = left + 1;
    }
    for (int i = 0; i < 7; i++) size[i] = off[i + 1] - off[i];
    size[7] = end - off[7];
  }
  int nch = 0;
  for (int i = 0; i < 8; i++) nch += size[i] != 0;
  T.nchild[c] = nch;
  int first = T.ncell;
  for (int i = 0; i < nch; i++) push_cell();
  T.child[c] = first;
  int k = 0;
  for (int i = 0; i < 8; i++) {
    double Xc[3] = {X[0], X[1], X[2]};
    double r = R / (1 << (level + 1));
    for (int d = 0; d < 3; d++) Xc[d] += r * (((i & 1 << d) >> d) * 2 - 1);
    if (size[i]) {
      build_cells(first + k, off[i], off[i] + size[i], Xc, R, level + 1);
      k++;
    }
  }
}

static void build_tree(const tco_params* prm) {
  int n = T.n;
  double mn[3], mx[3], X0[3], R0 = 0;
  for (int d = 0; d < 3; d++) {
    const double* a = d == 0 ? T.x : d == 1 ? T.y : T.z;
    mn[d] = mx[d] = a[0];
    for (int i = 0; i < n; i++) { mn[d] = fmin(a[i], mn[d]); mx[d] = fmax(a[i], mx[d]); }
    X0[d] = (mx[d] + mn[d]) / 2;
  }
  if (prm->use_shift) { /* taichi_with_jerks/build_tree.h:253-268, before R0 */
    double box = -1;
    for (int d = 0; d < 3; d++) if (mx[d] - mn[d] > box) box = mx[d] - mn[d];
    for (int d = 0; d < 3; d++) X0[d] += (prm->shift_u[d] - 0.5) * box / 25;
  }
  for (int d = 0; d < 3; d++) { R0 = fmax(X0[d] - mn[d], R0); R0 = fmax(mx[d] - X0[d], R0); }
  R0 *= 1.00001;
  okey* keys = malloc(sizeof(okey) * n);
  double maxint = (double)(1u << 28);
  for (int i = 0; i < n; i++) {
    double xf = (T.x[i] - (X0[0] - R0)) / (2.0 * R0);
    double yf = (T.y[i] - (X0[1] - R0)) / (2.0 * R0);
    double zf = (T.z[i] - (X0[2] - R0)) / (2.0 * R0);
    uint32_t ix = (uint32_t)(int64_t)floor(xf * maxint), iy = (uint32_t)(int64_t)floor(yf * maxint),
             iz = (uint32_t)(int64_t)floor(zf * maxint);
    spread_key(ix, iy, iz, &keys[i].hi, &keys[i].lo);
    keys[i].idx = i;
  }
  qsort(keys, n, sizeof(okey), okey_cmp);
  /* permute bodies into sorted order */
  double* tmp = malloc(sizeof(double) * n);
  double** arrs[7] = {&T.x, &T.y, &T.z, &T.vx, &T.vy, &T.vz, &T.m};
  for (int a = 0; a < 7; a++) {
    for (int i = 0; i < n; i++) tmp[i] = (*arrs[a])[keys[i].idx];
    memcpy(*arrs[a], tmp, sizeof(double) * n);
  }
  unsigned char* t8 = malloc(n);
  for (int i = 0; i < n; i++) t8[i] = T.sink[keys[i].idx];
  memcpy(T.sink, t8, n);
  for (int i = 0; i < n; i++) t8[i] = T.source[keys[i].idx];
  memcpy(T.source, t8, n);
  for (int i = 0; i < n; i++) T.perm[i] = keys[i].idx;
  free(t8);
  free(tmp);
  free(keys);
  T.ncell = 0;
  T.max_level = 0;
  push_cell();
  build_cells(0, 0, n, X0, R0, 0);
}

/* ------------------------------------------------------------------------------------ */
/* Upward pass, traverse_eager.h:9-34, with Miniball centres (kernel_fast_lean.h:707-737, */
/* :833-892; R = r_mb + 1e-6) and t-design points around grandchildren (:859-869).        */
/* ------------------------------------------------------------------------------------ */
static void upward(void) {
  int p = T.p, nt = NT(p), jerk = T.variant == TCO_VARIANT_JERKS;
  double* pts = NULL;
  int ptcap = 0;
  for (int c = T.ncell - 1; c >= 0; c--) {
    int np = 0;
    T.has_sink[c] = 0;
    if (T.nchild[c] == 0) {
      if (T.nbody[c] > ptcap) { ptcap = T.nbody[c] * 2; pts = realloc(pts, 3 * sizeof(double) * ptcap); }
      for (int i = T.begin[c]; i < T.begin[c] + T.nbody[c]; i++) {
        pts[3 * np] = T.x[i]; pts[3 * np + 1] = T.y[i]; pts[3 * np + 2] = T.z[i];
        np++;
        if (T.sink[i]) T.has_sink[c] = 1;
      }
    } else {
      for (int ch = T.child[c]; ch < T.child[c] + T.nchild[c]; ch++) {
        if (T.has_sink[ch]) T.has_sink[c] = 1;
        int need = T.nchild[ch] == 0 ? T.nbody[ch] : 64 * T.nchild[ch];
        if (np + need > ptcap) { ptcap = 2 * (np + need); pts = realloc(pts, 3 * sizeof(double) * ptcap); }
        if (T.nchild[ch] == 0) {
          for (int i = T.begin[ch]; i < T.begin[ch] + T.nbody[ch]; i++) {
            pts[3 * np] = T.x[i]; pts[3 * np + 1] = T.y[i]; pts[3 * np + 2] = T.z[i];
            np++;
          }
        } else {
          for (int g = T.child[ch]; g < T.child[ch] + T.nchild[ch]; g++)
            for (int k = 0; k < 64; k++) {
              for (int d = 0; d < 3; d++) pts[3 * np + d] = T.X[3 * g + d] + T.R[g] * tc_tdesign[3 * k + d];
              np++;
            }
        }
      }
    }
    double cc[3], r2;
    tco_miniball(np, pts, cc, &r2);
    memcpy(T.X + 3 * c, cc, sizeof(cc));
    T.R[c] = sqrt(r2) + 1e-6;
    double* M = T.M + (size_t)c * nt;
    double* Md = jerk ? T.Md + (size_t)c * nt : NULL;
    if (T.nchild[c] == 0) {
      int b = T.begin[c], nb = T.nbody[c];
      double* mq = malloc(sizeof(double) * nb);
      for (int i = 0; i < nb; i++) mq[i] = T.m[b + i] * T.source[b + i];
      tco_p2m(p, nb, T.x + b, T.y + b, T.z + b, T.vx + b, T.vy + b, T.vz + b, mq, T.X + 3 * c, M, Md);
      free(mq);
    } else {
      for (int ch = T.child[c]; ch < T.child[c] + T.nchild[c]; ch++) {
        double dX[3] = {T.X[3 * ch] - T.X[3 * c], T.X[3 * ch + 1] - T.X[3 * c + 1], T.X[3 * ch + 2] - T.X[3 * c + 2]};
        tco_m2m(p, T.M + (size_t)ch * nt, jerk ? T.Md + (size_t)ch * nt : NULL, dX, M, Md);
      }
    }
  }
  free(pts);
}

/* ------------------------------------------------------------------------------------ */
/* Dual traversal with the theta MAC: traverse_eager.h:151-203 (top: tiny-cell P2P at   */
/* :160) and taichi_with_jerks/traverse_eager.h:125-155.  Records visited pairs.         */
/* ------------------------------------------------------------------------------------ */
static void rec(int kind, int a, int b) {
  long long* cnt = kind ? &T.np2p : &T.nm2l;
  long long* cap = kind ? &T.p2p_cap : &T.m2l_cap;
  int** ta = kind ? &T.p2p_t : &T.m2l_t;
  int** sa = kind ? &T.p2p_s : &T.m2l_s;
  if (*cnt == *cap) {
    *cap = *cap ? 2 * *cap : 4096;
    *ta = realloc(*ta, sizeof(int) * *cap);
    *sa = realloc(*sa, sizeof(int) * *cap);
  }
  (*ta)[*cnt] = a;
  (*sa)[*cnt] = b;
  (*cnt)++;
}

static void horizontal(int i, int j) {
  double dx = T.X[3 * i] - T.X[3 * j], dy = T.X[3 * i + 1] - T.X[3 * j + 1], dz = T.X[3 * i + 2] - T.X[3 * j + 2];
  double R2 = (dx * dx + dy * dy + dz * dz) * T.theta * T.theta;
  double rs = T.R[i] + T.R[j];
  if (R2 > rs * rs) {
    if (T.variant == TCO_VARIANT_TOP &&
        ((T.nbody[i] <= 2 && T.nbody[j] <= 8) || (T.nbody[j] <= 2 && T.nbody[i] <= 8)))
      rec(1, i, j);
    else
      rec(0, i, j);
  } else if (T.nchild[i] == 0 && T.nchild[j] == 0) {
    rec(1, i, j);
  } else if (T.nchild[j] == 0 || (T.R[i] >= T.R[j] && T.nchild[i] != 0)) {
    for (int c = T.child[i]; c < T.child[i] + T.nchild[i]; c++) horizontal(c, j);
  } else {
    for (int c = T.child[j]; c < T.child[j] + T.nchild[j]; c++) horizontal(i, c);
  }
}

/* P2P_simple (kernel_fast_lean.h:268-459) and jerk P2P (taichi_with_jerks :499-699) */
static void p2p(int ci, int cj, double* out) {
  int jerk = T.variant == TCO_VARIANT_JERKS;
  for (int i = T.begin[ci]; i < T.begin[ci] + T.nbody[ci]; i++) {
    if (!T.sink[i]) continue;
    double ax = 0, ay = 0, az = 0, pot = 0, jx = 0, jy = 0, jz = 0;
    for (int j = T.begin[cj]; j < T.begin[cj] + T.nbody[cj]; j++) {
      if (!T.source[j]) continue;
      double dx = T.x[j] - T.x[i], dy = T.y[j] - T.y[i], dz = T.z[j] - T.z[i];
      double r2 = dx * dx + dy * dy + dz * dz;
      if (!(r2 > 0)) continue;
      double invr = 1.0 / sqrt(r2), invr2 = invr * invr;
      double f = T.m[j] * invr;
      pot += f;
      f *= invr2;
      ax += dx * f; ay += dy * f; az += dz * f;
      if (jerk) {
        double dvx = T.vx[j] - T.vx[i], dvy = T.vy[j] - T.vy[i], dvz = T.vz[j] - T.vz[i];
        double vr = 3 * (dx * dvx + dy * dvy + dz * dvz);
        jx += dvx * f; jy += dvy * f; jz += dvz * f;
        f *= -invr2 * vr;
        jx += dx * f; jy += dy * f; jz += dz * f;
      }
    }
    double* o = out + 7 * (size_t)i;
    o[0] += pot; o[1] += ax; o[2] += ay; o[3] += az; o[4] += jx; o[5] += jy; o[6] += jz;
  }
}

/* P2P in the time-step pass (get_steps, top-level tree): kernel_fast_lean.h:462-548 (the
 * SIMD / DOUBLE_P2P branch the reference builds with).  Per target i and this source cell:
 * acc and pot as in P2P_simple (sources only), and the pairwise step
 *   tau1 = dt/sqrt2 r sqrt(r/mi) / (1 - dtau1/2),  dtau1 = min(1, 3/2 tau1 (d.dv)/r^2)
 *   tau2 = dt r/|dv|       / (1 - dtau2/2),  dtau2 = min(1, tau2 (d.dv)/r^2 (1 + mi/(v^2 r)))
 * minimised over the cell's bodies; the target's timestep gains 1/min^4.  As in the
 * reference, mi starts at the target's mass and accumulates every body of the cell met so
 * far (sources or not, self excluded), in the cell's body order. */
static void p2p_steps(int ci, int cj, double dtp, double* out, double* ts) {
  for (int i = T.begin[ci]; i < T.begin[ci] + T.nbody[ci]; i++) {
    double ax = 0, ay = 0, az = 0, pot = 0, tmin = 1e38, mi = T.m[i];
    for (int j = T.begin[cj]; j < T.begin[cj] + T.nbody[cj]; j++) {
      double mj = T.m[j];
      double dx = T.x[j] - T.x[i], dy = T.y[j] - T.y[i], dz = T.z[j] - T.z[i];
      double dvx = T.vx[j] - T.vx[i], dvy = T.vy[j] - T.vy[i], dvz = T.vz[j] - T.vz[i];
      double r2 = dx * dx + dy * dy + dz * dz;
      double v2 = dvx * dvx + dvy * dvy + dvz * dvz + 1e-20;
      if (!(r2 > 0)) { mj = 0; r2 = 1e38; }
      mi += mj;
      double vdotdr2 = (dx * dvx + dy * dvy + dz * dvz) / r2;
      double r = sqrt(r2), invr = 1 / r;
      double tau = dtp / M_SQRT2 * r * sqrt(r / mi);
      double dtau = 3 * tau * vdotdr2 / 2;
      if (!(dtau < 1)) dtau = 1;
      tau /= (1 - dtau / 2);
      if (tau < tmin) tmin = tau;
      tau = dtp * r / sqrt(v2);
      dtau = tau * vdotdr2 * (1 + mi / (v2 * r));
      if (!(dtau < 1)) dtau = 1;
      tau /= (1 - dtau / 2);
      if (tau < tmin) tmin = tau;
      mj *= invr;
      if (T.source[j]) {
        pot += mj;
        double f = mj * (invr * invr);
        ax += dx * f; ay += dy * f; az += dz * f;
      }
    }
    tmin *= tmin;
    tmin *= tmin;
    if (!T.sink[i]) continue;
    double* o = out + 7 * (size_t)i;
    o[0] += pot; o[1] += ax; o[2] += ay; o[3] += az;
    ts[i] += 1 / tmin;
  }
}

static void free_tree(void) {
  free(T.perm); free(T.x); free(T.y); free(T.z); free(T.vx); free(T.vy); free(T.vz); free(T.m);
  free(T.sink); free(T.source); free(T.X); free(T.R); free(T.has_sink);
  free(T.M); free(T.Md); free(T.L); free(T.Ld);
  free(T.begin); free(T.nbody); free(T.nchild); free(T.child); free(T.level); free(T.gx); free(T.R0c);
  free(T.m2l_t); free(T.m2l_s); free(T.p2p_t); free(T.p2p_s);
  memset(&T, 0, sizeof(T));
}

void tco_direct(int n, const double* x, const double* y, const double* z, const double* vx,
                const double* vy, const double* vz, const double* m, int nt, const int* targets,
                double* ax, double* ay, double* az, double* pot, double* jx, double* jy,
                double* jz) {
  for (int t = 0; t < nt; t++) {
    int i = targets ? targets[t] : t;
    double a[3] = {0, 0, 0}, ph = 0, jj[3] = {0, 0, 0};
    for (int j = 0; j < n; j++) {
      double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
      double r2 = dx * dx + dy * dy + dz * dz;
      if (!(r2 > 0)) continue;
      double invr = 1.0 / sqrt(r2), invr2 = invr * invr, f = m[j] * invr;
      ph += f;
      f *= invr2;
      a[0] += dx * f; a[1] += dy * f; a[2] += dz * f;
      if (vx) {
        double dvx = vx[j] - vx[i], dvy = vy[j] - vy[i], dvz = vz[j] - vz[i];
        double vr = 3 * (dx * dvx + dy * dvy + dz * dvz);
        jj[0] += dvx * f; jj[1] += dvy * f; jj[2] += dvz * f;
        double g = -f * invr2 * vr;
        jj[0] += dx * g; jj[1] += dy * g; jj[2] += dz * g;
      }
    }
    ax[t] = a[0]; ay[t] = a[1]; az[t] = a[2]; pot[t] = ph;
    if (jx) { jx[t] = jj[0]; jy[t] = jj[1]; jz[t] = jj[2]; }
  }
}

static int evaluate(const tco_params* prm, int n, const double* x, const double* y, const double* z,
                    const double* vx, const double* vy, const double* vz, const double* m,
                    const unsigned char* flags, double* ax, double* ay, double* az, double* pot,
                    double* jx, double* jy, double* jz, tco_stats* st, int steps, double dtp,
                    double* timestep);

int tco_evaluate(const tco_params* prm, int n, const double* x, const double* y, const double* z,
                 const double* vx, const double* vy, const double* vz, const double* m,
                 const unsigned char* flags, double* ax, double* ay, double* az, double* pot,
                 double* jx, double* jy, double* jz, tco_stats* st) {
  return evaluate(prm, n, x, y, z, vx, vy, vz, m, flags, ax, ay, az, pot, jx, jy, jz, st, 0, 0.0, NULL);
}

int tco_evaluate_steps(const tco_params* prm, double dt_param, int n, const double* x, const double* y,
                       const double* z, const double* vx, const double* vy, const double* vz, const double* m,
                       const unsigned char* flags, double* ax, double* ay, double* az, double* pot,
                       double* timestep, tco_stats* st) {
  if (prm->variant != TCO_VARIANT_TOP || !timestep) return -1;
  return evaluate(prm, n, x, y, z, vx, vy, vz, m, flags, ax, ay, az, pot, NULL, NULL, NULL, st, 1, dt_param,
                  timestep);
}

static int evaluate(const tco_params* prm, int n, const double* x, const double* y, const double* z,
                    const double* vx, const double* vy, const double* vz, const double* m,
                    const unsigned char* flags, double* ax, double* ay, double* az, double* pot,
                    double* jx, double* jy, double* jz, tco_stats* st, int steps, double dtp,
                    double* timestep) {
  if (n <= 0 || prm->p < 1 || prm->p > PMAX_O) return -1;
  int jerk = prm->variant == TCO_VARIANT_JERKS;
  free_tree();
  tco_init(prm->p);
  T.n = n; T.p = prm->p; T.variant = prm->variant; T.theta = prm->theta; T.ncrit = prm->ncrit;
  T.perm = malloc(sizeof(int) * n);
  double** arrs[7] = {&T.x, &T.y, &T.z, &T.vx, &T.vy, &T.vz, &T.m};
  const double* src[7] = {x, y, z, vx, vy, vz, m};
  for (int a = 0; a < 7; a++) {
    *arrs[a] = malloc(sizeof(double) * n);
    if (src[a]) memcpy(*arrs[a], src[a], sizeof(double) * n);
    else memset(*arrs[a], 0, sizeof(double) * n);
  }
  T.sink = malloc(n);
  T.source = malloc(n);
  for (int i = 0; i < n; i++) {
    T.sink[i] = flags ? (flags[i] & 1) : 1;
    T.source[i] = flags ? ((flags[i] >> 1) & 1) : 1;
  }
  double* out = calloc((size_t)7 * n, sizeof(double));
  double* ts = steps ? calloc((size_t)n, sizeof(double)) : NULL;
  if (n < prm->direct_below && !steps) {
    /* direct(), traverse_eager.h:349-370: every target against every source */
    for (int i = 0; i < n; i++) T.perm[i] = i;
    T.ncell = 0;
    for (int i = 0; i < n; i++) {
      if (!T.sink[i]) continue;
      double* o = out + 7 * (size_t)i;
      for (int j = 0; j < n; j++) {
        if (!T.source[j]) continue;
        double dx = T.x[j] - T.x[i], dy = T.y[j] - T.y[i], dz = T.z[j] - T.z[i];
        double r2 = dx * dx + dy * dy + dz * dz;
        if (!(r2 > 0)) continue;
        double invr = 1.0 / sqrt(r2), invr2 = invr * invr, f = T.m[j] * invr;
        o[0] += f;
        f *= invr2;
        o[1] += dx * f; o[2] += dy * f; o[3] += dz * f;
        if (jerk) {
          double dvx = T.vx[j] - T.vx[i], dvy = T.vy[j] - T.vy[i], dvz = T.vz[j] - T.vz[i];
          double vr = 3 * (dx * dvx + dy * dvy + dz * dvz);
          o[4] += dvx * f; o[5] += dvy * f; o[6] += dvz * f;
          double g = -f * invr2 * vr;
          o[4] += dx * g; o[5] += dy * g; o[6] += dz * g;
        }
      }
    }
  } else {
    build_tree(prm);
    int nc = T.ncell, nt = NT(prm->p);
    T.X = calloc((size_t)3 * nc, sizeof(double));
    T.R = calloc(nc, sizeof(double));
    T.has_sink = calloc(nc, 1);
    T.M = calloc((size_t)nc * nt, sizeof(double));
    T.L = calloc((size_t)nc * nt, sizeof(double));
    if (jerk) {
      T.Md = calloc((size_t)nc * nt, sizeof(double));
      T.Ld = calloc((size_t)nc * nt, sizeof(double));
    }
    upward();
    horizontal(0, 0);
    if (steps) {
      /* time-step pass (traverse_eager.h:151-203 with get_steps): no M2L, no local
       * expansions; every recorded P2P pair with the criterion */
      for (long long k = 0; k < T.np2p; k++)
        if (T.has_sink[T.p2p_t[k]]) p2p_steps(T.p2p_t[k], T.p2p_s[k], dtp, out, ts);
      goto done;
    }
    /* M2L over the visited pairs (top: mutual form, kernel_fast_lean.h:1036 -> one call
     * per direction, skipped when neither cell has a sink; jerks: one-sided). */
    for (long long k = 0; k < T.nm2l; k++) {
      int i = T.m2l_t[k], j = T.m2l_s[k];
      double dX[3] = {T.X[3 * i] - T.X[3 * j], T.X[3 * i + 1] - T.X[3 * j + 1], T.X[3 * i + 2] - T.X[3 * j + 2]};
      if (jerk) {
        if (T.has_sink[i])
          tco_m2l_rotate(prm->p, T.M + (size_t)j * nt, T.Md + (size_t)j * nt, dX, T.L + (size_t)i * nt,
                         T.Ld + (size_t)i * nt);
      } else {
        if (i > j || (!T.has_sink[i] && !T.has_sink[j])) continue;
        double mdX[3] = {-dX[0], -dX[1], -dX[2]};
        if (T.has_sink[i]) tco_m2l_rotate(prm->p, T.M + (size_t)j * nt, NULL, dX, T.L + (size_t)i * nt, NULL);
        if (T.has_sink[j]) tco_m2l_rotate(prm->p, T.M + (size_t)i * nt, NULL, mdX, T.L + (size_t)j * nt, NULL);
      }
    }
    for (long long k = 0; k < T.np2p; k++)
      if (T.has_sink[T.p2p_t[k]]) p2p(T.p2p_t[k], T.p2p_s[k], out);
    /* downward pass, traverse_eager.h:326-346 (parents precede children in cell order) */
    for (int c = 0; c < nc; c++) {
      if (T.nchild[c]) {
        for (int ch = T.child[c]; ch < T.child[c] + T.nchild[c]; ch++) {
          double dX[3] = {T.X[3 * c] - T.X[3 * ch], T.X[3 * c + 1] - T.X[3 * ch + 1], T.X[3 * c + 2] - T.X[3 * ch + 2]};
          tco_l2l(prm->p, T.L + (size_t)c * nt, jerk ? T.Ld + (size_t)c * nt : NULL, dX, T.L + (size_t)ch * nt,
                  jerk ? T.Ld + (size_t)ch * nt : NULL);
        }
      } else {
        for (int i = T.begin[c]; i < T.begin[c] + T.nbody[c]; i++) {
          if (!T.sink[i]) continue;
          double dX[3] = {T.X[3 * c] - T.x[i], T.X[3 * c + 1] - T.y[i], T.X[3 * c + 2] - T.z[i]};
          double v[3] = {T.vx[i], T.vy[i], T.vz[i]};
          tco_l2p(prm->p, T.L + (size_t)c * nt, jerk ? T.Ld + (size_t)c * nt : NULL, dX, v, out + 7 * (size_t)i);
        }
      }
    }
  }
done:
  for (int s = 0; s < n; s++) {
    int i = T.perm[s];
    const double* o = out + 7 * (size_t)s;
    pot[i] = o[0]; ax[i] = o[1]; ay[i] = o[2]; az[i] = o[3];
    if (jx) { jx[i] = o[4]; jy[i] = o[5]; jz[i] = o[6]; }
    if (ts) timestep[i] = ts[s];
  }
  if (st) {
    st->n_cells = T.ncell;
    long long nl = 0;
    for (int c = 0; c < T.ncell; c++) nl += T.nchild[c] == 0;
    st->n_leaves = nl;
    st->n_m2l = T.nm2l;
    st->n_p2p = T.np2p;
    long long inter = 0;
    for (long long k = 0; k < T.np2p; k++) inter += (long long)T.nbody[T.p2p_t[k]] * T.nbody[T.p2p_s[k]];
    st->n_p2p_inter = inter;
    st->max_level = T.max_level;
  }
  free(out);
  free(ts);
  return 0;
}

int tco_last_ncell(void) { return T.ncell; }

void tco_last_cells(int* begin, int* nbody, int* nchild, int* child, int* level, double* X,
                    double* R, int* perm) {
  for (int c = 0; c < T.ncell; c++) {
    begin[c] = T.begin[c]; nbody[c] = T.nbody[c]; nchild[c] = T.nchild[c]; child[c] = T.child[c];
    level[c] = T.level[c];
    if (X) memcpy(X + 3 * c, T.X + 3 * c, 3 * sizeof(double));
    if (R) R[c] = T.R[c];
  }
  if (perm) memcpy(perm, T.perm, sizeof(int) * T.n);
}

void tco_last_expansions(double* M, double* Md, double* L, double* Ld) {
  size_t sz = (size_t)T.ncell * NT(T.p) * sizeof(double);
  if (M) memcpy(M, T.M, sz);
  if (L) memcpy(L, T.L, sz);
  if (Md && T.Md) memcpy(Md, T.Md, sz);
  if (Ld && T.Ld) memcpy(Ld, T.Ld, sz);
}

long long tco_last_list(int kind, int* tgt, int* src) {
  long long n = kind ? T.np2p : T.nm2l;
  if (tgt) memcpy(tgt, kind ? T.p2p_t : T.m2l_t, sizeof(int) * n);
  if (src) memcpy(src, kind ? T.p2p_s : T.m2l_s, sizeof(int) * n);
  return n;
}

/* ---- integrator diagnostics and compensated drift (integrator.h:42, :642-656, :887-925) ---- */
void tco_system_diagnostics(int n, const double* m, const double* x, const double* y, const double* z,
                            const double* vx, const double* vy, const double* vz, const double* pot,
                            double* out) {
  long double kin = 0, pe = 0, mass = 0, pos[3] = {0, 0, 0}, vel[3] = {0, 0, 0};
  for (int i = 0; i < n; i++) {
    volatile double v2 = vx[i] * vx[i];
    volatile double t;
    v2 = v2 + vy[i] * vy[i];
    v2 = v2 + vz[i] * vz[i];
    t = m[i] * v2;
    kin += t / 2;
    t = m[i] * pot[i];
    pe += t / 2;
  }
  for (int i = 0; i < n; i++) {
    pos[0] += (long double)m[i] * x[i];
    pos[1] += (long double)m[i] * y[i];
    pos[2] += (long double)m[i] * z[i];
    vel[0] += (long double)m[i] * vx[i];
    vel[1] += (long double)m[i] * vy[i];
    vel[2] += (long double)m[i] * vz[i];
    mass += (long double)m[i];
  }
  out[0] = (double)kin;
  out[1] = (double)pe;
  out[2] = (double)mass;
  for (int d = 0; d < 3; d++) {
    out[3 + d] = (double)(pos[d] / mass);
    out[6 + d] = (double)(vel[d] / mass);
  }
}

void tco_drift_compsum(int n, double* s, double* e, const double* v, double dt) {
  for (int i = 0; i < n; i++) {
    double a = s[i];
    e[i] = fma(dt, v[i], e[i]);
    s[i] = a + e[i];
    e[i] += a - s[i];
  }
}
