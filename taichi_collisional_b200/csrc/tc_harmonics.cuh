// Complex helpers and solid-harmonic column recurrences (device).
//
// make_Gnm (kernel_fast_lean.h:235-266) builds the regular solid harmonics G[n][m] with
//   G[m][m]   = G[m-1][m-1] * (x + i y) / (2m)
//   G[m+1][m] = z G[m][m]
//   G[n][m]   = ((2n-1) z G[n-1][m] - r^2 G[n-2][m]) / (n^2 - m^2)
// and G[n][-m] = (-1)^m conj(G[n][m]).  For fixed m this is a recurrence in n alone, so a
// GPU thread can produce one column m with O(1) state; the device kernels use that form.
// make_Gnmdot (taichi_with_jerks/kernel_fast_lean.h:272-304) needs columns m-1, m, m+1 of the
// previous degree, which TcCols3 carries together.
#pragma once
#include "tc_common.cuh"

namespace tc {

struct cd {
  double x, y;
};
__device__ __forceinline__ cd mk(double a, double b) { return cd{a, b}; }
__device__ __forceinline__ cd operator+(cd a, cd b) { return cd{a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ cd operator-(cd a, cd b) { return cd{a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ cd operator*(cd a, cd b) { return cd{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
__device__ __forceinline__ cd operator*(double s, cd a) { return cd{s * a.x, s * a.y}; }
__device__ __forceinline__ cd conj(cd a) { return cd{a.x, -a.y}; }
__device__ __forceinline__ cd& operator+=(cd& a, cd b) { a.x += b.x; a.y += b.y; return a; }

// One column c >= 0 of G, advanced one degree at a time.
struct TcCol {
  int c;
  cd diag;      // G[c][c]
  cd g1, g2;    // G[n-1][c], G[n-2][c]
  __device__ __forceinline__ void init(int col, cd dg) { c = col; diag = dg; g1 = mk(0, 0); g2 = mk(0, 0); }
  // returns G[n][c] for the next n (call with n = 0, 1, 2, ... in order)
  __device__ __forceinline__ cd step(int n, double dz, double r2) {
    cd g;
    if (n < c) g = mk(0, 0);
    else if (n == c) g = diag;
    else if (n == c + 1) g = dz * diag;
    else {
      double m2 = (double)(n * n - c * c);
      g = ((2 * n - 1.) / m2 * dz) * g1 - (r2 / m2) * g2;
    }
    g2 = g1;
    g1 = g;
    return g;
  }
};

// Diagonal G[j][j] for j = 0..jmax, returning the values at j = a-1, a, a+1 (0 when < 0).
__device__ __forceinline__ void tc_diag3(int a, double dx, double dy, cd& dm1, cd& d0, cd& dp1) {
  cd d = mk(1, 0);
  dm1 = mk(0, 0);
  d0 = a == 0 ? d : mk(0, 0);
  dp1 = mk(0, 0);
  if (a == 0) {
    dp1 = d * mk(dx / 2, dy / 2);
    return;
  }
  for (int j = 1; j <= a + 1; j++) {
    d = d * mk(dx / (2 * j), dy / (2 * j));
    if (j == a - 1) dm1 = d;
    if (j == a) d0 = d;
    if (j == a + 1) dp1 = d;
  }
  if (a == 1) dm1 = mk(1, 0);
}

// Three neighbouring columns a-1, a, a+1 of G (column -1 is -conj(column 1)).
struct TcCols3 {
  TcCol A, B, C;
  int a;
  __device__ __forceinline__ void init(int col, double dx, double dy) {
    a = col;
    cd dm1, d0, dp1;
    tc_diag3(col, dx, dy, dm1, d0, dp1);
    A.init(col > 0 ? col - 1 : 1, col > 0 ? dm1 : dp1);
    B.init(col, d0);
    C.init(col + 1, dp1);
  }
  // G[n][a-1], G[n][a], G[n][a+1]
  __device__ __forceinline__ void step(int n, double dz, double r2, cd& ga, cd& gb, cd& gc) {
    gc = C.step(n, dz, r2);
    gb = B.step(n, dz, r2);
    cd t = A.step(n, dz, r2);
    ga = a > 0 ? t : mk(-gc.x, gc.y);  // G[n][-1] = -conj(G[n][1])
  }
};

// real storage (n*n+n+m: +m Re, -m Im of the m >= 0 coefficient) -> complex at (n, m), any m
__device__ __forceinline__ cd tc_r2c(const double* r, int n, int m) {
  int is = n * n + n;
  if (m == 0) return mk(r[is], 0);
  if (m > 0) return mk(r[is + m], r[is - m]);
  int am = -m;
  double s = (am & 1) ? -1.0 : 1.0;
  return mk(s * r[is + am], -s * r[is - am]);
}

}  // namespace tc
