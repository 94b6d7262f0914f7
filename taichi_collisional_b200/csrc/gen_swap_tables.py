#!/usr/bin/env python3
"""Derive the constant x<->z "swap" matrices of the rotation-based M2L from first principles.

The reference applies a fixed per-degree linear map four times in every M2L
(kernel_fast_lean.h:1113-1118, :1147-1152, :1203-1208, :1238-1243 and the
generated straight-line code in multipole_rotation_matrix/rotate_order_{3..30}.txt,
included by kernel_rotate.h:25-52; degrees 1-2 are hard-coded at kernel_rotate.h:11-22).
That map is the change of coordinates (x, y, z) -> (z, y, x) expressed on the
coefficients of the regular solid harmonics G_n^m produced by ``make_Gnm``
(kernel_fast_lean.h:235-266), in the reference's real storage (index n*n+n+m:
+m holds Re, -m holds Im of the m>=0 complex coefficient; kernel_fast_lean.h:179-191)
and scaled by (n+|m|)!(n-|m|)! ("homogeneous form", kernel_fast_lean.h:1083-1084).

Here the map is derived with exact rational arithmetic:

  B_k(x,y,z)   = Re/Im of G_n^|m| built by the same recurrence as make_Gnm
  B_k o swap   = sum_j A[k][j] B_j          (solved exactly over Q)
  S[k][j]      = D_k A[k][j] / D_j,  D_k = (n+|m|)!(n-|m|)!

Every S entry is an integer times 2^-(n-1) (degree >= 1); tests compare the derived
integers with the reference's rotate_order files entry by entry.

Outputs (written next to this script):
  swap_tables.h   CSR table (host + device) and straight-line per-degree device
                  functions ``tc_swap_deg<N>`` used by the CUDA M2L kernels.

Run:  python gen_swap_tables.py [PMAX]     (default PMAX = 20)
"""
from fractions import Fraction
import math
import os
import sys


def _padd(a, b, s=Fraction(1)):
    out = dict(a)
    for k, v in b.items():
        out[k] = out.get(k, Fraction(0)) + s * v
        if out[k] == 0:
            del out[k]
    return out


def _pscale(a, s):
    if s == 0:
        return {}
    return {k: v * s for k, v in a.items()}


def _pmul_mono(a, mono):
    dx, dy, dz = mono
    return {(k[0] + dx, k[1] + dy, k[2] + dz): v for k, v in a.items()}


def _cmul_lin(c, lx, ly, s):
    """(re, im) complex polynomial times (x*lx + i*y*ly) * s."""
    re, im = c
    # (re + i im) * (x + i y)  ->  re*x - im*y  +  i (re*y + im*x)
    nre = _padd(_pmul_mono(re, (1, 0, 0)), _pmul_mono(im, (0, 1, 0)), Fraction(-1))
    nim = _padd(_pmul_mono(re, (0, 1, 0)), _pmul_mono(im, (1, 0, 0)))
    return (_pscale(nre, s), _pscale(nim, s))


def regular_harmonics(pmax):
    """G[n][m] (m >= 0) as exact complex polynomials, same recurrence as make_Gnm."""
    G = [[None] * (n + 1) for n in range(pmax + 1)]
    G[0][0] = ({(0, 0, 0): Fraction(1)}, {})
    r2 = {(2, 0, 0): Fraction(1), (0, 2, 0): Fraction(1), (0, 0, 2): Fraction(1)}
    for n in range(1, pmax + 1):
        G[n][n] = _cmul_lin(G[n - 1][n - 1], 1, 1, Fraction(1, 2 * n))
        for m in range(0, n - 1):
            m2 = n * n - m * m
            a_re = _pscale(_pmul_mono(G[n - 1][m][0], (0, 0, 1)), Fraction(2 * n - 1, m2))
            a_im = _pscale(_pmul_mono(G[n - 1][m][1], (0, 0, 1)), Fraction(2 * n - 1, m2))
            b_re = {}
            b_im = {}
            for mono in ((2, 0, 0), (0, 2, 0), (0, 0, 2)):
                b_re = _padd(b_re, _pmul_mono(G[n - 2][m][0], mono))
                b_im = _padd(b_im, _pmul_mono(G[n - 2][m][1], mono))
            G[n][m] = (_padd(a_re, b_re, Fraction(-1, m2)), _padd(a_im, b_im, Fraction(-1, m2)))
        G[n][n - 1] = (_pmul_mono(G[n - 1][n - 1][0], (0, 0, 1)),
                       _pmul_mono(G[n - 1][n - 1][1], (0, 0, 1)))
    return G


def _basis(G, n):
    """Real basis of degree n in storage order m = -n..n."""
    out = []
    for m in range(-n, n + 1):
        re, im = G[n][abs(m)]
        out.append(im if m < 0 else re)
    return out


def _swap_xz(poly):
    return {(k[2], k[1], k[0]): v for k, v in poly.items()}


def _solve(Amat, rhs):
    """Exact Gauss-Jordan: solve Amat X = rhs (lists of Fractions), returns X."""
    n = len(Amat)
    M = [row[:] + r[:] for row, r in zip(Amat, rhs)]
    ncol = len(M[0])
    for col in range(n):
        piv = next(r for r in range(col, n) if M[r][col] != 0)
        M[col], M[piv] = M[piv], M[col]
        inv = 1 / M[col][col]
        M[col] = [v * inv for v in M[col]]
        for r in range(n):
            if r != col and M[r][col] != 0:
                f = M[r][col]
                M[r] = [a - f * b for a, b in zip(M[r], M[col])]
    return [row[n:ncol] for row in M]


def swap_matrix(G, n):
    """S (list of lists of Fractions, (2n+1)^2) for degree n; rows = output index."""
    basis = _basis(G, n)
    monos = [(a, n - a, 0) for a in range(n + 1)] + [(a, n - 1 - a, 1) for a in range(n)]
    # Bmat[mono][j] = coefficient of mono in basis j
    Bmat = [[basis[j].get(mo, Fraction(0)) for j in range(2 * n + 1)] for mo in monos]
    targets = [_swap_xz(b) for b in basis]
    rhs = [[targets[k].get(mo, Fraction(0)) for k in range(2 * n + 1)] for mo in monos]
    X = _solve(Bmat, rhs)          # X[j][k]: coefficient of basis j in target k
    A = [[X[j][k] for j in range(2 * n + 1)] for k in range(2 * n + 1)]
    D = [math.factorial(n + abs(m)) * math.factorial(n - abs(m)) for m in range(-n, n + 1)]
    return [[A[k][j] * D[k] / D[j] for j in range(2 * n + 1)] for k in range(2 * n + 1)]


def orthogonal_form(S, n):
    """T = E S E^-1 (float64 entries), orthogonal; E_k = c_k / sqrt(D_k)."""
    D = [math.factorial(n + abs(m)) * math.factorial(n - abs(m)) for m in range(-n, n + 1)]
    E = [(1.0 if m == 0 else math.sqrt(2.0)) / math.sqrt(D[m + n]) for m in range(-n, n + 1)]
    out = []
    for k in range(2 * n + 1):
        row = []
        for j in range(2 * n + 1):
            v = S[k][j]
            row.append(0.0 if v == 0 else float(v) * E[k] / E[j])
        out.append(row)
    return out


def derive(pmax):
    G = regular_harmonics(pmax)
    return [swap_matrix(G, n) for n in range(pmax + 1)]


def integer_rows(S, n):
    """Entries scaled by 2^(n-1) (degree >= 1): must all be integers."""
    scale = Fraction(2) ** (n - 1) if n >= 1 else Fraction(1)
    out = []
    for row in S:
        r = []
        for v in row:
            w = v * scale
            assert w.denominator == 1, (n, v)
            r.append(int(w))
        out.append(r)
    return out


def _fmt(v):
    return repr(float(v)) if float(v) != int(float(v)) or abs(float(v)) >= 2 ** 53 else "%d.0" % int(v)


def write_header(mats, path):
    pmax = len(mats) - 1
    nterm = (pmax + 1) ** 2
    rowptr, cols, vals = [0], [], []
    for n, S in enumerate(mats):
        for k in range(2 * n + 1):
            for j in range(2 * n + 1):
                if S[k][j] != 0:
                    cols.append(n * n + j)
                    vals.append(S[k][j])
            rowptr.append(len(cols))
    L = []
    L.append("// Generated by gen_swap_tables.py -- do not edit.")
    L.append("// Per-degree x<->z swap matrices of the rotation M2L in scaled real storage")
    L.append("// (index n*n+n+m), derived with exact rational arithmetic.")
    L.append("#pragma once")
    L.append("#define TC_SWAP_PMAX %d" % pmax)
    L.append("#define TC_SWAP_NNZ %d" % len(cols))
    L.append("#ifdef __CUDACC__")
    L.append("#define TC_SWAP_HD __host__ __device__")
    L.append("#else")
    L.append("#define TC_SWAP_HD")
    L.append("#endif")
    L.append("static const int tc_swap_rowptr[%d] = {%s};" % (nterm + 1, ",".join(map(str, rowptr))))
    L.append("static const unsigned short tc_swap_col[%d] = {%s};" % (len(cols), ",".join(map(str, cols))))
    L.append("static const double tc_swap_val[%d] = {%s};" % (len(vals), ",".join(_fmt(v) for v in vals)))
    L.append("#ifdef __CUDACC__")
    L.append("// Straight-line per-degree application: o[k] = sum_j S_n[k][j] v[j], k,j in [0,2n+1).")
    L.append("template <int N> struct TcSwapDeg;")
    for n, S in enumerate(mats):
        L.append("template <> struct TcSwapDeg<%d> {" % n)
        L.append("  template <typename T> static __device__ __forceinline__ void apply(const T* v, T* o) {")
        for k in range(2 * n + 1):
            terms = []
            for j in range(2 * n + 1):
                if S[k][j] != 0:
                    terms.append("T(%s) * v[%d]" % (_fmt(S[k][j]), j))
            L.append("    o[%d] = %s;" % (k, " + ".join(terms) if terms else "T(0)"))
        L.append("  }")
        L.append("};")
    L.append("// Orthogonal form used by the mixed-precision M2L: T_n = E S_n E^-1 with")
    L.append("// E = diag(sqrt((n+|m|)!(n-|m|)!) c_m / ((n+|m|)!(n-|m|)!)), c_0 = 1, c_m = sqrt(2).")
    L.append("template <int N> struct TcSwapOrthDeg;")
    for n, S in enumerate(mats):
        T = orthogonal_form(S, n)
        L.append("template <> struct TcSwapOrthDeg<%d> {" % n)
        L.append("  template <typename T> static __device__ __forceinline__ void apply(const T* v, T* o) {")
        for k in range(2 * n + 1):
            terms = ["T(%r) * v[%d]" % (T[k][j], j) for j in range(2 * n + 1) if T[k][j] != 0.0]
            L.append("    o[%d] = %s;" % (k, " + ".join(terms) if terms else "T(0)"))
        L.append("  }")
        L.append("};")
    L.append("#endif")
    with open(path, "w") as f:
        f.write("\n".join(L) + "\n")


def main():
    pmax = int(sys.argv[1]) if len(sys.argv) > 1 else 20
    mats = derive(pmax)
    for n in range(1, pmax + 1):
        integer_rows(mats[n], n)
    here = os.path.dirname(os.path.abspath(__file__))
    write_header(mats, os.path.join(here, "swap_tables.h"))


if __name__ == "__main__":
    main()
