#!/usr/bin/env python3
"""Column plans of the tensor-core M2L (tc_m2l_tc.cuh).

The tensor-core M2L applies the constant per-pair contractions of the rotation M2L -- the
x<->z swap (one orthogonal matrix per degree) and the z-translation (one matrix per order m)
-- as tcgen05 MMAs over 128-pair tiles (M = 128 rows, one thread per row).

Swap layout ("super-bins").  The swap x<->z leaves y alone, and Re / Im of G_n^m are even /
odd in y, so the swap of degree n is two blocks: real parts (m = 0..n) and imaginary parts
(m = 1..n).  A super-bin is 32 columns, a real half and an imaginary half of 16, holding two
degrees D1 >= D2 with D1 + D2 <= 14:
    position i <= D1          : (D1, m = i)
    position i >= 15 - D2     : (D2, m = 15 - i)
(real half: +m; imaginary half: -m, its m = 0 positions stay zero), and one super-bin also
carries degree 0 at position D1 + 1.  Every position's order m is then i, 15 - i or 0, so one
loop body rotates every super-bin (the phase e^{i m a} of position i is selected from two
fixed register indices), and each half is one block-diagonal 16 x 16 product.

Translation layout.  Along z the order m is kept and input degree k maps to output degree n
with n + k <= Q, the same matrix for the real and imaginary parts: for every m <= Q/2 one
block of size Q - 2m + 1 (row j <-> degree m + j).  Blocks are packed into 16-wide bins; bin
u occupies 32 columns, the real parts in its first 16 and the imaginary parts (same
positions) in its last 16, and both use the same matrix.

Output: m2l_tc_plan.h with, per order Q, the super-bin and translation tables (host
constexpr copies for building the bin matrices, __constant__ copies for the kernel).

Run:  python gen_tc_plan.py        (writes m2l_tc_plan.h next to this script)
"""
import os

ORDERS = (4, 6, 8, 10, 12)


def nat(n, m):
    return n * n + n + m


def superbins(q):
    """[(D1, D2, carries_degree_0)], D2 = -1 for none."""
    degs = list(range(q, 0, -1))
    out = []
    while degs:
        d1 = degs.pop(0)
        d2 = -1
        for e in degs:
            if d1 + e <= 14:
                d2 = e
                break
        if d2 >= 0:
            degs.remove(d2)
        out.append([d1, d2, 0])
    # degree 0 rides at position D1 + 1 of the last super-bin with room
    for sb in reversed(out):
        d1, d2 = sb[0], sb[1]
        if d1 + 1 < (15 - d2 if d2 >= 0 else 16):
            sb[2] = 1
            break
    else:
        out.append([0, -1, 0])
    return [tuple(s) for s in out]


def positions(sb):
    """(re_positions, im_positions): lists of 16 entries (n, m) or None."""
    d1, d2, z = sb
    re, im = [None] * 16, [None] * 16
    for i in range(16):
        if i <= d1:
            re[i] = (d1, i)
            im[i] = (d1, -i) if i >= 1 else None
        elif d2 >= 0 and i >= 15 - d2:
            m = 15 - i
            re[i] = (d2, m)
            im[i] = (d2, -m) if m >= 1 else None
        elif z and i == d1 + 1:
            re[i] = (0, 0)
    return re, im


def trans_plan(q):
    """[(m, bin u, offset within bin)], number of bins."""
    blocks = [(m, q - 2 * m + 1) for m in range(0, q // 2 + 1)]
    order = sorted(blocks, key=lambda b: -b[1])
    bins = []
    place = {}
    for m, size in order:
        for u, used in enumerate(bins):
            if used + size <= 16:
                place[m] = (u, used)
                bins[u] += size
                break
        else:
            place[m] = (len(bins), 0)
            bins.append(size)
    return [(m,) + place[m] for m in range(q // 2 + 1)], len(bins)


def trans_positions(q):
    """per bin u: 16 entries (n, m >= 0) or None, for the real arrangement."""
    tp, nb = trans_plan(q)
    out = [[None] * 16 for _ in range(nb)]
    for m, u, off in tp:
        for j in range(q - 2 * m + 1):
            out[u][off + j] = (m + j, m)
    return out


def emit(q):
    nt = (q + 1) ** 2
    sbs = superbins(q)
    nsb = len(sbs)
    seen = []
    for sb in sbs:
        re, im = positions(sb)
        seen += [nat(*p) for p in re + im if p is not None]
    assert sorted(seen) == list(range(nt)), q
    tp, ntb = trans_plan(q)
    half_nat = []
    for sb in sbs:
        re, im = positions(sb)
        half_nat.append([nat(*p) if p else -1 for p in re])
        half_nat.append([nat(*p) if p else -1 for p in im])
    tpos = trans_positions(q)
    tnat = [[nat(*p) if p else -1 for p in b] for b in tpos]
    dnat = [x for h in half_nat for x in h]
    L = []
    A = L.append

    def arr(v):
        return ",".join(map(str, v))

    A("__constant__ signed char c_tc_sb_%d[%d][3] = {%s};" % (q, nsb, ",".join("{%d,%d,%d}" % s for s in sbs)))
    A("__constant__ signed char c_tc_tr_%d[%d][2] = {%s};" % (q, q // 2 + 1, ",".join("{%d,%d}" % (u, o) for _, u, o in tp)))
    A("__constant__ short c_tc_dnat_%d[%d] = {%s};" % (q, 32 * nsb, arr(dnat)))
    # natural -> swap column; natural -> translation column (-1: not translated);
    # translation column -> natural (-1: padding)
    dcol = [0] * nt
    for j, k in enumerate(dnat):
        if k >= 0:
            dcol[k] = j
    tcol = [-1] * nt
    tnat_flat = [-1] * (32 * ntb)
    for m, u, off in tp:
        for j in range(q - 2 * m + 1):
            n = m + j
            for part, sgn in ((0, 1), (1, -1)):
                if m == 0 and part == 1:
                    continue
                c = 32 * u + 16 * part + off + j
                tcol[nat(n, sgn * m)] = c
                tnat_flat[c] = nat(n, sgn * m)
    A("__constant__ short c_tc_dcol_%d[%d] = {%s};" % (q, nt, arr(dcol)))
    A("__constant__ short c_tc_tcol_%d[%d] = {%s};" % (q, nt, arr(tcol)))
    A("__constant__ short c_tc_tnat_%d[%d] = {%s};" % (q, 32 * ntb, arr(tnat_flat)))
    A("template <> struct TcTcPlan<%d> {" % q)
    A("  static constexpr int NT = %d, NSB = %d, NH = %d, AW = %d, NTB = %d, TW = %d;" %
      (nt, nsb, 2 * nsb, 32 * nsb, ntb, 32 * ntb))
    A("  static constexpr short half_nat[%d][16] = {%s};" % (2 * nsb, ",".join("{%s}" % arr(h) for h in half_nat)))
    A("  static constexpr short trans_nat[%d][16] = {%s};" % (ntb, ",".join("{%s}" % arr(t) for t in tnat)))
    A("  static __device__ __forceinline__ int sb_d1(int s) { return c_tc_sb_%d[s][0]; }" % q)
    A("  static __device__ __forceinline__ int sb_d2(int s) { return c_tc_sb_%d[s][1]; }" % q)
    A("  static __device__ __forceinline__ int sb_zero(int s) { return c_tc_sb_%d[s][2]; }" % q)
    A("  static __device__ __forceinline__ int tr_bin(int m) { return c_tc_tr_%d[m][0]; }" % q)
    A("  static __device__ __forceinline__ int tr_off(int m) { return c_tc_tr_%d[m][1]; }" % q)
    A("  static __device__ __forceinline__ int d_nat(int j) { return c_tc_dnat_%d[j]; }" % q)
    A("  static __device__ __forceinline__ int d_col(int k) { return c_tc_dcol_%d[k]; }" % q)
    A("  static __device__ __forceinline__ int t_col(int k) { return c_tc_tcol_%d[k]; }" % q)
    A("  static __device__ __forceinline__ int t_nat(int c) { return c_tc_tnat_%d[c]; }" % q)
    A("};")
    return L


def main():
    here = os.path.dirname(os.path.abspath(__file__))
    L = ["// Generated by gen_tc_plan.py -- do not edit.",
         "// Tensor-core M2L plans: swap super-bins (two degrees per 32 columns, real half |",
         "// imaginary half, the second degree stored from the far end) and translation bins.",
         "#pragma once",
         "#define TC_TC_QMAX %d" % max(ORDERS),
         "namespace tc {",
         "template <int Q> struct TcTcPlan;"]
    for q in ORDERS:
        L.extend(emit(q))
    L.append("}  // namespace tc")
    with open(os.path.join(here, "m2l_tc_plan.h"), "w") as f:
        f.write("\n".join(L) + "\n")


if __name__ == "__main__":
    main()
