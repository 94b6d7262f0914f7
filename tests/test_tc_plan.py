"""The tensor-core far field's plan and constant matrices, checked on the CPU.

The kernel (taichi_collisional_b200/csrc/tc_m2l_tc.cuh) evaluates the rotation M2L as
phase rotations plus products with constant block matrices laid out by m2l_tc_plan.h.
Here the same pipeline is replayed in float64 with numpy from the generator's plan and the
library's TF32 (hi + lo) bin matrices, and compared with the oracle's FP64 rotation M2L
(taichi_with_jerks/kernel_fast_lean.h:1130-1371 restated in oracle/tc_oracle.c).
"""
import math
import os
import sys

import numpy as np
import pytest

import oracle
import taichi_collisional_b200 as tcb

sys.path.insert(0, os.path.join(os.path.dirname(tcb.__file__), "csrc"))
import gen_tc_plan as plan  # noqa: E402


def bin_index(n, k):
    return (n >> 3) * 128 + (k >> 2) * 32 + (n & 7) * 4 + (k & 3)


def bins_as_matrices(q):
    hi, lo = tcb.tc_bins(q)
    full = hi.astype(np.float64) + lo.astype(np.float64)
    mats = np.zeros((full.shape[0], 16, 16))
    for o in range(16):
        for k in range(16):
            mats[:, o, k] = full[:, bin_index(o, k)]
    return mats


def pair_geo(d):
    dx, dy, dz = d
    rxy = math.hypot(dx, dy)
    r = math.sqrt(dx * dx + dy * dy + dz * dz)
    ez1 = complex(dy / rxy, dx / rxy) if rxy > 0 else complex(1, 0)
    ex1 = complex(dz / r, -rxy / r)
    return 1.0 / r, ez1, ex1


def rotate(v, q, e1, inv):
    e = e1
    for m in range(1, q + 1):
        for n in range(m, q + 1):
            i, j = n * n + n - m, n * n + n + m
            im, re = v[i], v[j]
            if not inv:
                v[i], v[j] = e.real * im + e.imag * re, e.real * re - e.imag * im
            else:
                v[i], v[j] = e.real * im - e.imag * re, e.real * re + e.imag * im
        e = e * e1


def swap(v, q, mats):
    out = np.zeros_like(v)
    for s_, sb in enumerate(plan.superbins(q)):
        for part, hh in zip(plan.positions(sb), (2 * s_, 2 * s_ + 1)):
            idx = [plan.nat(*nm) if nm else None for nm in part]
            x = np.array([v[i] if i is not None else 0.0 for i in idx])
            y = mats[hh] @ x
            for o, i in enumerate(idx):
                if i is not None:
                    out[i] = y[o]
    return out


def translate(v, q, mats, nh):
    out = np.zeros_like(v)
    for u, pos in enumerate(plan.trans_positions(q)):
        for sgn in (1, -1):
            idx = [plan.nat(n, sgn * m) if (n is not None and not (sgn < 0 and m == 0)) else None
                   for n, m in [(p if p else (None, None)) for p in pos]]
            x = np.array([v[i] if i is not None else 0.0 for i in idx])
            y = mats[nh + u] @ x
            for o, i in enumerate(idx):
                if i is not None:
                    out[i] = y[o]
    return out


def tc_m2l(q, M, d, mats):
    nh = 2 * len(plan.superbins(q))
    rinv, ez1, ex1 = pair_geo(d)
    v = np.zeros((q + 1) ** 2)
    F = np.zeros_like(v)
    DoF = np.zeros_like(v)
    for n in range(q + 1):
        for m in range(-n, n + 1):
            a = abs(m)
            D = math.factorial(n + a) * math.factorial(n - a)
            F[n * n + n + m] = math.sqrt(D) * (math.sqrt(2.0) if a else 1.0)
            DoF[n * n + n + m] = D / F[n * n + n + m]
            v[n * n + n + m] = M[n * n + n + m] * F[n * n + n + m] * rinv ** n
    v[q * q] = 0.0
    v[q * q + 2 * q] = 0.0
    rotate(v, q, ez1, False)
    v = swap(v, q, mats)
    rotate(v, q, ex1, False)
    v = swap(v, q, mats)
    v = translate(v, q, mats, nh)
    v = swap(v, q, mats)
    rotate(v, q, ex1, True)
    v = swap(v, q, mats)
    rotate(v, q, ez1, True)
    return np.array([v[k] * DoF[k] * rinv ** (int(math.isqrt(k)) + 1) for k in range(len(v))])


@pytest.mark.parametrize("q", [4, 6, 8, 10, 12])
def test_plan_covers_every_coefficient(q):
    seen = []
    for sb in plan.superbins(q):
        d1, d2, _ = sb
        assert d1 + max(d2, 0) <= 14
        re, im = plan.positions(sb)
        for i in range(16):  # the order m of position i is i, 15 - i or 0
            for nm in (re[i], im[i]):
                if nm:
                    assert abs(nm[1]) in (i, 15 - i, 0)
        seen += [plan.nat(*nm) for nm in re + im if nm]
    assert sorted(seen) == list(range((q + 1) ** 2))
    tr = [p for b in plan.trans_positions(q) for p in b if p]
    assert sorted(tr) == sorted((k, m) for m in range(q // 2 + 1) for k in range(m, q - m + 1))


@pytest.mark.parametrize("q", [4, 6, 8, 10, 12])
def test_swap_bins_are_orthogonal(q):
    mats = bins_as_matrices(q)
    for s_, sb in enumerate(plan.superbins(q)):
        for part, hh in zip(plan.positions(sb), (2 * s_, 2 * s_ + 1)):
            live = [i for i, nm in enumerate(part) if nm]
            T = mats[hh][np.ix_(live, live)]
            assert np.abs(T @ T.T - np.eye(len(live))).max() < 1e-6
            dead = [i for i in range(16) if i not in live]
            assert not np.any(mats[hh][dead, :]) and not np.any(mats[hh][:, dead])


@pytest.mark.parametrize("q", [4, 8, 12])
def test_tensor_core_pipeline_matches_rotation_m2l(q):
    L = oracle.lib()
    L.tco_init(q)
    dp = oracle._dp
    mats = bins_as_matrices(q)
    rng = np.random.default_rng(q)
    nt = (q + 1) ** 2
    for _ in range(4):
        pts = rng.normal(size=(30, 3)) * 0.3
        m = rng.uniform(0.5, 1.0, size=30)
        C = np.zeros(3)
        M = np.zeros(nt)
        xs, ys, zs = (np.ascontiguousarray(pts[:, k]) for k in range(3))
        L.tco_p2m(q, 30, xs.ctypes.data_as(dp), ys.ctypes.data_as(dp), zs.ctypes.data_as(dp), None, None, None,
                  m.ctypes.data_as(dp), C.ctypes.data_as(dp), M.ctypes.data_as(dp), None)
        d = rng.normal(size=3)
        d *= 3.0 / np.linalg.norm(d)
        Lr = np.zeros(nt)
        L.tco_m2l_rotate(q, M.ctypes.data_as(dp), None, d.ctypes.data_as(dp), Lr.ctypes.data_as(dp), None)
        Lt = tc_m2l(q, M, d, mats)
        # per degree, relative to the degree's norm (TF32 hi + lo matrices: ~1e-7)
        for n in range(q + 1):
            sl = slice(n * n, n * n + 2 * n + 1)
            ref = np.abs(Lr[sl]).max()
            assert np.abs(Lt[sl] - Lr[sl]).max() <= 2e-6 * ref + 1e-300, (n, Lt[sl], Lr[sl])
