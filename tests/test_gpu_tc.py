"""Tensor-core far field (precision=TC_PREC_MIXED_M2L, p <= 12) against the FP64 form.

The FP64 form reproduces the reference's FMM at 1e-12 (test_gpu_parity.py); the tensor-core
M2L (tcgen05, TF32 hi/lo products, FP32 rotations) must agree with it at FP32 level: the
local expansions per cell, and the accelerations per body, and its error against FP64
direct sums must stay at the FP32 floor.
"""
import numpy as np
import pytest

import oracle
import taichi_collisional_b200 as tcb
from taichi_collisional_b200 import ics

pytestmark = pytest.mark.gpu


def run(prec, x, y, z, m, vx, vy, vz, p, theta=0.4, ncrit=64):
    g = tcb.Gravity(p=p, ncrit=ncrit, theta=theta, variant=tcb.VARIANT_JERKS, precision=prec)
    out = g.evaluate(x, y, z, m, vx, vy, vz)
    st = g.stats()
    _, _, L, _ = g.expansions()
    g.close()
    return out, st, L


@pytest.mark.parametrize("p,n", [(4, 1 << 14), (8, 1 << 16), (12, 1 << 16)])
def test_tc_far_field_matches_fp64(p, n):
    x, y, z, vx, vy, vz, m = ics.plummer(n, 100 + p)
    o64, s64, e64 = run(tcb.PREC_FP64, x, y, z, m, vx, vy, vz, p)
    otc, stc, etc = run(tcb.PREC_MIXED_M2L, x, y, z, m, vx, vy, vz, p)
    assert stc["flags"] == 0
    assert stc["n_m2l"] == s64["n_m2l"] and stc["n_m2l"] > 0
    # local expansions, per cell and degree, relative to the degree's largest coefficient
    L64, Ltc = e64, etc
    for deg in range(p + 1):
        sl = slice(deg * deg, deg * deg + 2 * deg + 1)
        ref = np.abs(L64[:, sl]).max()
        assert np.abs(Ltc[:, sl] - L64[:, sl]).max() <= 1e-5 * ref, deg
    a64 = np.stack([o64["ax"], o64["ay"], o64["az"]], 1)
    atc = np.stack([otc["ax"], otc["ay"], otc["az"]], 1)
    rel = np.linalg.norm(atc - a64, axis=1) / np.linalg.norm(a64, axis=1)
    assert np.sqrt(np.mean(rel ** 2)) < 3e-7
    j64 = np.stack([o64["jx"], o64["jy"], o64["jz"]], 1)
    jtc = np.stack([otc["jx"], otc["jy"], otc["jz"]], 1)
    relj = np.linalg.norm(jtc - j64, axis=1) / np.linalg.norm(j64, axis=1)
    assert np.sqrt(np.mean(relj ** 2)) < 3e-6


def test_tc_far_field_error_at_fp32_floor():
    n = 1 << 17
    x, y, z, vx, vy, vz, m = ics.plummer_kroupa(n, 7)
    idx = np.random.default_rng(7).choice(n, 256, replace=False)
    d = oracle.direct(x, y, z, m, vx, vy, vz, targets=idx)
    a = np.stack([d["ax"], d["ay"], d["az"]], 1)
    errs = {}
    for prec in (tcb.PREC_FP64, tcb.PREC_MIXED_M2L):
        o, _, _ = run(prec, x, y, z, m, vx, vy, vz, 10)
        g = np.stack([o["ax"][idx], o["ay"][idx], o["az"][idx]], 1)
        errs[prec] = np.sqrt(np.mean((np.linalg.norm(g - a, axis=1) / np.linalg.norm(a, axis=1)) ** 2))
    # p = 10 truncation error (~1e-7) dominates the FP32 rounding
    assert errs[tcb.PREC_MIXED_M2L] <= 1.1 * errs[tcb.PREC_FP64]


def test_bounded_wait_runs_out_and_the_context_recovers():
    """The tensor-core far field waits for its products with a bounded wait.  With the limit set
    to a few clock cycles every wait runs out: the call returns TC_ERR_TIMEOUT (the kernel
    stops issuing, waits with the default limit for the products in flight and frees its tensor
    memory), and the same context then evaluates normally again once the limit is restored."""
    n = 1 << 13
    x, y, z, vx, vy, vz, m = ics.plummer(n, 77)
    ref, _, _ = run(tcb.PREC_MIXED_M2L, x, y, z, m, vx, vy, vz, 8)
    g = tcb.Gravity(p=8, ncrit=64, theta=0.4, variant=tcb.VARIANT_JERKS, precision=tcb.PREC_MIXED_M2L)
    g.set_wait_limit(4)
    with pytest.raises(tcb.TaichiError, match="timed out"):
        g.evaluate(x, y, z, m, vx, vy, vz)
    g.set_wait_limit(0)
    out = g.evaluate(x, y, z, m, vx, vy, vz)
    for k in ("ax", "ay", "az", "pot", "jx", "jy", "jz"):
        np.testing.assert_array_equal(out[k], ref[k], err_msg=k)
    g.close()
