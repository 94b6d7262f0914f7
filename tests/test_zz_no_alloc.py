"""The allocation-free direct-sum entry point (tc_evaluate_direct_noalloc).

Some callers cannot allocate device memory (their own allocator owns the GPU memory they
may touch, or their time step must not stall on cudaMalloc's implicit synchronisation).
For them the library keeps its working storage in one fixed static device array.  These
checks call that entry point through the C ABI, twice in a row with different inputs, and
compare each result with the allocating entry point (tc_evaluate on its direct branch) and
with the CPU oracle's FP64 direct sum, also with sink-only, source-only and sink+source
bodies mixed.  This file is collected last on purpose; it must pass alone and after the
other tests."""
import ctypes as C

import numpy as np
import pytest

import taichi_collisional_b200 as tcb
from taichi_collisional_b200 import ics

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _reference_result(arrays, jerk):
    x, y, z, vx, vy, vz, m = arrays
    g = tcb.Gravity(p=8, ncrit=64, theta=0.5, variant=tcb.VARIANT_JERKS if jerk else tcb.VARIANT_TOP,
                    direct_below=1 << 30)
    out = g.evaluate(x, y, z, m, vx, vy, vz) if jerk else g.evaluate(x, y, z, m)
    assert g.stats()["n_cells"] == 0  # the allocating entry point took its direct branch
    g.close()
    return out


def _oracle_result(arrays, jerk, flags=None):
    """FP64 direct sums of the CPU oracle; with flags, only bit-1 bodies act as sources and
    bodies without bit 0 (not sinks) get zeros, as the library defines them."""
    import oracle
    x, y, z, vx, vy, vz, m = arrays
    msrc = m if flags is None else np.where(flags & 2, m, 0.0)
    ref = oracle.direct(x, y, z, msrc, *((vx, vy, vz) if jerk else (None, None, None)))
    if flags is not None:
        for k in ref:
            ref[k] = np.where(flags & 1, ref[k], 0.0)
    return ref


def _noalloc(arrays, jerk, flags=None):
    import torch
    L = tcb.load_library()
    t = [torch.tensor(a, dtype=torch.float64, device="cuda") for a in arrays]
    x, y, z, vx, vy, vz, m = t
    n = len(arrays[0])
    keys = ("ax", "ay", "az", "pot", "jx", "jy", "jz")
    out = {k: torch.full((n,), np.nan, dtype=torch.float64, device="cuda") for k in keys}
    fl = None if flags is None else torch.tensor(flags, dtype=torch.uint8, device="cuda")
    P = lambda a: C.c_void_p(a.data_ptr()) if a is not None else None  # noqa: E731
    rc = L.tc_evaluate_direct_noalloc(n, P(x), P(y), P(z), P(vx) if jerk else None, P(vy) if jerk else None,
                                      P(vz) if jerk else None, P(m), P(fl), P(out["ax"]), P(out["ay"]),
                                      P(out["az"]), P(out["pot"]), P(out["jx"]) if jerk else None,
                                      P(out["jy"]) if jerk else None, P(out["jz"]) if jerk else None,
                                      int(jerk), None)
    assert rc == 0
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


def _compare(got, ref, keys):
    for k in keys:
        scale = np.sqrt(np.mean(ref[k] ** 2))
        assert np.abs(got[k] - ref[k]).max() <= TOL * scale, k


@pytest.mark.parametrize("jerk", [True, False])
def test_noalloc_matches_allocating_entry_point_twice(jerk):
    keys = ("ax", "ay", "az", "pot", "jx", "jy", "jz") if jerk else ("ax", "ay", "az", "pot")
    first = ics.plummer(5000, seed=101)
    second = ics.plummer_kroupa(3000, seed=102)  # smaller: stale entries of call 1 must not leak
    for arrays in (first, second):
        got = _noalloc(arrays, jerk)
        ref = _reference_result(arrays, jerk)
        _compare(got, ref, keys)
        _compare(got, _oracle_result(arrays, jerk), keys)


@pytest.mark.parametrize("jerk", [True, False])
def test_noalloc_sink_and_source_flags_match_the_oracle(jerk):
    """The flags the block-time-step integrator's direct kicks pass: 1 sink only, 2 source
    only, 3 both; two calls in a row with different flag patterns."""
    keys = ("ax", "ay", "az", "pot", "jx", "jy", "jz") if jerk else ("ax", "ay", "az", "pot")
    rng = np.random.default_rng(7)
    for n, seed in ((2000, 201), (700, 202)):
        arrays = ics.plummer_kroupa(n, seed=seed)
        flags = rng.integers(1, 4, n).astype(np.uint8)
        got = _noalloc(arrays, jerk, flags)
        _compare(got, _oracle_result(arrays, jerk, flags), keys)


def test_noalloc_rejects_sizes_above_its_fixed_array():
    L = tcb.load_library()
    n = tcb.NOALLOC_MAX_N + 1
    rc = L.tc_evaluate_direct_noalloc(n, *([C.c_void_p(16)] * 7), None, *([C.c_void_p(16)] * 7), 1, None)
    assert rc == 3  # TC_ERR_CAPACITY, before touching any pointer
