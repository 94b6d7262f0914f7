"""The oracle's restatements of the reference integrator's diagnostics, compensated drift and
split (oracle/tc_oracle.c, oracle/__init__.py) against the reference's own code: the committed
fixture made from it (tests/golden/integ_*, tests/golden/make_golden.py --integ-only) and, when
the reference tree is present, the harness library itself on random inputs."""
import os

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIX = os.path.join(ROOT, "tests", "golden", "integ_plummer_kroupa2k.npz")


def _vec(d):
    return np.array([d["kinetic"], d["potential"], d["mass"], *d["cm_pos"], *d["cm_vel"]])


@pytest.fixture(scope="module")
def fx():
    return dict(np.load(FIX))


def test_diagnostics_match_reference_fixture(fx):
    got = _vec(oracle.system_diagnostics(*[fx[k] for k in ("m", "x", "y", "z", "vx", "vy", "vz", "pot")]))
    # long-double sums in the same order; the per-term FP64 products may differ by one rounding
    # where the reference's build fuses them, so allow a few ulp of the sum
    np.testing.assert_allclose(got, fx["diag"], rtol=4e-16, atol=0)


def test_compensated_drift_is_bit_exact(fx):
    s = [fx["x"], fx["y"], fx["z"]]
    e = [np.zeros_like(fx["x"]) for _ in range(3)]
    v = [fx["vx"], fx["vy"], fx["vz"]]
    for _ in range(3):
        for d in range(3):
            s[d], e[d] = oracle.drift_compsum(s[d], e[d], v[d], float(fx["dt"]))
    for d, a in enumerate("xyz"):
        assert np.array_equal(s[d], fx["drift_" + a])
        assert np.array_equal(e[d], fx["drift_e" + a])


def test_split_order_matches_reference_fixture(fx):
    perm, nf = oracle.split_order(fx["ts"], float(fx["dt"]))
    assert nf == int(fx["split_nfast"])
    assert np.array_equal(perm, fx["split_perm"])


@pytest.mark.parametrize("case", ["ties", "all_fast", "all_slow", "one_fast", "negative_dt"])
def test_split_edge_cases(case):
    rng = np.random.default_rng(5)
    n, dt = 37, 0.25
    ts = {"ties": np.round(rng.random(n) * 4) / 8, "all_fast": np.full(n, 0.1), "all_slow": np.full(n, 0.3),
          "one_fast": np.where(np.arange(n) == 20, 0.1, 0.3), "negative_dt": rng.random(n) * 0.5}[case]
    if case == "negative_dt":
        dt = -dt
    perm, nf = oracle.split_order(ts, dt)
    assert sorted(perm) == list(range(n))
    if case == "one_fast":
        assert nf == 0  # fast.n == 1 is folded into slow (integrator.h:623-627)
    else:
        assert np.all(ts[perm[:nf]] < abs(dt)) and np.all(ts[perm[nf:]] >= abs(dt))
    if oracle.integ_ref_available():
        rp, rnf = oracle.ref_split(ts, dt)
        assert rnf == nf and np.array_equal(rp, perm)


@pytest.mark.skipif(not oracle.integ_ref_available(), reason="reference harness not built")
def test_against_reference_harness_random_inputs():
    rng = np.random.default_rng(9)
    for n in (1, 7, 1000, 50000):
        m = rng.random(n) / n
        x, y, z, vx, vy, vz = rng.standard_normal((6, n))
        pot = rng.random(n)
        a = _vec(oracle.system_diagnostics(m, x, y, z, vx, vy, vz, pot))
        b = _vec(oracle.ref_system_diagnostics(m, x, y, z, vx, vy, vz, pot))
        np.testing.assert_allclose(a, b, rtol=4e-16, atol=1e-300)
        ex = rng.standard_normal(n) * 1e-17
        s, e = oracle.drift_compsum(x, ex, vx, 1.0 / 128)
        r = oracle.ref_drift(x, y, z, ex, ex, ex, vx, vy, vz, 1.0 / 128)
        assert np.array_equal(s, r[0]) and np.array_equal(e, r[3])
    for _ in range(300):
        n = int(rng.integers(2, 80))
        ts = np.round(rng.random(n) * 8) / 8
        dt = float(rng.random())
        p1, f1 = oracle.split_order(ts, dt)
        p2, f2 = oracle.ref_split(ts, dt)
        assert f1 == f2 and np.array_equal(p1, p2)


@pytest.mark.parametrize("gradient", [False, True])
def test_shim_driven_reference_integrators_load(gradient):
    """The reference's integrator compiled over this library through the shim -- its HOLD build
    and its default GRADIENT / OUTPUTACC build (the check of tc_evolve_omelyan) -- loads and
    exports the step entry point (the GPU tests run it)."""
    import ctypes
    path = oracle.integ_shim_path(gradient)
    if not os.path.exists(path):
        pytest.skip("shim-driven reference integrator not built")
    lib = ctypes.CDLL(path)
    assert hasattr(lib, "tcr_evolve_hold")
