"""The CPU oracle (oracle/tc_oracle.c) pinned against the reference's own outputs:
the golden fixtures (tests/golden/make_golden.py, generated by the reference's headers
compiled behind oracle/ref_harness.cpp) and, when oracle/_ref is built, fresh runs of the
reference on new inputs."""
import math
import os

import numpy as np
import pytest

import oracle
from taichi_collisional_b200 import ics
from tests._util import cell_keys, pair_set, ref_cell_levels, rel_err, rel_vec_err, vec

TOL = 1e-12


def _run_oracle(d):
    v = int(d["variant"])
    su = None if v == oracle.VARIANT_TOP else d["shift_u"]
    return oracle.evaluate(d["x"], d["y"], d["z"], d["m"], d["vx"], d["vy"], d["vz"], p=int(d["p"]),
                           theta=float(d["theta"]), ncrit=int(d["ncrit"]), variant=v, shift_u=su)


def test_golden_forces(golden_cases):
    assert len(golden_cases) >= 4
    for name, d in golden_cases.items():
        o = _run_oracle(d)
        assert rel_vec_err(vec(o, "a"), vec(d, "a")).max() < TOL, name
        assert rel_err(o["pot"], d["pot"]).max() < TOL, name
        if int(d["variant"]) == oracle.VARIANT_JERKS:
            assert rel_vec_err(vec(o, "j"), vec(d, "j")).max() < TOL, name


def test_golden_cells_and_lists(golden_cases):
    for name, d in golden_cases.items():
        _run_oracle(d)
        c = oracle.last_cells()
        # the oracle keeps the reference's depth-first cell order: compare entry by entry
        assert np.array_equal(c["begin"], d["cell_begin"]), name
        assert np.array_equal(c["nbody"], d["cell_nbody"]), name
        assert np.array_equal(c["nchild"], d["cell_nchild"]), name
        assert np.array_equal(np.where(c["nchild"] > 0, c["child"], -1), np.where(d["cell_nchild"] > 0, d["cell_child"], -1)), name
        scale = np.abs(d["cell_X"]).max()
        assert np.abs(c["X"] - d["cell_X"]).max() < 1e-13 * scale, name
        assert np.abs(c["R"] - d["cell_R"]).max() < 1e-13 * scale, name
        L = oracle.last_lists()
        lev = ref_cell_levels(d["cell_nchild"], d["cell_child"])
        keys = cell_keys(d["cell_begin"], d["cell_nbody"], lev)
        for k in ("m2l", "p2p"):
            assert pair_set(L[k][0], L[k][1], keys) == pair_set(d[k + "_t"], d[k + "_s"], keys), (name, k)


def test_reference_lists_are_symmetric(golden_cases):
    # the one-sided M2L of the device path equals the reference's mutual M2L
    # (kernel_fast_lean.h:1036) only because every visited pair is visited both ways
    for name, d in golden_cases.items():
        for k in ("m2l", "p2p"):
            s = set(zip(d[k + "_t"].tolist(), d[k + "_s"].tolist()))
            assert all((b, a) in s for a, b in s), (name, k)
            assert len(s) == len(d[k + "_t"])


def test_known_answer_single_source():
    """taichi_with_jerks/test.cxx:25-175 geometry: one unit mass at the origin moving with
    v = (10,10,10); target at (120,100,300) moving with v = (1,2,3).  P2M -> M2M -> M2L
    (rotation and textbook O(p^4) forms) -> L2P against the exact point-mass answer."""
    L = oracle.lib()
    p = 12
    L.tco_init(p)
    nt = (p + 1) ** 2
    dp = oracle._dp
    one = np.ones(1)
    zero = np.zeros(1)
    vel = np.full(1, 10.0)
    Cj = np.zeros(3)
    M = np.zeros(nt)
    Md = np.zeros(nt)
    L.tco_p2m(p, 1, zero.ctypes.data_as(dp), zero.ctypes.data_as(dp), zero.ctypes.data_as(dp),
              vel.ctypes.data_as(dp), vel.ctypes.data_as(dp), vel.ctypes.data_as(dp), one.ctypes.data_as(dp),
              Cj.ctypes.data_as(dp), M.ctypes.data_as(dp), Md.ctypes.data_as(dp))
    CJ = np.array([1.0, 1.0, 2.0])
    M2 = np.zeros(nt)
    Md2 = np.zeros(nt)
    dX = Cj - CJ
    L.tco_m2m(p, M.ctypes.data_as(dp), Md.ctypes.data_as(dp), dX.ctypes.data_as(dp), M2.ctypes.data_as(dp),
              Md2.ctypes.data_as(dp))
    Ci = np.array([120.0, 100.0, 300.0])
    Lr = np.zeros(nt)
    Ldr = np.zeros(nt)
    Lo = np.zeros(nt)
    d2 = Ci - CJ
    L.tco_m2l_rotate(p, M2.ctypes.data_as(dp), Md2.ctypes.data_as(dp), d2.ctypes.data_as(dp),
                     Lr.ctypes.data_as(dp), Ldr.ctypes.data_as(dp))
    L.tco_m2l_direct(p, M2.ctypes.data_as(dp), d2.ctypes.data_as(dp), Lo.ctypes.data_as(dp))
    # the reference's rotation drops the (p, +-p) multipole terms from L[0] (factorial_table[2p] == 0)
    assert np.abs(Lr[1:] - Lo[1:]).max() < 1e-12 * np.abs(Lo).max()
    out = np.zeros(7)
    dB = Ci - Ci
    v = np.array([1.0, 2.0, 3.0])
    L.tco_l2p(p, Lr.ctypes.data_as(dp), Ldr.ctypes.data_as(dp), dB.ctypes.data_as(dp), v.ctypes.data_as(dp),
              out.ctypes.data_as(dp))
    r = Ci
    rn = math.sqrt((r * r).sum())
    pot = 1 / rn
    acc = -r / rn ** 3
    dv = np.array([10.0, 10.0, 10.0]) - v
    jerk = dv / rn ** 3 - 3 * np.dot(-r, dv) * (-r) / rn ** 5
    assert abs(out[0] - pot) < 1e-12 * pot
    assert np.abs(out[1:4] - acc).max() < 1e-10 * np.abs(acc).max()
    assert np.abs(out[4:7] - jerk).max() < 1e-8 * np.abs(jerk).max()


@pytest.mark.parametrize("p", [3, 6, 10, 16])
def test_m2l_rotation_equals_textbook(p):
    L = oracle.lib()
    L.tco_init(p)
    rng = np.random.default_rng(p)
    nt = (p + 1) ** 2
    dp = oracle._dp
    for _ in range(5):
        pts = rng.normal(size=(20, 3)) * 0.3
        m = rng.uniform(0.5, 1.0, size=20)
        C = np.zeros(3)
        M = np.zeros(nt)
        xs, ys, zs = (np.ascontiguousarray(pts[:, k]) for k in range(3))
        L.tco_p2m(p, 20, xs.ctypes.data_as(dp), ys.ctypes.data_as(dp), zs.ctypes.data_as(dp), None, None, None,
                  m.ctypes.data_as(dp), C.ctypes.data_as(dp), M.ctypes.data_as(dp), None)
        d = rng.normal(size=3)
        d *= 4.0 / np.linalg.norm(d)
        Lr, Lo = np.zeros(nt), np.zeros(nt)
        L.tco_m2l_rotate(p, M.ctypes.data_as(dp), None, d.ctypes.data_as(dp), Lr.ctypes.data_as(dp), None)
        L.tco_m2l_direct(p, M.ctypes.data_as(dp), d.ctypes.data_as(dp), Lo.ctypes.data_as(dp))
        assert np.abs(Lr[1:] - Lo[1:]).max() < 1e-12 * np.abs(Lo).max()


def test_miniball_known_cases():
    L = oracle.lib()
    dp = oracle._dp
    pts = np.array([[1.0, 0, 0], [-1, 0, 0], [0, 0.5, 0], [0, 0, 0.2]])
    c, r2 = np.zeros(3), np.zeros(1)
    L.tco_miniball(4, pts.ctypes.data_as(dp), c.ctypes.data_as(dp), r2.ctypes.data_as(dp))
    assert np.allclose(c, 0, atol=1e-15) and abs(r2[0] - 1) < 1e-15
    rng = np.random.default_rng(1)
    pts = rng.normal(size=(500, 3))
    L.tco_miniball(500, pts.ctypes.data_as(dp), c.ctypes.data_as(dp), r2.ctypes.data_as(dp))
    d2 = ((pts - c) ** 2).sum(1)
    assert d2.max() <= r2[0] * (1 + 1e-12)
    assert (d2 >= r2[0] * (1 - 1e-12)).sum() >= 2  # supported by boundary points


def test_direct_sum_small():
    x, y, z, vx, vy, vz, m = ics.plummer(64, seed=5)
    d = oracle.direct(x, y, z, m, vx, vy, vz)
    ax = np.zeros(64)
    for i in range(64):
        dx = x - x[i]
        r = np.sqrt(dx ** 2 + (y - y[i]) ** 2 + (z - z[i]) ** 2)
        r[i] = np.inf
        ax[i] = (m * dx / r ** 3).sum()
    assert np.abs(d["ax"] - ax).max() < 1e-12 * np.abs(ax).max()


@pytest.mark.skipif(not (oracle.ref_available(oracle.VARIANT_JERKS, 8) and oracle.ref_available(oracle.VARIANT_TOP, 10)),
                    reason="oracle/_ref not built")
@pytest.mark.parametrize("variant,p,n,seed,ncrit,theta", [
    (oracle.VARIANT_JERKS, 8, 3000, 21, 32, 0.5),
    (oracle.VARIANT_TOP, 10, 2500, 22, 40, 0.4),
    (oracle.VARIANT_JERKS, 12, 2000, 23, 64, 0.6),
])
def test_oracle_against_reference_build(variant, p, n, seed, ncrit, theta):
    if not oracle.ref_available(variant, p):
        pytest.skip("no reference build for p=%d" % p)
    x, y, z, vx, vy, vz, m = ics.plummer_kroupa(n, seed)
    r = oracle.ref_evaluate(x, y, z, m, vx, vy, vz, p=p, theta=theta, ncrit=ncrit, variant=variant, seed=seed)
    su = oracle.ref_shift_uniforms(variant, p, seed) if variant == oracle.VARIANT_JERKS else None
    o = oracle.evaluate(x, y, z, m, vx, vy, vz, p=p, theta=theta, ncrit=ncrit, variant=variant, shift_u=su)
    assert rel_vec_err(vec(o, "a"), vec(r, "a")).max() < TOL
    assert rel_err(o["pot"], r["pot"]).max() < TOL
    if variant == oracle.VARIANT_JERKS:
        assert rel_vec_err(vec(o, "j"), vec(r, "j")).max() < TOL
    assert o["stats"]["n_cells"] == r["ncell"]


@pytest.mark.parametrize("name", ["steps_top_kroupa2k_p8", "steps_top_plummer40_p8"])
def test_oracle_time_step_pass_matches_reference(name):
    # get_steps = true on the top-level tree: near-field pot / acc and the accumulated
    # 1 / tau^4 of kernel_fast_lean.h:462-548, against the reference's own output
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    o = oracle.evaluate_steps(d["x"], d["y"], d["z"], d["m"], d["vx"], d["vy"], d["vz"], p=int(d["p"]),
                              theta=float(d["theta"]), ncrit=int(d["ncrit"]), dt_param=float(d["dt_param"]),
                              flags=d["flags"])
    sink = (d["flags"] & 1) > 0
    ts = d["timestep"]
    assert np.all(ts[sink] > 0) and np.all(ts[~sink] == 0)
    assert np.abs(o["timestep"] - ts).max() <= 1e-13 * np.abs(ts).max()
    assert np.all(np.abs(o["timestep"][sink] - ts[sink]) <= 1e-13 * ts[sink])
    for k in ("ax", "ay", "az", "pot"):
        assert np.abs(o[k] - d[k]).max() <= 1e-13 * np.abs(d[k]).max()
