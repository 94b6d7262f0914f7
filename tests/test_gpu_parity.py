"""Device path (through the C ABI) against the reference's outputs and the CPU oracle.

Tolerance: plain FP64 must reproduce the reference FMM within 1e-12 relative per particle
(acceleration, potential, jerk; bodies whose value is below 1e-3 of the rms are measured
against the rms).  Cells and interaction lists must be identical as sets."""
import os

import numpy as np
import pytest

import oracle
import taichi_collisional_b200 as tcb
from taichi_collisional_b200 import ics
from tests._util import cell_keys, pair_set, ref_cell_levels, rel_err, rel_vec_err, vec

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _gravity_for(d, **kw):
    v = int(d["variant"])
    su = None if v == tcb.VARIANT_TOP else d["shift_u"]
    return tcb.Gravity(p=int(d["p"]), ncrit=int(d["ncrit"]), theta=float(d["theta"]), variant=v, shift_u=su,
                       direct_below=0, **kw)


def _check_forces(out, ref, jerk):
    assert rel_vec_err(vec(out, "a"), vec(ref, "a")).max() < TOL
    assert rel_err(out["pot"], ref["pot"]).max() < TOL
    if jerk:
        assert rel_vec_err(vec(out, "j"), vec(ref, "j")).max() < TOL


def test_golden_forces_cells_lists(golden_cases):
    for name, d in golden_cases.items():
        g = _gravity_for(d)
        out = g.evaluate(d["x"], d["y"], d["z"], d["m"], d["vx"], d["vy"], d["vz"])
        _check_forces(out, d, int(d["variant"]) == tcb.VARIANT_JERKS)
        c = g.cells()
        ref_lev = ref_cell_levels(d["cell_nchild"], d["cell_child"])
        rkeys = cell_keys(d["cell_begin"], d["cell_nbody"], ref_lev)
        gkeys = cell_keys(c["begin"], c["nbody"], c["level"])
        assert sorted(rkeys) == sorted(gkeys), name
        ridx = {k: i for i, k in enumerate(rkeys)}
        order = np.array([ridx[k] for k in gkeys])
        scale = np.abs(d["cell_X"]).max()
        assert np.abs(c["X"] - d["cell_X"][order]).max() < 1e-13 * scale, name
        assert np.abs(c["R"] - d["cell_R"][order]).max() < 1e-13 * scale, name
        assert np.array_equal(c["nchild"], d["cell_nchild"][order]), name
        lists = g.lists()
        for k in ("m2l", "p2p"):
            assert pair_set(lists[k][0], lists[k][1], gkeys) == pair_set(d[k + "_t"], d[k + "_s"], rkeys), (name, k)
        # bodies of every cell are the reference's bodies (order inside a leaf may differ)
        perm = c["perm"]
        ref_idx = d["body_index"]
        for ci in np.nonzero(c["nchild"] == 0)[0][:50]:
            b, nb = c["begin"][ci], c["nbody"][ci]
            assert set(perm[b:b + nb].tolist()) == set(ref_idx[b:b + nb].tolist())
        g.close()


def test_device_pointer_path_matches_host_path(golden_cases):
    import torch
    d = golden_cases["jerks_kroupa1500_p10"]
    g = _gravity_for(d)
    host = g.evaluate(d["x"], d["y"], d["z"], d["m"], d["vx"], d["vy"], d["vz"])
    t = {k: torch.tensor(d[k], dtype=torch.float64, device="cuda") for k in ("x", "y", "z", "m", "vx", "vy", "vz")}
    dev = g.evaluate(t["x"], t["y"], t["z"], t["m"], t["vx"], t["vy"], t["vz"])
    for k in host:
        assert np.array_equal(host[k], dev[k].cpu().numpy()), k
    g.close()


CASES = [
    # variant, p, n, seed, ncrit, theta, generator
    (tcb.VARIANT_JERKS, 4, 6000, 31, 64, 0.5, "plummer"),
    (tcb.VARIANT_JERKS, 6, 5000, 32, 32, 0.4, "plummer_kroupa"),
    (tcb.VARIANT_TOP, 8, 8000, 33, 64, 0.5, "plummer"),
    (tcb.VARIANT_JERKS, 10, 6000, 34, 64, 0.4, "plummer_kroupa"),
    (tcb.VARIANT_TOP, 12, 5000, 35, 48, 0.4, "plummer_kroupa"),
    (tcb.VARIANT_JERKS, 12, 7000, 36, 64, 0.4, "plummer_kroupa"),
    (tcb.VARIANT_JERKS, 16, 4000, 37, 64, 0.5, "plummer"),
    (tcb.VARIANT_TOP, 16, 3000, 38, 32, 0.7, "plummer"),
]


@pytest.mark.parametrize("variant,p,n,seed,ncrit,theta,gen", CASES)
def test_random_against_oracle(variant, p, n, seed, ncrit, theta, gen):
    x, y, z, vx, vy, vz, m = getattr(ics, gen)(n, seed)
    su = np.random.default_rng(seed).uniform(size=3) if variant == tcb.VARIANT_JERKS else None
    o = oracle.evaluate(x, y, z, m, vx, vy, vz, p=p, theta=theta, ncrit=ncrit, variant=variant, shift_u=su)
    g = tcb.Gravity(p=p, ncrit=ncrit, theta=theta, variant=variant, shift_u=su, direct_below=0)
    out = g.evaluate(x, y, z, m, vx, vy, vz)
    _check_forces(out, o, variant == tcb.VARIANT_JERKS)
    st = g.stats()
    assert st["n_cells"] == o["stats"]["n_cells"]
    assert st["n_m2l"] == o["stats"]["n_m2l"]
    assert st["n_p2p"] == o["stats"]["n_p2p"]
    g.close()


@pytest.mark.parametrize("variant", [tcb.VARIANT_TOP, tcb.VARIANT_JERKS])
def test_sink_and_source_flags(variant):
    x, y, z, vx, vy, vz, m = ics.plummer(5000, seed=41)
    rng = np.random.default_rng(41)
    flags = rng.integers(0, 4, size=5000).astype(np.uint8)
    o = oracle.evaluate(x, y, z, m, vx, vy, vz, p=8, theta=0.5, ncrit=32, variant=variant, flags=flags)
    g = tcb.Gravity(p=8, ncrit=32, theta=0.5, variant=variant, direct_below=0)
    out = g.evaluate(x, y, z, m, vx, vy, vz, flags=flags)
    sink = (flags & 1) == 1
    assert np.all(out["ax"][~sink] == 0) and np.all(out["pot"][~sink] == 0)
    ref = {k: o[k][sink] for k in o if k != "stats"}
    got = {k: out[k][sink] for k in out}
    _check_forces(got, ref, variant == tcb.VARIANT_JERKS)
    g.close()


@pytest.mark.parametrize("variant", [tcb.VARIANT_TOP, tcb.VARIANT_JERKS])
def test_direct_branch(variant):
    # N below the reference's direct threshold (top: ncrit, jerks: 8000) -> direct sum
    x, y, z, vx, vy, vz, m = ics.plummer(3000, seed=42)
    g = tcb.Gravity(p=8, ncrit=64, theta=0.5, variant=variant, direct_below=-1)
    out = g.evaluate(x, y, z, m, vx, vy, vz)
    if variant == tcb.VARIANT_JERKS:
        d = oracle.direct(x, y, z, m, vx, vy, vz)
        _check_forces(out, d, True)
        assert g.stats()["n_cells"] == 0
    else:
        assert g.stats()["n_cells"] > 0  # 3000 >= ncrit: FMM
    g.close()


def test_tiny_inputs():
    g = tcb.Gravity(p=8, ncrit=64, theta=0.5, variant=tcb.VARIANT_JERKS, direct_below=0)
    one = g.evaluate(np.zeros(1), np.zeros(1), np.zeros(1), np.ones(1), np.zeros(1), np.zeros(1), np.zeros(1))
    assert all(np.all(one[k] == 0) for k in one)
    x = np.array([0.0, 1.0]); z0 = np.zeros(2)
    two = g.evaluate(x, z0, z0, np.array([1.0, 2.0]), z0, np.array([0.0, 1.0]), z0)
    assert abs(two["ax"][0] - 2.0) < 1e-15 and abs(two["ax"][1] + 1.0) < 1e-15
    assert abs(two["pot"][0] - 2.0) < 1e-15 and abs(two["jy"][0] - 2.0) < 1e-15
    g.close()


def test_non_finite_input_is_reported():
    x, y, z, vx, vy, vz, m = ics.plummer(10000, seed=43)
    x[17] = np.nan
    g = tcb.Gravity(p=8, ncrit=64, theta=0.5, variant=tcb.VARIANT_JERKS, direct_below=0)
    with pytest.raises(tcb.TaichiError, match="non-finite"):
        g.evaluate(x, y, z, m, vx, vy, vz)
    x[17] = 0.1  # the context stays usable
    g.evaluate(x, y, z, m, vx, vy, vz)
    g.close()


def test_coincident_bodies_hit_depth_limit():
    # more than ncrit bodies at one point: the reference recursion never ends; here the
    # cell stops at level 21 and the call reports it while still returning direct sums
    x, y, z, vx, vy, vz, m = ics.plummer(9000, seed=44)
    x[:100] = y[:100] = z[:100] = 0.25
    g = tcb.Gravity(p=6, ncrit=64, theta=0.5, variant=tcb.VARIANT_JERKS, direct_below=0)
    with pytest.raises(tcb.TaichiError, match="depth"):
        g.evaluate(x, y, z, m, vx, vy, vz)
    g.close()


def test_runs_are_bitwise_deterministic():
    x, y, z, vx, vy, vz, m = ics.plummer_kroupa(60000, seed=45)
    g = tcb.Gravity(p=10, ncrit=64, theta=0.4, variant=tcb.VARIANT_JERKS)
    a = g.evaluate(x, y, z, m, vx, vy, vz)
    b = g.evaluate(x, y, z, m, vx, vy, vz)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    g.close()


@pytest.mark.parametrize("variant", [tcb.VARIANT_TOP, tcb.VARIANT_JERKS])
def test_context_reused_at_growing_n(variant):
    """One context evaluating ever larger inputs (its cell, list and frontier capacities were
    sized by the smaller calls) gives the same results, bit for bit, as a fresh context."""
    g = tcb.Gravity(p=8, ncrit=64, theta=0.4, variant=variant, direct_below=0)
    for n in (130, 2000, 8000, 32768, 100000):
        x, y, z, vx, vy, vz, m = ics.plummer_kroupa(n, seed=50 + n % 7)
        a = g.evaluate(x, y, z, m, vx, vy, vz)
        f = tcb.Gravity(p=8, ncrit=64, theta=0.4, variant=variant, direct_below=0)
        b = f.evaluate(x, y, z, m, vx, vy, vz)
        f.close()
        for k in a:
            assert np.array_equal(a[k], b[k]), (n, k)
    g.close()


def test_large_n_against_direct_sum():
    n = 1 << 20
    x, y, z, vx, vy, vz, m = ics.plummer(n, seed=46)
    g = tcb.Gravity(p=10, ncrit=64, theta=0.4, variant=tcb.VARIANT_JERKS)
    out = g.evaluate(x, y, z, m, vx, vy, vz)
    idx = np.random.default_rng(46).choice(n, 512, replace=False)
    d = oracle.direct(x, y, z, m, vx, vy, vz, targets=idx)
    ea = rel_vec_err(vec({k: out[k][idx] for k in out}, "a"), vec(d, "a"))
    ej = rel_vec_err(vec({k: out[k][idx] for k in out}, "j"), vec(d, "j"))
    assert np.sqrt((ea ** 2).mean()) < 5e-7
    assert np.sqrt((ej ** 2).mean()) < 5e-5
    st = g.stats()
    assert 30e6 < st["n_m2l"] < 40e6  # ~34.4 M at N = 2^20, theta = 0.4, ncrit = 64
    g.close()


@pytest.mark.parametrize("device", [False, True])
def test_direct_sums_match_oracle(device):
    # tc_direct_sums (the accuracy probe of bench.py) against the oracle's FP64 direct sum,
    # with jerks, from host arrays and from device tensors
    n = 20000
    x, y, z, vx, vy, vz, m = ics.plummer_kroupa(n, 5)
    idx = np.random.default_rng(5).choice(n, 300, replace=False)
    ref = oracle.direct(x, y, z, m, vx, vy, vz, targets=idx)
    g = tcb.Gravity(p=8, ncrit=64, theta=0.5, variant=tcb.VARIANT_JERKS)
    args = (x, y, z, m)
    vel = (vx, vy, vz)
    if device:
        import torch
        args = tuple(torch.tensor(a, device="cuda") for a in args)
        vel = tuple(torch.tensor(a, device="cuda") for a in vel)
    got = g.direct_sums(*args, idx, *vel)
    g.close()
    assert rel_err(got["pot"], ref["pot"]).max() < 1e-12
    assert rel_vec_err(vec(got, "a"), vec(ref, "a")).max() < 1e-12
    assert rel_vec_err(vec(got, "j"), vec(ref, "j")).max() < 1e-11


@pytest.mark.parametrize("name", ["steps_top_kroupa2k_p8", "steps_top_plummer40_p8"])
@pytest.mark.parametrize("device", [False, True])
def test_time_step_pass_matches_reference(name, device):
    # get_force_and_potential(bodies, true) of the top-level tree: near-field pot / acc and
    # each body's sum of 1 / tau^4, against the reference's own output (tests/golden)
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    g = tcb.Gravity(p=int(d["p"]), ncrit=int(d["ncrit"]), theta=float(d["theta"]), variant=tcb.VARIANT_TOP)
    args = [d[k] for k in ("x", "y", "z", "m", "vx", "vy", "vz")]
    fl = d["flags"]
    if device:
        import torch
        args = [torch.tensor(a, device="cuda") for a in args]
        fl = torch.tensor(fl, device="cuda")
    out = g.evaluate_steps(*args, float(d["dt_param"]), flags=fl)
    if device:
        out = {k: v.cpu().numpy() for k, v in out.items()}
    st = g.stats()
    g.close()
    assert st["n_m2l"] > 0 or st["n_cells"] == 1
    ts = d["timestep"]
    sink = (d["flags"] & 1) > 0
    assert np.all(out["timestep"][~sink] == 0)
    assert np.all(np.abs(out["timestep"][sink] - ts[sink]) <= 1e-12 * ts[sink])
    for k in ("ax", "ay", "az", "pot"):
        assert np.abs(out[k] - d[k]).max() <= 1e-12 * np.abs(d[k]).max()


def test_time_step_pass_is_top_tree_only():
    x, y, z, vx, vy, vz, m = ics.plummer(256, 3)
    g = tcb.Gravity(p=8, ncrit=32, theta=0.5, variant=tcb.VARIANT_JERKS)
    with pytest.raises(tcb.TaichiError):
        g.evaluate_steps(x, y, z, m, vx, vy, vz, 0.025)
    g.close()


def test_error_mac_matches_reference():
    """The top tree's own get_force_and_potential (integrator.h:459-562): the low-order
    pre-pass's acc_old, the error-controlled MAC's lists, the forces -- against the reference
    run by tests/golden/make_golden.py (emac_* fixtures)."""
    import glob
    files = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "emac_top_*.npz")))
    assert files
    for f in files:
        d = dict(np.load(f))
        name = os.path.basename(f)
        g = tcb.Gravity(p=int(d["p"]), ncrit=int(d["ncrit"]), theta=0.4, variant=tcb.VARIANT_TOP,
                        precision=tcb.PREC_FP64)
        g.set_error_mac(True, float(d["force_accuracy"]))
        out = g.evaluate(d["x"], d["y"], d["z"], d["m"])
        acc_old = g.acc_old()
        assert np.max(np.abs(acc_old - d["acc_old"]) / np.abs(d["acc_old"])) < 1e-12, name
        c = g.cells()
        ref_lev = ref_cell_levels(d["cell_nchild"], d["cell_child"])
        rkeys = cell_keys(d["cell_begin"], d["cell_nbody"], ref_lev)
        gkeys = cell_keys(c["begin"], c["nbody"], c["level"])
        assert sorted(rkeys) == sorted(gkeys), name
        lists = g.lists()
        for k in ("m2l", "p2p"):
            assert pair_set(lists[k][0], lists[k][1], gkeys) == pair_set(d[k + "_t"], d[k + "_s"], rkeys), (name, k)
        assert rel_err(out["pot"], d["pot"]).max() < 1e-12, name
        assert rel_vec_err(vec(out, "a"), vec(d, "a")).max() < 1e-12, name
        g.close()


def test_error_mac_time_step_pass_matches_reference():
    """get_force_and_potential(bodies, true) of the top tree: pre-pass, error-controlled MAC,
    time-step pass with a sink / source subset, against the reference's own run."""
    d = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "emac_steps_top_kroupa2k_p8.npz")))
    g = tcb.Gravity(p=int(d["p"]), ncrit=int(d["ncrit"]), theta=0.4, variant=tcb.VARIANT_TOP,
                    precision=tcb.PREC_FP64)
    g.set_error_mac(True, float(d["force_accuracy"]))
    out = g.evaluate_steps(d["x"], d["y"], d["z"], d["m"], d["vx"], d["vy"], d["vz"], float(d["dt_param"]),
                           flags=d["flags"])
    sink = (d["flags"] & 1) != 0
    assert np.all(np.abs(out["timestep"][sink] - d["timestep"][sink]) <= 1e-12 * d["timestep"][sink])
    for k in ("pot", "ax", "ay", "az"):
        assert np.abs(out[k][sink] - d[k][sink]).max() <= 1e-12 * np.abs(d[k]).max(), k
    acc_old = g.acc_old()
    assert np.max(np.abs(acc_old - d["acc_old"]) / np.abs(d["acc_old"])) < 1e-12
    g.close()


def test_jerks_error_mac_matches_reference():
    """The jerks tree's own get_force_and_potential (taichi_with_jerks/integrator.h:308-432):
    the order-2 pre-pass with its FP32 vector near field (acc_old = |F|), the one-sided error
    MAC of taichi_with_jerks/traverse_eager.h:59-122 (lists identical), and the forces and jerks
    within 1e-12 -- against the reference run by tests/golden/make_golden.py (emac_jerks_*)."""
    import glob
    files = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "emac_jerks_*.npz")))
    assert files
    for f in files:
        d = dict(np.load(f))
        name = os.path.basename(f)
        g = tcb.Gravity(p=int(d["p"]), ncrit=int(d["ncrit"]), theta=0.4, variant=tcb.VARIANT_JERKS,
                        precision=tcb.PREC_FP64, shift_u=d["shift_u"], direct_below=0)
        g.set_error_mac(True, float(d["force_accuracy"]))
        out = g.evaluate(d["x"], d["y"], d["z"], d["m"], d["vx"], d["vy"], d["vz"])
        acc_old = g.acc_old()
        # FP32 sums in the reference's operation order; FP64 sums over source cells in another order
        assert np.max(np.abs(acc_old - d["acc_old"]) / np.abs(d["acc_old"])) < 1e-9, name
        c = g.cells()
        ref_lev = ref_cell_levels(d["cell_nchild"], d["cell_child"])
        rkeys = cell_keys(d["cell_begin"], d["cell_nbody"], ref_lev)
        gkeys = cell_keys(c["begin"], c["nbody"], c["level"])
        assert sorted(rkeys) == sorted(gkeys), name
        lists = g.lists()
        for k in ("m2l", "p2p"):
            assert pair_set(lists[k][0], lists[k][1], gkeys) == pair_set(d[k + "_t"], d[k + "_s"], rkeys), (name, k)
        _check_forces(out, d, True)
        g.close()


@pytest.mark.parametrize("variant", [tcb.VARIANT_TOP, tcb.VARIANT_JERKS])
def test_softened_near_field_and_direct_sums(variant):
    """Plummer softening (tc_params.softening, no counterpart in the reference): the direct-sum
    branch and tc_direct_sums equal a numpy FP64 softened direct sum; the FMM's near field is
    softened and its far field stays Newtonian (O(eps^2 / r^2) at far-field separations), so
    the FMM stays within its own truncation error of the softened direct sum."""
    n, eps = 3000, 1e-3
    x, y, z, vx, vy, vz, m = ics.plummer(n, 17)
    X = np.stack([x, y, z], 1)
    d = X[None, :, :] - X[:, None, :]
    r2 = (d ** 2).sum(-1)
    s2 = r2 + eps * eps
    inv = np.where(r2 > 0, 1.0 / np.sqrt(s2), 0.0)
    pot = (m[None, :] * inv).sum(1)
    acc = (m[None, :, None] * d * (inv ** 3)[:, :, None]).sum(1)
    jerk = variant == tcb.VARIANT_JERKS
    vel = (vx, vy, vz) if jerk else (None, None, None)
    g = tcb.Gravity(p=10, ncrit=32, theta=0.4, variant=variant, direct_below=1 << 30, softening=eps)
    out = g.evaluate(x, y, z, m, *vel)
    assert rel_err(out["pot"], pot).max() < 1e-12
    assert rel_vec_err(vec(out, "a"), acc).max() < 1e-12
    ds = g.direct_sums(x, y, z, m, np.arange(0, n, 7), *vel)
    assert np.abs(ds["pot"] - pot[::7]).max() < 1e-12 * np.abs(pot).max()
    g.close()
    for prec in (tcb.PREC_FP64, tcb.PREC_MIXED):
        g = tcb.Gravity(p=10, ncrit=32, theta=0.4, variant=variant, direct_below=0, precision=prec, softening=eps)
        out = g.evaluate(x, y, z, m, *vel)
        e = rel_vec_err(vec(out, "a"), acc)
        assert np.sqrt(np.mean(e ** 2)) < 2e-5, prec
        g0 = tcb.Gravity(p=10, ncrit=32, theta=0.4, variant=variant, direct_below=0, precision=prec)
        out0 = g0.evaluate(x, y, z, m, *vel)
        assert rel_vec_err(vec(out0, "a"), acc).max() > 1e-6  # softening changed the near field
        g.close()
        g0.close()


def test_small_plain_case_against_the_live_reference():
    """The small plain-method configuration -- 16,384 equal-mass Plummer bodies, the top tree,
    p = 8, theta = 0.5, ncrit = 64 -- against the reference's own FMM run here (oracle/_ref,
    compiled from its sources), per particle within 1e-12, and against FP64 direct sums."""
    if not oracle.ref_available(oracle.VARIANT_TOP, 8):
        pytest.skip("the reference build (oracle/_ref) is not present")
    n = 16384
    x, y, z, vx, vy, vz, m = ics.plummer(n, 2029)
    ref = oracle.ref_evaluate(x, y, z, m, p=8, theta=0.5, ncrit=64, variant=oracle.VARIANT_TOP,
                              nthreads=os.cpu_count() or 1)
    g = tcb.Gravity(p=8, ncrit=64, theta=0.5, variant=tcb.VARIANT_TOP, direct_below=0)
    out = g.evaluate(x, y, z, m)
    g.close()
    assert rel_vec_err(vec(out, "a"), vec(ref, "a")).max() < TOL
    assert rel_err(out["pot"], ref["pot"]).max() < TOL
    idx = np.random.default_rng(5).choice(n, 512, replace=False)
    d = oracle.direct(x, y, z, m, targets=idx)
    e = rel_vec_err(vec({k: out[k][idx] for k in ("ax", "ay", "az")}, "a"), vec(d, "a"))
    assert np.sqrt(np.mean(e ** 2)) < 1e-3  # the FMM's own truncation error at p = 8, theta = 0.5
