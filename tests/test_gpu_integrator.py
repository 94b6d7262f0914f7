"""The integrator around the force evaluation on the GPU: system diagnostics
(tc_system_diagnostics), the compensated drift (tc_drift_compensated), the split by time step
(tc_split_order) and one step of the block-time-step scheme (tc_evolve_hold_dkd), each against
the reference's own integrator.h -- through the committed fixtures made from it
(tests/golden/integ_*, evolve_*) and, where the harness library was built, the reference's
integrator driving this library's force evaluation through the C++ shim."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def _cuda(a, dtype=torch.float64):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _gravity(**kw):
    import taichi_collisional_b200 as t
    return t.Gravity(variant=t.VARIANT_TOP, precision=t.PREC_FP64, **kw)


def _vec(d):
    return np.array([d["kinetic"], d["potential"], d["mass"], *d["cm_pos"], *d["cm_vel"]])


@pytest.fixture(scope="module")
def integ():
    return dict(np.load(os.path.join(GOLD, "integ_plummer_kroupa2k.npz")))


def test_diagnostics_match_reference_fixture(integ):
    g = _gravity(p=8, ncrit=64, theta=0.5)
    got = _vec(g.system_diagnostics(*[_cuda(integ[k]) for k in ("m", "x", "y", "z", "vx", "vy", "vz", "pot")]))
    # the reference sums in long double, these sums in double-double: a few ulp apart at most
    np.testing.assert_allclose(got[:3], integ["diag"][:3], rtol=4e-16, atol=0)
    # the centre of mass of these centred bodies cancels to ~1e-17: compare against the size of
    # the terms (the long-double sums carry ~1e-20 of that)
    m = integ["m"]
    scale = np.array([np.abs(m * integ[k]).sum() for k in ("x", "y", "z", "vx", "vy", "vz")]) / m.sum()
    assert np.all(np.abs(got[3:] - integ["diag"][3:]) <= 1e-17 * scale)
    g.close()


def test_diagnostics_large_n_and_reproducible():
    from taichi_collisional_b200 import ics
    n = 1 << 21
    x, y, z, vx, vy, vz, m = ics.plummer_kroupa(n, 17)
    pot = np.random.default_rng(3).random(n) * 2.0
    g = _gravity(p=8, ncrit=64, theta=0.5)
    args = [_cuda(a) for a in (m, x, y, z, vx, vy, vz, pot)]
    a = _vec(g.system_diagnostics(*args))
    b = _vec(g.system_diagnostics(*args))
    assert np.array_equal(a, b)  # fixed reduction order
    ref = _vec(oracle.system_diagnostics(m, x, y, z, vx, vy, vz, pot))
    np.testing.assert_allclose(a[:3], ref[:3], rtol=1e-15)
    scale = np.array([np.abs(m * x).sum(), np.abs(m * y).sum(), np.abs(m * z).sum(), np.abs(m * vx).sum(),
                      np.abs(m * vy).sum(), np.abs(m * vz).sum()]) / m.sum()
    assert np.all(np.abs(a[3:] - ref[3:]) <= 1e-15 * scale)
    g.close()


def test_compensated_drift_bit_exact(integ):
    g = _gravity(p=8, ncrit=64, theta=0.5)
    s = [_cuda(integ[k]) for k in ("x", "y", "z")]
    e = [torch.zeros_like(s[0]) for _ in range(3)]
    v = [_cuda(integ[k]) for k in ("vx", "vy", "vz")]
    for _ in range(3):
        g.drift_compensated(*s, *e, *v, float(integ["dt"]))
    torch.cuda.synchronize()
    for d, a in enumerate("xyz"):
        assert np.array_equal(s[d].cpu().numpy(), integ["drift_" + a])
        assert np.array_equal(e[d].cpu().numpy(), integ["drift_e" + a])
    g.close()


def test_split_order_matches_reference(integ):
    g = _gravity(p=8, ncrit=64, theta=0.5)
    perm, nf = g.split_order(_cuda(integ["ts"]), float(integ["dt"]))
    assert nf == int(integ["split_nfast"])
    assert np.array_equal(perm.cpu().numpy(), integ["split_perm"])
    # large n with ties, and the one-fast-body rule, against the oracle's restatement
    rng = np.random.default_rng(8)
    for n, ts, dt in ((3_000_000, 2.0 ** -rng.integers(3, 10, 3_000_000), 1.0 / 64),
                      (5000, np.where(np.arange(5000) == 4321, 0.1, 0.3), 0.25),
                      (4097, rng.random(4097), -0.5), (1, np.array([0.1]), 0.25)):
        perm, nf = g.split_order(_cuda(ts), dt)
        p_ref, nf_ref = oracle.split_order(ts, dt)
        assert nf == nf_ref
        assert np.array_equal(perm.cpu().numpy(), p_ref)
    g.close()


def _evolve_state(gen, n, seed):
    from taichi_collisional_b200 import ics
    x, y, z, vx, vy, vz, m = getattr(ics, gen)(n, seed)
    zero = np.zeros(n)
    return dict(x=x, y=y, z=z, vx=vx, vy=vy, vz=vz, m=m, ex=zero, ey=zero, ez=zero, timestep=zero, pot=zero,
                id=np.arange(n, dtype=np.int32))


def _run_device(st0, *, p, ncrit, theta, fa, dtp, dt, gradient=False):
    import taichi_collisional_b200 as t
    g = _gravity(p=p, ncrit=ncrit, theta=theta)
    g.set_error_mac(True, fa)
    dev = {k: _cuda(st0[k]) for k in t.EVOLVE_KEYS}
    dev["id"] = _cuda(st0["id"], torch.int32)
    stats = (g.evolve_omelyan if gradient else g.evolve_hold_dkd)(dev, dtp, dt)
    out = {k: v.cpu().numpy() for k, v in dev.items()}
    g.close()
    return out, stats


@pytest.fixture(scope="module")
def evolve_case():
    f = dict(np.load(os.path.join(GOLD, "evolve_hold_plummer_kroupa1k.npz")))
    st0 = _evolve_state(str(f["gen"]), int(f["n"]), int(f["seed"]))
    kw = dict(p=8, ncrit=int(f["ncrit"]), theta=float(f["theta"]), fa=float(f["force_accuracy"]),
              dtp=float(f["dt_param"]), dt=float(f["dt"]))
    out, stats = _run_device(st0, **kw)
    return f, st0, kw, out, stats


@pytest.mark.skipif(not os.path.exists(oracle.integ_shim_path()), reason="shim-driven reference integrator not built")
def test_evolve_matches_reference_integrator_over_the_same_forces(evolve_case):
    """The reference's own do_evolve / evolve_split_hold_dkd, compiled against this library
    through the shim, sees the same force evaluation; the device-resident scheme must make the
    same splits, kicks and drifts: the same final order and the same state up to the rounding of
    the direct kicks of small systems (host loop vs device kernel)."""
    f, st0, kw, out, stats = evolve_case
    ref, simtime = oracle.ref_evolve_hold(st0, ncrit=kw["ncrit"], theta=kw["theta"], force_accuracy=kw["fa"],
                                          dt_param=kw["dtp"], dt=kw["dt"], shim=True)
    assert simtime == stats["simtime"]
    assert np.array_equal(out["id"], ref["id"])
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        np.testing.assert_allclose(out[k], ref[k], rtol=1e-12, atol=1e-14, err_msg=k)
    for k in ("timestep", "pot"):
        np.testing.assert_allclose(out[k], ref[k], rtol=1e-10, atol=0, err_msg=k)


def test_evolve_close_to_reference_fixture(evolve_case):
    """Against the reference's integrator with its own force evaluation (CPU FMM, whose error-MAC
    pre-pass carries acc_old between calls): the same step within the force error."""
    f, st0, kw, out, stats = evolve_case
    assert float(f["simtime"]) == stats["simtime"]
    o_dev = np.argsort(out["id"])
    o_ref = np.argsort(f["out_id"])
    disp = np.sqrt(sum((f["out_" + k][o_ref] - st0[k]) ** 2 for k in "xyz"))
    err = np.sqrt(sum((out[k][o_dev] - f["out_" + k][o_ref]) ** 2 for k in "xyz"))
    dv = np.sqrt(sum((f["out_" + k][o_ref] - st0[k]) ** 2 for k in ("vx", "vy", "vz")))
    verr = np.sqrt(sum((out[k][o_dev] - f["out_" + k][o_ref]) ** 2 for k in ("vx", "vy", "vz")))
    same_rung = np.mean(np.floor(np.log2(out["timestep"][o_dev])) == np.floor(np.log2(f["out_timestep"][o_ref])))
    print("evolve vs reference: max |dx| / max disp %.3e, median %.3e; max |dv| / max dv %.3e; same rung %.4f"
          % (err.max() / disp.max(), np.median(err / disp), verr.max() / dv.max(), same_rung))
    assert same_rung > 0.99
    assert np.median(err / disp) < 1e-6
    assert err.max() / disp.max() < 1e-3
    assert verr.max() / dv.max() < 1e-3
    assert stats["n_evaluations"] > 0 and stats["max_level"] >= 1


@pytest.mark.skipif(not os.path.exists(oracle.integ_shim_path(True)),
                    reason="shim-driven reference integrator (GRADIENT build) not built")
def test_gradient_scheme_matches_reference_integrator_over_the_same_forces():
    """The reference's default scheme, evolve_split_omelyan of its GRADIENT / OUTPUTACC build,
    compiled against this library through the shim, against tc_evolve_omelyan on the same 1,024
    bodies and step: the same splits (every body gets its system's least time step), the same
    dt / 6 kicks, drifts and force-gradient kicks at the shifted positions -- the same final order,
    time and state up to rounding."""
    f = dict(np.load(os.path.join(GOLD, "evolve_hold_plummer_kroupa1k.npz")))
    st0 = _evolve_state(str(f["gen"]), int(f["n"]), int(f["seed"]))
    kw = dict(p=8, ncrit=int(f["ncrit"]), theta=float(f["theta"]), fa=float(f["force_accuracy"]),
              dtp=float(f["dt_param"]), dt=float(f["dt"]))
    out, stats = _run_device(st0, gradient=True, **kw)
    ref, simtime = oracle.ref_evolve_gradient(st0, ncrit=kw["ncrit"], theta=kw["theta"], force_accuracy=kw["fa"],
                                              dt_param=kw["dtp"], dt=kw["dt"])
    assert simtime == stats["simtime"]
    assert np.array_equal(out["id"], ref["id"])
    assert np.unique(out["timestep"]).size == 1  # the GRADIENT build's shared least time step
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        np.testing.assert_allclose(out[k], ref[k], rtol=1e-12, atol=1e-14, err_msg=k)
    for k in ("timestep", "pot"):
        np.testing.assert_allclose(out[k], ref[k], rtol=1e-10, atol=0, err_msg=k)
    assert stats["max_level"] >= 1 and stats["n_evaluations"] > 0

