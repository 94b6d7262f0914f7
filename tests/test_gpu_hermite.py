"""Hermite 4th-order step (tc_hermite_predict / tc_hermite_correct) around the jerks tree's
evaluation.  It has no counterpart in the reference, so it is checked on its own terms: the
update formulas against numpy on the same forces, and fourth-order behaviour on a circular
two-body orbit (energy and closure over one period, against the FP64 leapfrog kick-drift)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _eval(g, s, out):
    g.evaluate(s["x"], s["y"], s["z"], s["m"], s["vx"], s["vy"], s["vz"], out=out)


def test_hermite_update_formulas_match_numpy():
    import taichi_collisional_b200 as t
    from taichi_collisional_b200 import ics
    n, dt = 600, 1.0 / 512
    x, y, z, vx, vy, vz, m = ics.plummer_kroupa(n, 3)
    s = {k: torch.tensor(a, device="cuda") for k, a in zip(("x", "y", "z", "vx", "vy", "vz", "m"),
                                                           (x, y, z, vx, vy, vz, m))}
    g = t.Gravity(p=8, ncrit=32, theta=0.5, variant=t.VARIANT_JERKS, precision=t.PREC_FP64)
    a = {k: torch.empty(n, dtype=torch.float64, device="cuda") for k in ("ax", "ay", "az", "pot", "jx", "jy", "jz")}
    _eval(g, s, a)
    a0 = {k: v.cpu().numpy().copy() for k, v in a.items()}
    save = torch.empty(12 * n, dtype=torch.float64, device="cuda")
    g.hermite_predict(s["x"], s["y"], s["z"], s["vx"], s["vy"], s["vz"], a, save, dt)
    X0, V0 = (x, y, z), (vx, vy, vz)
    for d, (kx, kv, ka, kj) in enumerate(zip("xyz", ("vx", "vy", "vz"), ("ax", "ay", "az"), ("jx", "jy", "jz"))):
        xp = X0[d] + dt * (V0[d] + dt * (a0[ka] / 2 + dt * (a0[kj] / 6)))
        vp = V0[d] + dt * (a0[ka] + dt * (a0[kj] / 2))
        np.testing.assert_allclose(s[kx].cpu().numpy(), xp, rtol=1e-14, atol=1e-16)
        np.testing.assert_allclose(s[kv].cpu().numpy(), vp, rtol=1e-14, atol=1e-16)
    _eval(g, s, a)
    a1 = {k: v.cpu().numpy().copy() for k, v in a.items()}
    g.hermite_correct(s["x"], s["y"], s["z"], s["vx"], s["vy"], s["vz"], a, save, dt)
    for d, (kx, kv, ka, kj) in enumerate(zip("xyz", ("vx", "vy", "vz"), ("ax", "ay", "az"), ("jx", "jy", "jz"))):
        v1 = V0[d] + dt / 2 * (a0[ka] + a1[ka]) + dt * dt / 12 * (a0[kj] - a1[kj])
        x1 = X0[d] + dt / 2 * (V0[d] + v1) + dt * dt / 12 * (a0[ka] - a1[ka])
        np.testing.assert_allclose(s[kv].cpu().numpy(), v1, rtol=1e-14, atol=1e-16)
        np.testing.assert_allclose(s[kx].cpu().numpy(), x1, rtol=1e-14, atol=1e-16)


def _energy(s, out):
    m = s["m"].cpu().numpy()
    v2 = sum(s[k].cpu().numpy() ** 2 for k in ("vx", "vy", "vz"))
    return 0.5 * np.sum(m * v2) - 0.5 * np.sum(m * out["pot"].cpu().numpy())


def _binary():
    # equal masses on a circular orbit of separation 1 (period 2 pi)
    x = np.array([0.5, -0.5]); y = np.zeros(2); z = np.zeros(2)
    vx = np.zeros(2); vy = np.array([0.5, -0.5]); vz = np.zeros(2); m = np.array([0.5, 0.5])
    return {k: torch.tensor(a, device="cuda") for k, a in zip(("x", "y", "z", "vx", "vy", "vz", "m"),
                                                              (x, y, z, vx, vy, vz, m))}


def test_hermite_is_fourth_order_on_a_circular_binary():
    import taichi_collisional_b200 as t
    g = t.Gravity(p=8, ncrit=32, theta=0.5, variant=t.VARIANT_JERKS, precision=t.PREC_FP64)
    errs = {}
    for steps in (64, 128):
        dt = 2 * np.pi / steps
        for scheme in ("hermite", "leapfrog"):
            s = _binary()
            a = {k: torch.empty(2, dtype=torch.float64, device="cuda") for k in ("ax", "ay", "az", "pot", "jx", "jy", "jz")}
            _eval(g, s, a)
            e0 = _energy(s, a)
            save = torch.empty(24, dtype=torch.float64, device="cuda")
            for _ in range(steps):
                if scheme == "hermite":
                    g.hermite_predict(s["x"], s["y"], s["z"], s["vx"], s["vy"], s["vz"], a, save, dt)
                    _eval(g, s, a)
                    g.hermite_correct(s["x"], s["y"], s["z"], s["vx"], s["vy"], s["vz"], a, save, dt)
                    _eval(g, s, a)
                else:
                    g.kick_drift(s["x"], s["y"], s["z"], s["vx"], s["vy"], s["vz"], a["ax"], a["ay"], a["az"], 0.5 * dt, dt)
                    _eval(g, s, a)
                    g.kick_drift(s["x"], s["y"], s["z"], s["vx"], s["vy"], s["vz"], a["ax"], a["ay"], a["az"], 0.5 * dt, 0.0)
            torch.cuda.synchronize()
            de = abs(_energy(s, a) - e0) / abs(e0)
            dx = abs(s["x"][0].item() - 0.5) + abs(s["y"][0].item())
            errs[(scheme, steps)] = (de, dx)
    # fourth order: halving dt cuts the closure error by ~16 (leapfrog: ~4)
    h64, h128 = errs[("hermite", 64)][1], errs[("hermite", 128)][1]
    l64, l128 = errs[("leapfrog", 64)][1], errs[("leapfrog", 128)][1]
    assert h64 / h128 > 10, errs
    assert l64 / l128 < 6, errs
    assert errs[("hermite", 128)][0] < 1e-6 and errs[("hermite", 128)][1] < 1e-4, errs
    assert h128 < 1e-2 * l128, errs
