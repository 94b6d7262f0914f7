"""The evaluation as one captured CUDA graph (tc_set_graph).

Graph replays must give the same bits as the normal path: the captured sequence runs the
same kernels on the same data, only with device-sized launches.  Checked on replays with new
body positions in the same buffers, after a capacity overflow (which re-runs the call on the
normal path and re-plans), and with pinned host buffers.
"""
import numpy as np
import pytest


torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _setup(n, seed=11):
    import taichi_collisional_b200 as t
    from taichi_collisional_b200 import ics
    x, y, z, vx, vy, vz, m = ics.plummer_kroupa(n, seed)
    d = {k: torch.tensor(a, device="cuda") for k, a in zip(("x", "y", "z", "vx", "vy", "vz", "m"),
                                                           (x, y, z, vx, vy, vz, m))}
    return t, d


def _eval(g, d, out):
    g.evaluate(d["x"], d["y"], d["z"], d["m"], d["vx"], d["vy"], d["vz"], out=out)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy().copy() for k, v in out.items()}


def _outs(n):
    return {k: torch.empty(n, dtype=torch.float64, device="cuda") for k in ("ax", "ay", "az", "pot", "jx", "jy", "jz")}


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_graph_replay_matches_direct_launches(prec):
    n = 1 << 16
    t, d = _setup(n)
    P = {"mixed": t.PREC_MIXED, "fp64": t.PREC_FP64}[prec]
    gd = t.Gravity(p=12, ncrit=64, theta=0.4, variant=t.VARIANT_JERKS, precision=P, judge_n=64)
    gg = t.Gravity(p=12, ncrit=64, theta=0.4, variant=t.VARIANT_JERKS, precision=P, judge_n=64)
    gg.set_graph(True)
    outg = _outs(n)
    first = _eval(gg, d, outg)  # normal path, then capture
    assert gg.graph_ready(), gg.graph_note()
    for step in range(3):
        if step:
            # move the bodies in place: the captured graph reads the same buffers
            for k in ("x", "y", "z"):
                d[k] += 1e-3 * d["v" + k]
        ref = _eval(gd, d, _outs(n))
        got = _eval(gg, d, outg)
        assert gg.graph_ready()
        for k in ref:
            np.testing.assert_array_equal(got[k], ref[k], err_msg="%s step %d" % (k, step))
        sg, sd = gg.stats(), gd.stats()
        for k in ("n_cells", "n_leaves", "n_m2l", "n_p2p", "n_p2p_inter", "max_level"):
            assert sg[k] == sd[k], k
        assert sg["judge_rms"] == sd["judge_rms"]
        assert sg["n_launches"] > 0
    assert set(first) == set(ref)


def test_graph_replans_after_a_capacity_overflow():
    import taichi_collisional_b200 as t
    n = 1 << 15
    rng = np.random.default_rng(3)
    # planned on bodies along a line (few interaction pairs per cell) ...
    x = np.linspace(-1.0, 1.0, n)
    y = 1e-3 * rng.standard_normal(n)
    z = 1e-3 * rng.standard_normal(n)
    m = np.full(n, 1.0 / n)
    v = 0.1 * rng.standard_normal((3, n))
    d = {k: torch.tensor(a, device="cuda") for k, a in zip(("x", "y", "z", "vx", "vy", "vz", "m"),
                                                           (x, y, z, v[0], v[1], v[2], m))}
    g = t.Gravity(p=8, ncrit=64, theta=0.5, variant=t.VARIANT_JERKS, precision=t.PREC_FP64)
    gd = t.Gravity(p=8, ncrit=64, theta=0.5, variant=t.VARIANT_JERKS, precision=t.PREC_FP64)
    g.set_graph(True)
    out = _outs(n)
    _eval(g, d, out)
    assert g.graph_ready()
    planned = g.stats()["n_m2l"]
    # ... then replayed on a uniform cube in the same buffers: far more pairs than planned
    for k in ("x", "y", "z"):
        d[k].copy_(torch.tensor(rng.uniform(-1.0, 1.0, n), device="cuda"))
    ref = _eval(gd, d, _outs(n))
    assert gd.stats()["n_m2l"] > 2 * planned
    got = _eval(g, d, out)  # the replay overflows; the call re-runs normally and re-plans
    for k in ref:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    assert g.graph_ready()
    got2 = _eval(g, d, out)  # a replay of the new plan
    for k in ref:
        np.testing.assert_array_equal(got2[k], ref[k], err_msg=k)
    assert g.stats()["n_m2l"] == gd.stats()["n_m2l"]


def test_graph_with_pinned_host_buffers():
    n = 1 << 15
    t, d = _setup(n, seed=5)
    hin = {k: v.cpu().pin_memory() for k, v in d.items()}
    hout = {k: torch.empty(n, dtype=torch.float64).pin_memory() for k in ("ax", "ay", "az", "pot", "jx", "jy", "jz")}
    g = t.Gravity(p=10, ncrit=64, theta=0.4, variant=t.VARIANT_JERKS, precision=t.PREC_MIXED)
    gd = t.Gravity(p=10, ncrit=64, theta=0.4, variant=t.VARIANT_JERKS, precision=t.PREC_MIXED)
    g.set_graph(True)
    ref = _eval(gd, d, _outs(n))
    for _ in range(3):
        g.evaluate(hin["x"].numpy(), hin["y"].numpy(), hin["z"].numpy(), hin["m"].numpy(), hin["vx"].numpy(),
                   hin["vy"].numpy(), hin["vz"].numpy(), out={k: v.numpy() for k, v in hout.items()})
        assert g.graph_ready()
        for k in ref:
            np.testing.assert_array_equal(hout[k].numpy(), ref[k], err_msg=k)


def test_graph_survives_buffer_reallocation_by_other_calls():
    """A captured graph bakes in the context's buffers.  tc_evaluate_steps on the same context
    (top tree, small n) needs a larger near-field chunk buffer than tc_evaluate planned, so it
    frees and reallocates it; the next matching tc_evaluate must not replay into the freed
    memory.  Its results must equal a context that never used a graph."""
    import taichi_collisional_b200 as t
    from taichi_collisional_b200 import ics
    n = 20000
    x, y, z, vx, vy, vz, m = ics.plummer_kroupa(n, 21)
    d = {k: torch.tensor(a, device="cuda") for k, a in zip(("x", "y", "z", "vx", "vy", "vz", "m"),
                                                           (x, y, z, vx, vy, vz, m))}
    out = {k: torch.empty(n, dtype=torch.float64, device="cuda") for k in ("ax", "ay", "az", "pot")}
    g = t.Gravity(p=8, ncrit=64, theta=0.5, variant=t.VARIANT_TOP, precision=t.PREC_FP64, direct_below=0)
    gd = t.Gravity(p=8, ncrit=64, theta=0.5, variant=t.VARIANT_TOP, precision=t.PREC_FP64, direct_below=0)
    g.set_graph(True)

    def run(gg, o):
        gg.evaluate(d["x"], d["y"], d["z"], d["m"], out=o)
        torch.cuda.synchronize()
        return {k: v.cpu().numpy().copy() for k, v in o.items()}

    run(g, out)
    assert g.graph_ready(), g.graph_note()
    ref = run(gd, {k: torch.empty_like(v) for k, v in out.items()})
    g.evaluate_steps(d["x"], d["y"], d["z"], d["m"], d["vx"], d["vy"], d["vz"], 0.025)
    torch.cuda.synchronize()
    for _ in range(2):
        got = run(g, out)
        for k in ref:
            np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    assert g.graph_ready()


def test_whole_leapfrog_step_as_one_graph():
    """tc_step_leapfrog with the graph on (kick-drift, evaluation, judge and kick captured as one
    graph) gives the same bits, step after step, as the same steps launched directly."""
    n = 1 << 15
    t, d = _setup(n, seed=9)
    d2 = {k: v.clone() for k, v in d.items()}
    g = t.Gravity(p=10, ncrit=64, theta=0.4, variant=t.VARIANT_JERKS, precision=t.PREC_MIXED, judge_n=32)
    gd = t.Gravity(p=10, ncrit=64, theta=0.4, variant=t.VARIANT_JERKS, precision=t.PREC_MIXED, judge_n=32)
    g.set_graph(True)
    out, out2 = _outs(n), _outs(n)
    for o in (out, out2):
        for v in o.values():
            v.zero_()
    for step in range(4):
        g.step_leapfrog(d, out, 1.0 / 2048)
        gd.step_leapfrog(d2, out2, 1.0 / 2048)
        torch.cuda.synchronize()
        if step:
            assert g.graph_ready(), g.graph_note()
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            assert torch.equal(d[k], d2[k]), (k, step)
        for k in out:
            assert torch.equal(out[k], out2[k]), (k, step)
