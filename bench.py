#!/usr/bin/env python3
"""Benchmark: particle-steps/s of the FMM gravity step on one B200 (replicas on N GPUs).

Workload (one "step"): FP64 leapfrog kick+drift, one full force evaluation (acceleration,
potential and jerk; jerks tree, theta-MAC), closing kick -- on a Plummer sphere of
N = 4,194,304 bodies with Kroupa (2001) masses, p = 12, theta = 0.4, ncrit = 64.  Inputs are
seeded synthetic data (no dataset is involved) and stay resident in HBM; the state
(7 x 32 MiB) is larger than L2, so every step streams from HBM.

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]
  python bench.py --evolve N [--steps K --warmup W]   # the block-time-step integrator instead
  python bench.py --diagnostics N [--steps K --warmup W]   # the energy / centre-of-mass sums

N > 1 (torchrun, one process per GPU): independent replicas, no data-path collective; the
timed region is bracketed by barriers and the slowest rank's device time is reported.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s at N=4M, mixed+learned vs FP64 GPU FMM at equal force error"
UNIT = "particle-steps/s"
WORKLOAD = {"workload": "plummer_kroupa_N4194304_p12_theta0.4_ncrit64_jerks", "n": 4194304, "p": 12,
            "theta": 0.4, "ncrit": 64, "tree": "taichi_with_jerks", "step": "kick-drift + force/jerk eval + kick",
            "l2": "inputs larger than L2 (7 x 32 MiB state)", "ics": "plummer_kroupa"}


def metric_name():
    """The headline metric on the headline workload; the workload's own name otherwise."""
    if WORKLOAD["workload"] == "plummer_kroupa_N4194304_p12_theta0.4_ncrit64_jerks":
        return METRIC
    return "particle-steps/s of the leapfrog step (%s), mixed vs FP64 GPU FMM" % WORKLOAD["workload"]


def set_workload(args):
    """The workload named by the flags (the defaults are the headline: 4M Plummer/Kroupa, p = 12,
    theta = 0.4, ncrit = 64; --ics fractal --n 2097152 --ncrit 32 is the deep fractal cluster,
    --ics plummer --n 1048576 --p 10 the equal-mass million-body case)."""
    eps = args.softening
    # the step of the timed leapfrog: the cold fractal cluster's unsoftened close pairs need a far
    # shorter one than the Plummer sphere's (1/4096 blows it up within a few steps)
    dt = args.dt if args.dt > 0 else (1e-6 if args.ics == "fractal" else 1.0 / 4096)
    WORKLOAD.update(n=args.n, p=args.p, theta=args.theta, ncrit=args.ncrit, ics=args.ics, softening=eps, dt=dt)
    WORKLOAD["workload"] = "%s_N%d_p%d_theta%g_ncrit%d_jerks" % (args.ics, args.n, args.p, args.theta, args.ncrit)
    if eps > 0:
        WORKLOAD["workload"] += "_eps%g" % eps
    WORKLOAD["l2"] = ("inputs larger than L2 (7 x %.0f MiB state)" % (8 * args.n / 2 ** 20) if 56 * args.n > 126e6
                      else "inputs fit in L2")
CPU_SAMPLE_N = 131072


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=WORKLOAD["n"])
    ap.add_argument("--p", type=int, default=WORKLOAD["p"])
    ap.add_argument("--theta", type=float, default=WORKLOAD["theta"])
    ap.add_argument("--ncrit", type=int, default=WORKLOAD["ncrit"])
    ap.add_argument("--ics", default="plummer_kroupa", choices=["plummer_kroupa", "plummer", "fractal"])
    ap.add_argument("--small-run", action="store_true",
                    help="the small plain-method case: 16,384 equal-mass bodies, p = 8, theta = 0.5, one "
                         "evaluation against the reference and FP64 direct sums, then 0.125 time units of the "
                         "block-time-step integrator with softening 1e-4")
    ap.add_argument("--energy-drift", action="store_true",
                    help="energy drift over one time unit of leapfrog steps, FP64 and mixed forms "
                         "(defaults there: 16,777,216 Plummer/Kroupa bodies, p = 16, theta = 0.5)")
    ap.add_argument("--dt", type=float, default=0.0,
                    help="the leapfrog step (default 1/4096; 1e-6 on the fractal cluster; --energy-drift: 1/64)")
    ap.add_argument("--softening", type=float, default=0.0,
                    help="Plummer softening of the pair interactions (the far field stays unsoftened, so it "
                         "should be well below the smallest M2L separation)")
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed", "mixed_m2l"])
    ap.add_argument("--judge", type=int, default=256, help="bodies checked against FP64 direct sums each step")
    ap.add_argument("--selector", type=int, default=2, choices=[0, 1, 2],
                    help="per-pair far-field order: 0 fixed p, 1 analytic estimate, 2 learned (the default: trained "
                         "on the GPU on pairs of this workload before the timed region)")
    ap.add_argument("--train-ics", default=None, choices=["plummer_kroupa", "plummer", "fractal"],
                    help="--selector 2: train on these initial conditions (same n) instead of the workload's own")
    ap.add_argument("--selector-tol", type=float, default=3e-9,
                    help="per-pair truncation error budget relative to the target cell's least |a|")
    ap.add_argument("--no-fp64-arm", action="store_true", help="skip timing the plain FP64 form alongside")
    ap.add_argument("--accuracy-targets", type=int, default=4096,
                    help="seeded bodies at which both forms are compared with FP64 direct sums (untimed)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-graph", action="store_true",
                    help="launch each evaluation's kernels directly instead of replaying one captured CUDA graph")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-budget", type=float, default=1500.0,
                    help="--impl reference: stop timing further steps once this many seconds have passed")
    ap.add_argument("--diagnostics", type=int, default=0, metavar="N",
                    help="time the system diagnostics (energies, centre of mass) over N bodies instead")
    ap.add_argument("--evolve", type=int, default=0, metavar="N",
                    help="time one step of the reference's block-time-step integrator on N bodies instead")
    ap.add_argument("--scheme", default="hold", choices=["hold", "gradient"],
                    help="--evolve: the HOLD scheme or the force-gradient (Omelyan) scheme of the reference's "
                         "default build")
    return ap.parse_args()


def make_ics(n, seed, kind=None):
    from taichi_collisional_b200 import ics
    return getattr(ics, kind or WORKLOAD["ics"])(n, seed)


# ---------------------------------------------------------------------------------------
# algorithmic work per unit
# ---------------------------------------------------------------------------------------
def m2l_flops_per_pair(p, jerk):
    """FP64 operations of one rotation M2L (per source array): scaling 2 x NT, 4 phase
    rotations (12 flops per (n, m>0): complex multiply + next power), 4 swaps (2 per
    non-zero), z-translation (2 per term) and the accumulation (NT)."""
    sys.path.insert(0, os.path.join(ROOT, "taichi_collisional_b200", "csrc"))
    import gen_swap_tables as g
    mats = g.derive(p)
    nnz = sum(1 for n in range(p + 1) for row in mats[n] for v in row if v != 0)
    nt = (p + 1) ** 2
    rot = 4 * 12 * p * (p + 1) // 2
    trans = 0
    for n in range(p + 1):
        trans += (p - n + 1)
        for m in range(1, min(n, p - n) + 1):
            trans += 2 * (p - n - m + 1)
    per_array = 2 * nt + rot + 4 * 2 * nnz + 2 * trans + nt
    return per_array * (2 if jerk else 1)


P2P_FLOPS = {False: 23, True: 60}


# ---------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        self.proc = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(gpu_index)], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.strip().split(",") for r in self.f.read().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].strip().lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        load = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": float(np.median(load)), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------------------
# CPU baseline: the reference's own code (oracle/_ref) or the oracle port
# ---------------------------------------------------------------------------------------
def cpu_runner(x, y, z, vx, vy, vz, m, p, theta, ncrit):
    """One force evaluation (acc + pot + jerk, theta MAC) by the reference's own OpenMP +
    vectorclass build on all host cores (oracle/_ref), or by the oracle port when that build is
    absent.  Returns (run() -> dict of outputs, kind, cores)."""
    import oracle
    cores = os.cpu_count() or 1
    if oracle.ref_available(oracle.VARIANT_JERKS, p):
        os.environ.setdefault("OMP_PROC_BIND", "close")

        def run():
            return oracle.ref_evaluate(x, y, z, m, vx, vy, vz, p=p, theta=theta, ncrit=ncrit,
                                       variant=oracle.VARIANT_JERKS, seed=1, nthreads=cores)
        return run, "reference", cores

    def run_port():
        return oracle.evaluate(x, y, z, m, vx, vy, vz, p=p, theta=theta, ncrit=ncrit, variant=oracle.VARIANT_JERKS,
                               direct_below=0)
    return run_port, "port", 1


def cpu_baseline(n_sample, p, theta, ncrit, gpu_check=None):
    """The CPU build on a bounded sample of the workload (one evaluation of n_sample bodies).
    With gpu_check(x, y, z, vx, vy, vz, m, shift_u) -> outputs, also states how far this
    library's FP64 form is from the reference's own output on the same sample (max over
    particles of the relative acceleration, potential and jerk differences)."""
    import oracle
    x, y, z, vx, vy, vz, m = make_ics(n_sample, 2026)
    run, kind, cores = cpu_runner(x, y, z, vx, vy, vz, m, p, theta, ncrit)
    t0 = time.perf_counter()
    ref = run()
    dt = time.perf_counter() - t0
    sample = ("1 force evaluation (acc+pot+jerk, theta-MAC) of a N=%d Plummer/Kroupa sample, p=%d, theta=%g, "
              "ncrit=%d; the per-particle cost grows ~log N, so the N=4M rate is lower (bench.py --impl reference "
              "times the full N)" % (n_sample, p, theta, ncrit))
    res = {"value": n_sample / dt, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}
    if gpu_check is not None and kind == "reference":
        su = oracle.ref_shift_uniforms(oracle.VARIANT_JERKS, p, 1)
        got = gpu_check(x, y, z, vx, vy, vz, m, su)
        par = {"n": n_sample, "form": "fp64", "against": "the reference's own evaluation (oracle/_ref)"}
        for key, comps in (("acc", ("ax", "ay", "az")), ("jerk", ("jx", "jy", "jz"))):
            a = np.stack([got[c] for c in comps], 1)
            b = np.stack([ref[c] for c in comps], 1)
            e = np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)
            par[key + "_max_rel"] = float(e.max())
        par["pot_max_rel"] = float(np.max(np.abs(got["pot"] - ref["pot"]) / np.abs(ref["pot"])))
        res["parity"] = par
    return res


def run_reference(args, rank):
    """The reference arm: the reference's own CPU build (oracle/_ref, compiled from its sources)
    on the full workload -- the same N, distribution, p, theta, ncrit and step (kick-drift, one
    force evaluation with jerks, kick) as the GPU arm -- on every host core.  Each step is one
    full evaluation at N; steps beyond the time budget are not run, and the line states the
    number actually timed."""
    if rank != 0:
        return
    try:
        n, p = args.n, args.p
        x, y, z, vx, vy, vz, m = make_ics(n, 2026)
        run, kind, cores = cpu_runner(x, y, z, vx, vy, vz, m, p, WORKLOAD["theta"], WORKLOAD["ncrit"])
        dt = WORKLOAD["dt"]
        acc = {"ax": np.zeros(n), "ay": np.zeros(n), "az": np.zeros(n)}

        def step():
            for c in "xyz":
                vel = {"x": vx, "y": vy, "z": vz}[c]
                pos = {"x": x, "y": y, "z": z}[c]
                vel += 0.5 * dt * acc["a" + c]
                pos += dt * vel
            out = run()
            for c in "xyz":
                acc["a" + c][:] = out["a" + c]
                vel = {"x": vx, "y": vy, "z": vz}[c]
                vel += 0.5 * dt * acc["a" + c]

        out = run()
        for c in "xyz":
            acc["a" + c][:] = out["a" + c]
        t_start = time.perf_counter()
        warm = 0
        for _ in range(min(args.warmup, 1)):
            step()
            warm += 1
        times = []
        while len(times) < args.steps:
            t0 = time.perf_counter()
            step()
            times.append(time.perf_counter() - t0)
            if time.perf_counter() - t_start + times[-1] > args.ref_budget:
                break
    except Exception as e:  # pragma: no cover - reported, not hidden
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build failed: %s" % e}))
        return
    k = len(times)
    sec = sum(times)
    value = n * k / sec
    note = ("%d of the %d requested steps timed (time budget %.0f s; one untimed warm-up step of the %d requested)"
            % (k, args.steps, args.ref_budget, args.warmup)) if k < args.steps or warm < args.warmup else None
    sample = ("%d full step(s) at N=%d (kick-drift, one force evaluation acc+pot+jerk with the theta MAC, kick), "
              "p=%d, theta=%g, ncrit=%d, %s" % (k, n, p, WORKLOAD["theta"], WORKLOAD["ncrit"],
                                                "the reference's OpenMP + vectorclass build" if kind == "reference"
                                                else "the oracle port"))
    line = {"metric": metric_name(), "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": k, "warmup": warm, "ms_per_step": 1e3 * sec / k,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Plummer sphere, Kroupa IMF masses)",
            "config": workload_config(n, p, args.gpus),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "seconds_per_step": times}
    if note:
        line["note"] = note
    print(json.dumps(line))


def workload_config(n, p, world):
    """The workload both arms are timed on (identical for the reference arm and this one)."""
    return dict(WORKLOAD, n=n, p=p, parallelism="replicas" if world > 1 else "single")


EVOLVE_CPU_SAMPLE_N = 1024


def run_evolve(args):
    """One do_evolve step (evolve_split_hold_dkd, dt = 1/64, dt_param = 0.025) of the
    reference's block-time-step scheme, device-resident (tc_evolve_hold_dkd), with the top
    tree's error-controlled MAC (force_accuracy 2e-7) at p = 8, ncrit = 64: particle-steps/s
    over K steps, CUDA events around them; beside it the reference's own step (its CPU FMM and
    integrator, oracle/_ref) on a 1,024-body sample."""
    import torch
    import taichi_collisional_b200 as tcb
    n, dt, dtp, fa = args.evolve, 1.0 / 64, 0.025, 2e-7
    x, y, z, vx, vy, vz, m = make_ics(n, 2027)
    zero = np.zeros(n)
    host = dict(x=x, y=y, z=z, vx=vx, vy=vy, vz=vz, m=m, ex=zero, ey=zero, ez=zero, timestep=zero, pot=zero)
    st = {k: torch.tensor(v, dtype=torch.float64, device="cuda") for k, v in host.items()}
    st["id"] = torch.arange(n, dtype=torch.int32, device="cuda")
    g = tcb.Gravity(p=8, ncrit=64, theta=0.4, variant=tcb.VARIANT_TOP, precision=tcb.PREC_FP64)
    g.set_error_mac(True, fa)
    grad = args.scheme == "gradient"
    step = g.evolve_omelyan if grad else g.evolve_hold_dkd
    for _ in range(args.warmup):
        step(st, dtp, dt)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    e0.record()
    for _ in range(args.steps):
        stats.append(step(st, dtp, dt))
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    name = "force-gradient (Omelyan)" if grad else "HOLD"
    line = {"metric": "particle-steps/s of one %s block-time-step step (p=8, error MAC)" % name, "impl": "ours",
            "value": n / (ms * 1e-3), "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "dtype": "f64", "data": "synthetic (seeded Plummer/Kroupa)",
            "config": {"workload": "%s_plummer_kroupa_N%d_p8_fa2e-7_dt1/64" % ("omelyan" if grad else "hold_dkd", n),
                       "n": n, "p": 8, "ncrit": 64,
                       "force_accuracy": fa, "dt": dt, "dt_param": dtp},
            "per_step": {k: [s[k] for s in stats] for k in ("n_evaluations", "n_direct", "max_level")}}
    import oracle
    if not args.no_cpu_baseline and not grad and oracle.integ_ref_available():
        xs, ys, zs, vxs, vys, vzs, ms_ = make_ics(EVOLVE_CPU_SAMPLE_N, 2027)
        z0 = np.zeros(EVOLVE_CPU_SAMPLE_N)
        s0 = dict(x=xs, y=ys, z=zs, vx=vxs, vy=vys, vz=vzs, m=ms_, ex=z0, ey=z0, ez=z0, timestep=z0, pot=z0,
                  id=np.arange(EVOLVE_CPU_SAMPLE_N, dtype=np.int32))
        t0 = time.perf_counter()
        oracle.ref_evolve_hold(s0, ncrit=64, theta=0.4, force_accuracy=fa, dt_param=dtp, dt=dt)
        sec = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": EVOLVE_CPU_SAMPLE_N / sec, "unit": UNIT, "cores": os.cpu_count() or 1,
                                "kind": "reference", "sample": "one HOLD step of a %d-body Plummer/Kroupa sample "
                                "(the reference's integrator.h and CPU FMM, p = 8)" % EVOLVE_CPU_SAMPLE_N}
    print(json.dumps(line))
    g.close()


def run_diagnostics(args):
    """tc_system_diagnostics over N resident bodies (kinetic and potential energy, mass, centre of
    mass and its velocity: 64 algorithmic bytes read per body); CUDA events around K calls, the
    roofline against the measured HBM copy bandwidth."""
    import torch
    import taichi_collisional_b200 as tcb
    n = args.diagnostics
    x, y, z, vx, vy, vz, m = make_ics(n, 2028)
    pot = np.random.default_rng(5).random(n)
    arrs = [torch.tensor(a, dtype=torch.float64, device="cuda") for a in (m, x, y, z, vx, vy, vz, pot)]
    g = tcb.Gravity(p=8, ncrit=64, theta=0.4, variant=tcb.VARIANT_TOP, precision=tcb.PREC_FP64)
    for _ in range(args.warmup):
        d = g.system_diagnostics(*arrs)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        d = g.system_diagnostics(*arrs)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    gbs = 64.0 * n / (ms * 1e-3) / 1e9
    peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak = json.load(f).get("hbm_gbs")
    except (OSError, ValueError):
        pass
    line = {"metric": "bodies/s of the system diagnostics (energies, centre of mass)", "impl": "ours",
            "value": n / (ms * 1e-3), "unit": "bodies/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "dtype": "f64 (double-double sums)",
            "data": "synthetic (seeded Plummer/Kroupa)",
            "config": {"workload": "system_diagnostics_plummer_kroupa_N%d" % n, "n": n,
                       "l2": "inputs larger than L2 (8 x 8 B per body)" if 64 * n > 126e6 else "inputs fit in L2"},
            "roofline": {"kernel": "k_sys_diag_part", "bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                         "frac": gbs / peak if peak else None, "work": "64 B read per body (call: both kernels)"},
            "result": d}
    print(json.dumps(line))
    g.close()


def run_small(args):
    """The small plain-method case: 16,384 equal-mass Plummer bodies (Henon units, r < 10), the
    top-level tree, p = 8, theta = 0.5, ncrit = 64.
    (1) One FP64 evaluation against the reference's own FMM (oracle/_ref, compiled from its
        sources) and against FP64 direct sums.
    (2) 0.125 time units -- 8 do_evolve steps of dt = 1/64 -- of the block-time-step integrator
        (HOLD scheme, the top tree's error MAC with force_accuracy 2e-7, dt_param 0.025): with
        softening 1e-4 (energy drift), and without softening next to the reference's own
        integrator and CPU FMM on the same bodies (final positions and energies)."""
    import torch
    import oracle
    import taichi_collisional_b200 as tcb
    n, p, theta, ncrit, dt, nstep, fa, dtp = 16384, 8, 0.5, 64, 1.0 / 64, 8, 2e-7, 0.025
    x, y, z, vx, vy, vz, m = make_ics(n, 2029, "plummer")
    line = {"metric": "small plain-method case (parity and integrator)", "impl": "ours",
            "config": {"workload": "plummer_N16384_p8_theta0.5_ncrit64_top", "n": n, "p": p, "theta": theta,
                       "ncrit": ncrit, "integrator": "HOLD dkd, error MAC fa=2e-7, dt=1/64 x 8, dt_param=0.025"}}
    # (1) one evaluation
    g = tcb.Gravity(p=p, ncrit=ncrit, theta=theta, variant=tcb.VARIANT_TOP, precision=tcb.PREC_FP64, direct_below=0)
    out = g.evaluate(x, y, z, m)
    g.close()
    d = oracle.direct(x, y, z, m)
    av = lambda o: np.stack([o["ax"], o["ay"], o["az"]], 1)  # noqa: E731
    erel = lambda a, b: np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)  # noqa: E731
    ev = {"rms_rel_acc_err_vs_direct": float(np.sqrt(np.mean(erel(av(out), av(d)) ** 2)))}
    if oracle.ref_available(oracle.VARIANT_TOP, p):
        ref = oracle.ref_evaluate(x, y, z, m, p=p, theta=theta, ncrit=ncrit, variant=oracle.VARIANT_TOP,
                                  nthreads=os.cpu_count() or 1)
        ev["max_rel_acc_diff_vs_reference"] = float(erel(av(out), av(ref)).max())
        ev["max_rel_pot_diff_vs_reference"] = float(np.max(np.abs(out["pot"] - ref["pot"]) / np.abs(ref["pot"])))
        ev["reference_rms_rel_acc_err_vs_direct"] = float(np.sqrt(np.mean(erel(av(ref), av(d)) ** 2)))
    line["evaluation"] = ev

    # (2) the integrator
    def evolve(eps):
        gi = tcb.Gravity(p=p, ncrit=ncrit, theta=theta, variant=tcb.VARIANT_TOP, precision=tcb.PREC_FP64,
                         softening=eps)
        gi.set_error_mac(True, fa)
        zero = np.zeros(n)
        st = {k: torch.tensor(v, dtype=torch.float64, device="cuda") for k, v in
              dict(x=x, y=y, z=z, vx=vx, vy=vy, vz=vz, m=m, ex=zero, ey=zero, ez=zero, timestep=zero,
                   pot=zero).items()}
        st["id"] = torch.arange(n, dtype=torch.int32, device="cuda")

        def energy():
            o = gi.evaluate(st["x"], st["y"], st["z"], st["m"])
            dg = gi.system_diagnostics(st["m"], st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], o["pot"])
            return dg["kinetic"] - dg["potential"]
        e0 = energy()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(nstep):
            gi.evolve_hold_dkd(st, dtp, dt)
        torch.cuda.synchronize()
        sec = time.perf_counter() - t0
        e1 = energy()
        gi.close()
        return st, e0, e1, sec
    runs = {}
    for eps in (1e-4, 0.0):
        st, e0, e1, sec = evolve(eps)
        runs[eps] = st
        line["evolve_eps%g" % eps] = {"E0": e0, "E1": e1, "rel_energy_drift": abs(e1 - e0) / abs(e0),
                                      "seconds": sec, "particle_steps_per_s": n * nstep / sec}
    if oracle.integ_ref_available():
        zero = np.zeros(n)
        s0 = dict(x=x, y=y, z=z, vx=vx, vy=vy, vz=vz, m=m, ex=zero, ey=zero, ez=zero, timestep=zero, pot=zero,
                  id=np.arange(n, dtype=np.int32))
        t0 = time.perf_counter()
        for _ in range(nstep):
            s0, _ = oracle.ref_evolve_hold(s0, ncrit=ncrit, theta=0.4, force_accuracy=fa, dt_param=dtp, dt=dt)
        sec = time.perf_counter() - t0
        ours = {k: v.cpu().numpy() for k, v in runs[0.0].items()}
        o_pos = np.zeros((n, 3))
        r_pos = np.zeros((n, 3))
        o_pos[ours["id"]] = np.stack([ours["x"], ours["y"], ours["z"]], 1)
        r_pos[s0["id"]] = np.stack([s0["x"], s0["y"], s0["z"]], 1)
        disp = np.linalg.norm(r_pos - np.stack([x, y, z], 1), axis=1)
        dev = np.linalg.norm(o_pos - r_pos, axis=1)
        line["vs_reference_integrator_eps0"] = {
            "max_pos_diff_over_max_displacement": float(dev.max() / disp.max()),
            "median_pos_diff_over_displacement": float(np.median(dev / np.maximum(disp, 1e-300))),
            "reference_seconds": sec, "reference_cores": os.cpu_count() or 1}
    print(json.dumps(line))


def run_energy_drift(args):
    """Energy drift over one time unit of shared-step leapfrog (tc_step_leapfrog, one graph replay
    per step) for the FP64 form and the mixed form, from the same initial state.  Defaults: the
    largest configuration, 16,777,216 Plummer/Kroupa bodies, p = 16, theta = 0.5, ncrit = 64, jerks
    tree, dt = 1/64 (64 steps)."""
    import torch
    import taichi_collisional_b200 as tcb
    given = set(a.split("=")[0] for a in sys.argv[1:])
    n = args.n if "--n" in given else 16777216
    p = args.p if "--p" in given else 16
    theta = args.theta if "--theta" in given else 0.5
    ncrit = args.ncrit
    dt = args.dt if args.dt > 0 else 1.0 / 64
    nstep = int(round(1.0 / dt))
    x, y, z, vx, vy, vz, m = make_ics(n, 2030, "plummer_kroupa")
    line = {"metric": "relative energy drift over 1 time unit", "impl": "ours",
            "config": {"workload": "plummer_kroupa_N%d_p%d_theta%g_ncrit%d_jerks" % (n, p, theta, ncrit), "n": n,
                       "p": p, "theta": theta, "ncrit": ncrit, "dt": dt, "steps": nstep,
                       "integrator": "shared-step leapfrog (kick-drift-kick), one CUDA graph per step"}}
    for name, prec in (("fp64", tcb.PREC_FP64), ("mixed", tcb.PREC_MIXED)):
        st = {k: torch.tensor(a, dtype=torch.float64, device="cuda")
              for k, a in zip(("x", "y", "z", "vx", "vy", "vz", "m"), (x, y, z, vx, vy, vz, m))}
        out = {k: torch.zeros(n, dtype=torch.float64, device="cuda") for k in ("ax", "ay", "az", "pot", "jx", "jy",
                                                                                 "jz")}
        g = tcb.Gravity(p=p, ncrit=ncrit, theta=theta, variant=tcb.VARIANT_JERKS, precision=prec)
        if name == "mixed" and args.selector:
            if args.selector == 2:
                rep = g.train_selector(x, y, z, m, vx, vy, vz, nsamples=16384, iters=1500, seed=5)
                line["training"] = {k: rep[k] for k in ("samples", "val_loss", "seconds", "class_order")}
            g.set_selector(args.selector, args.selector_tol)
            line["selector"] = {"kind": ["fixed p", "analytic", "learned"][args.selector], "tol": args.selector_tol}
        g.set_graph(True)
        g.evaluate(st["x"], st["y"], st["z"], st["m"], st["vx"], st["vy"], st["vz"], out=out)

        def energy():
            dg = g.system_diagnostics(st["m"], st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], out["pot"])
            return dg["kinetic"] - dg["potential"]
        e0 = energy()
        torch.cuda.synchronize()
        e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e_start.record()
        for _ in range(nstep):
            g.step_leapfrog(st, out, dt)
        e_end.record()
        torch.cuda.synchronize()
        ms = e_start.elapsed_time(e_end)
        e1 = energy()
        line[name] = {"E0": e0, "E1": e1, "rel_energy_drift": abs(e1 - e0) / abs(e0), "ms_per_step": ms / nstep,
                      "particle_steps_per_s": n * nstep / (ms * 1e-3), "m2l_pairs": g.stats()["n_m2l"],
                      "m2l_flop_fraction": g.stats()["m2l_flop_fraction"]}
        g.close()
        del st, out
        torch.cuda.empty_cache()
    print(json.dumps(line))


def error_stats(out, idx_t, ref):
    """RMS and 99th percentile of |a - a_ref| / |a_ref| and |j - j_ref| / |j_ref| at the
    targets idx_t (out: device tensors of one evaluation, ref: direct sums at those bodies)."""
    res = {}
    for key, pre in (("acc", "a"), ("jerk", "j")):
        got = np.stack([out[pre + c][idx_t].cpu().numpy() for c in "xyz"], 1)
        want = np.stack([ref[pre + c] for c in "xyz"], 1)
        e = np.linalg.norm(got - want, axis=1) / np.linalg.norm(want, axis=1)
        res[key + "_rms"] = float(np.sqrt(np.mean(e ** 2)))
        res[key + "_p99"] = float(np.quantile(e, 0.99))
    return res


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    set_workload(args)
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.small_run:
        run_small(args)
        return
    if args.energy_drift:
        run_energy_drift(args)
        return
    if args.evolve:
        run_evolve(args)
        return
    if args.diagnostics:
        run_diagnostics(args)
        return
    import datetime

    import torch
    import taichi_collisional_b200 as tcb
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    n, p = args.n, args.p
    x, y, z, vx, vy, vz, m = make_ics(n, 2026 + rank)
    T = lambda a: torch.tensor(a, dtype=torch.float64, device=dev)  # noqa: E731
    st = {k: T(a) for k, a in zip(("x", "y", "z", "vx", "vy", "vz", "m"), (x, y, z, vx, vy, vz, m))}
    out = {k: torch.empty(n, dtype=torch.float64, device=dev) for k in ("ax", "ay", "az", "pot", "jx", "jy", "jz")}
    prec = {"fp64": tcb.PREC_FP64, "mixed": tcb.PREC_MIXED, "mixed_m2l": tcb.PREC_MIXED_M2L}[args.precision]
    g = tcb.Gravity(p=p, ncrit=WORKLOAD["ncrit"], theta=WORKLOAD["theta"], variant=tcb.VARIANT_JERKS,
                    precision=prec, device=local, judge_n=args.judge, softening=WORKLOAD["softening"])
    train = None
    if args.selector == 2:  # the learned selector, trained on the GPU on pairs of this workload (untimed)
        tr = (x, y, z, vx, vy, vz, m) if not args.train_ics else make_ics(n, 2026 + rank, args.train_ics)
        rep = g.train_selector(tr[0], tr[1], tr[2], tr[6], tr[3], tr[4], tr[5], nsamples=16384, iters=1500, seed=5)
        train = {k: rep[k] for k in ("samples", "iters", "train_loss", "val_loss", "seconds", "class_order")}
        train["ics"] = args.train_ics or WORKLOAD["ics"]
    if args.selector:
        g.set_selector(args.selector, args.selector_tol)
    g.set_graph(not args.no_graph)  # the first evaluation captures, the later ones replay
    dt = WORKLOAD["dt"]

    def evaluate():
        g.evaluate(st["x"], st["y"], st["z"], st["m"], st["vx"], st["vy"], st["vz"], out=out)

    def step():  # kick-drift, evaluation, kick: one CUDA graph replay with the graph on
        g.step_leapfrog(st, out, dt)

    evaluate()
    for _ in range(max(args.warmup, 0)):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    phase = {k: 0.0 for k in ("ms_tree", "ms_upward", "ms_traverse", "ms_m2l", "ms_p2p", "ms_downward")}
    launches = 0
    e0.record()
    for _ in range(args.steps):
        step()
        s = g.stats()
        for k in phase:
            phase[k] += s[k]
        launches += s["n_launches"] + (0 if g.graph_ready() else 2)  # the graph counts its two kicks
    e1.record()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * n * args.steps / (ms * 1e-3)
    stats = g.stats()

    # ---- the plain FP64 form, same step definition (kick-drift, evaluation, kick) and timing
    # rules, on its own copy of the state (the comparison arm)
    g64 = None
    fp64 = None
    if not args.no_fp64_arm and args.precision != "fp64":
        g64 = tcb.Gravity(p=p, ncrit=WORKLOAD["ncrit"], theta=WORKLOAD["theta"], variant=tcb.VARIANT_JERKS,
                          precision=tcb.PREC_FP64, device=local, judge_n=args.judge,
                          softening=WORKLOAD["softening"])
        g64.set_graph(not args.no_graph)
        st64 = {k: v.clone() for k, v in st.items()}
        out64 = {k: torch.empty_like(v) for k, v in out.items()}

        def step64():
            g64.step_leapfrog(st64, out64, dt)

        g64.evaluate(st64["x"], st64["y"], st64["z"], st64["m"], st64["vx"], st64["vy"], st64["vz"], out=out64)
        for _ in range(max(args.warmup, 0)):
            step64()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        h0.record()
        for _ in range(args.steps):
            step64()
        h1.record()
        torch.cuda.synchronize()
        ms64 = h0.elapsed_time(h1)
        if dist:
            t = torch.tensor([ms64], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms64 = float(t.item())
        s64 = g64.stats()
        fp64 = {"value": world * n * args.steps / (ms64 * 1e-3), "ms_per_step": ms64 / args.steps,
                "judge_rms_acc_err": s64["judge_rms"],
                "note": "same step as the headline (kick-drift, FP64 evaluation, kick: one graph replay)"}
        del st64

    # ---- accuracy (untimed): both forms against FP64 direct sums at 4,096 seeded bodies, on the
    # initial state and on the state after the warm-up and timed steps; RMS and 99th percentile
    # of the relative acceleration and jerk errors
    accuracy = {"judge_bodies": args.judge, "judge_rms_rel_acc_err": stats["judge_rms"]}
    if args.accuracy_targets > 0:
        nt = min(args.accuracy_targets, n)
        idx = np.sort(np.random.default_rng(2027 + rank).choice(n, nt, replace=False))
        idx_t = torch.tensor(idx, device=dev)
        accuracy["targets"] = nt
        init = {k: T(a) for k, a in zip(("x", "y", "z", "vx", "vy", "vz", "m"), make_ics(n, 2026 + rank))}
        states = []
        for label, s_ in (("initial", init), ("after %d steps" % (args.warmup + args.steps), st)):
            o1 = {k: torch.empty_like(v) for k, v in out.items()}
            g.evaluate(s_["x"], s_["y"], s_["z"], s_["m"], s_["vx"], s_["vy"], s_["vz"], out=o1)
            ref = g.direct_sums(s_["x"], s_["y"], s_["z"], s_["m"], idx, s_["vx"], s_["vy"], s_["vz"])
            row = {"state": label, args.precision: error_stats(o1, idx_t, ref)}
            if g64 is not None:
                o2 = {k: torch.empty_like(v) for k, v in out.items()}
                g64.evaluate(s_["x"], s_["y"], s_["z"], s_["m"], s_["vx"], s_["vy"], s_["vz"], out=o2)
                row["fp64"] = error_stats(o2, idx_t, ref)
                row["acc_rms_ratio"] = row[args.precision]["acc_rms"] / row["fp64"]["acc_rms"]
            states.append(row)
        accuracy["states"] = states
        # the headline's condition: the worse of the two states
        if g64 is not None:
            accuracy["acc_rms_ratio"] = max(r_["acc_rms_ratio"] for r_ in states)
        del init
    if g64 is not None:
        g64.close()

    # ---- end to end through the public API: pinned host state in, results out, every step
    e2e = None
    if not args.no_e2e:
        hin = {k: st[k].to("cpu").pin_memory() for k in st}
        hout = {k: torch.empty(n, dtype=torch.float64).pin_memory() for k in out}
        step()  # the accuracy leg's other buffers dropped the step's graph: capture it again, untimed
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        for _ in range(args.steps):
            for k in st:
                st[k].copy_(hin[k], non_blocking=True)
            step()
            for k in out:
                hout[k].copy_(out[k], non_blocking=True)
        f1.record()
        torch.cuda.synchronize()
        ems = f0.elapsed_time(f1)
        if dist:
            t = torch.tensor([ems], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        e2e = {"value": world * n * args.steps / (ems * 1e-3), "unit": UNIT, "h2d_bytes_per_step": 7 * 8 * n,
               "d2h_bytes_per_step": 7 * 8 * n, "ms_per_step": ems / args.steps}

    # ---- roofline of the dominant kernel
    per = {k: v / args.steps for k, v in phase.items()}
    fp64_peak = g.probe_peak(0) / 1e3  # TFLOP/s, measured FMA throughput of this GPU
    # with per-pair orders: the selected orders' share of the fixed-order flops, (q+1)^3 / (p+1)^3 per
    # pair (a batch of 32 pairs runs at its largest order, so the kernel does at least this work)
    m2l_flops = stats["n_m2l"] * m2l_flops_per_pair(p, True) * stats["m2l_flop_fraction"]
    p2p_flops = stats["n_p2p_inter"] * P2P_FLOPS[True]
    kern = {"k_m2l": (per["ms_m2l"], m2l_flops), "k_p2p": (per["ms_p2p"], p2p_flops)}
    dom = max(kern, key=lambda k: kern[k][0])
    ach = kern[dom][1] / (kern[dom][0] * 1e-3) / 1e12
    roof = {"kernel": dom, "bound": "fp64", "achieved": ach, "peak": fp64_peak, "unit": "TFLOP/s",
            "frac": ach / fp64_peak if fp64_peak > 0 else None, "traffic": None,
            "peak_source": "FP64 FMA throughput measured on this GPU by tc_probe_peak (MEASURED_PEAKS.json has "
                           "no FP64 figure)",
            "work": "%s: %.3e flop per launch" % (dom, kern[dom][1]),
            "phase_ms": {k: round(v, 3) for k, v in per.items()},
            "other": {k: {"ms": round(v[0], 3), "tflops": round(v[1] / (v[0] * 1e-3) / 1e12, 3) if v[0] else None}
                      for k, v in kern.items()}}
    if args.precision != "fp64" and per["ms_p2p"] > 0:
        # the mixed near field computes in FP32: its fraction of the measured FP32 FMA throughput
        fp32_peak = g.probe_peak(1) / 1e3
        ach32 = p2p_flops / (per["ms_p2p"] * 1e-3) / 1e12
        roof["other"]["k_p2p"].update(bound="fp32", peak=round(fp32_peak, 3),
                                      frac=round(ach32 / fp32_peak, 4) if fp32_peak > 0 else None)

    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            def gpu_fp64(xs, ys, zs, vxs, vys, vzs, ms_, su):
                gs = tcb.Gravity(p=p, ncrit=WORKLOAD["ncrit"], theta=WORKLOAD["theta"], variant=tcb.VARIANT_JERKS,
                                 precision=tcb.PREC_FP64, device=local, shift_u=su, direct_below=0)
                o = gs.evaluate(xs, ys, zs, ms_, vxs, vys, vzs)
                gs.close()
                return o
            cb = cpu_baseline(CPU_SAMPLE_N, p, WORKLOAD["theta"], WORKLOAD["ncrit"], gpu_check=gpu_fp64)
        except Exception as e:
            cb = {"value": None, "error": str(e)}
    if rank == 0:
        line = {"metric": metric_name(), "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
                "data": "synthetic (seeded Plummer sphere, Kroupa IMF masses)",
                "config": workload_config(n, p, world),
                "form": {"precision": args.precision,
                         "evaluation": "one CUDA graph replay" if g.graph_ready() else "direct launches",
                         "selector": ["fixed p", "analytic", "learned"][args.selector],
                         "selector_tol": args.selector_tol if args.selector else None,
                         "orders": dict(zip(stats["class_order"], stats["class_pairs"])),
                         "m2l_flop_fraction": stats["m2l_flop_fraction"], "training": train},
                "e2e": e2e, "gpu_launches": launches, "roofline": roof, "cpu_baseline": cb, "clocks": clocks,
                "accuracy": accuracy,
                "fp64_form": fp64,
                "lists": {"cells": stats["n_cells"], "m2l_pairs": stats["n_m2l"], "p2p_pairs": stats["n_p2p"],
                          "p2p_interactions": stats["n_p2p_inter"], "max_level": stats["max_level"],
                          "flags": stats["flags"]}}
        print(json.dumps(line))
    g.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
