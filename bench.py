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
            "l2": "inputs larger than L2 (7 x 32 MiB state)"}
CPU_SAMPLE_N = 131072


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=WORKLOAD["n"])
    ap.add_argument("--p", type=int, default=WORKLOAD["p"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed", "mixed_m2l"])
    ap.add_argument("--judge", type=int, default=256, help="bodies checked against FP64 direct sums each step")
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
                    help="time one step of the HOLD block-time-step integrator on N bodies instead")
    return ap.parse_args()


def make_ics(n, seed):
    from taichi_collisional_b200 import ics
    return ics.plummer_kroupa(n, seed)


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
        dt = 1.0 / 4096
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
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
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
    for _ in range(args.warmup):
        g.evolve_hold_dkd(st, dtp, dt)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    e0.record()
    for _ in range(args.steps):
        stats.append(g.evolve_hold_dkd(st, dtp, dt))
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    line = {"metric": "particle-steps/s of one HOLD block-time-step step (p=8, error MAC)", "impl": "ours",
            "value": n / (ms * 1e-3), "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "dtype": "f64", "data": "synthetic (seeded Plummer/Kroupa)",
            "config": {"workload": "hold_dkd_plummer_kroupa_N%d_p8_fa2e-7_dt1/64" % n, "n": n, "p": 8, "ncrit": 64,
                       "force_accuracy": fa, "dt": dt, "dt_param": dtp},
            "per_step": {k: [s[k] for s in stats] for k in ("n_evaluations", "n_direct", "max_level")}}
    import oracle
    if not args.no_cpu_baseline and oracle.integ_ref_available():
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
    if args.impl == "reference":
        run_reference(args, rank)
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
                    precision=prec, device=local, judge_n=args.judge)
    g.set_graph(not args.no_graph)  # the first evaluation captures, the later ones replay
    dt = 1.0 / 4096

    def evaluate():
        g.evaluate(st["x"], st["y"], st["z"], st["m"], st["vx"], st["vy"], st["vz"], out=out)

    def step():
        g.kick_drift(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], out["ax"], out["ay"], out["az"],
                     0.5 * dt, dt)
        evaluate()
        g.kick_drift(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], out["ax"], out["ay"], out["az"],
                     0.5 * dt, 0.0)

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
        launches += s["n_launches"] + 2
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

    # ---- accuracy (untimed): both forms on the current state against FP64 direct sums at
    # seeded bodies; RMS and 99th percentile of the relative acceleration and jerk errors
    accuracy = {"judge_bodies": args.judge, "judge_rms_rel_acc_err": stats["judge_rms"]}
    ref = idx_t = None
    if args.accuracy_targets > 0:
        nt = min(args.accuracy_targets, n)
        idx = np.sort(np.random.default_rng(2027 + rank).choice(n, nt, replace=False))
        idx_t = torch.tensor(idx, device=dev)
        g.evaluate(st["x"], st["y"], st["z"], st["m"], st["vx"], st["vy"], st["vz"], out=out)
        ref = g.direct_sums(st["x"], st["y"], st["z"], st["m"], idx, st["vx"], st["vy"], st["vz"])
        accuracy["targets"] = nt
        accuracy[args.precision] = error_stats(out, idx_t, ref)

    # ---- the plain FP64 form on the same state, same timing rules (the comparison arm)
    fp64 = None
    if not args.no_fp64_arm and args.precision != "fp64":
        g64 = tcb.Gravity(p=p, ncrit=WORKLOAD["ncrit"], theta=WORKLOAD["theta"], variant=tcb.VARIANT_JERKS,
                          precision=tcb.PREC_FP64, device=local, judge_n=args.judge)
        g64.set_graph(not args.no_graph)
        out64 = {k: torch.empty_like(v) for k, v in out.items()}
        g64.evaluate(st["x"], st["y"], st["z"], st["m"], st["vx"], st["vy"], st["vz"], out=out64)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        h0.record()
        for _ in range(args.steps):
            g64.evaluate(st["x"], st["y"], st["z"], st["m"], st["vx"], st["vy"], st["vz"], out=out64)
        h1.record()
        torch.cuda.synchronize()
        ms64 = h0.elapsed_time(h1)
        if dist:
            t = torch.tensor([ms64], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms64 = float(t.item())
        s64 = g64.stats()
        if ref is not None:
            accuracy["fp64"] = error_stats(out64, idx_t, ref)
            accuracy["acc_rms_ratio"] = accuracy[args.precision]["acc_rms"] / accuracy["fp64"]["acc_rms"]
        fp64 = {"value": world * n * args.steps / (ms64 * 1e-3), "ms_per_eval": ms64 / args.steps,
                "judge_rms_acc_err": s64["judge_rms"], "note": "force evaluations only (no kick/drift)"}
        g64.close()

    # ---- end to end through the public API: pinned host state in, results out, every step
    e2e = None
    if not args.no_e2e:
        hin = {k: st[k].to("cpu").pin_memory() for k in st}
        hout = {k: torch.empty(n, dtype=torch.float64).pin_memory() for k in out}
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
    m2l_flops = stats["n_m2l"] * m2l_flops_per_pair(p, True)
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
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
                "data": "synthetic (seeded Plummer sphere, Kroupa IMF masses)",
                "config": workload_config(n, p, world),
                "form": {"precision": args.precision,
                         "evaluation": "one CUDA graph replay" if g.graph_ready() else "direct launches"},
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
