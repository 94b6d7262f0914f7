#!/usr/bin/env python3
"""Generate the golden fixtures from the reference's own code (oracle/_ref).

Run from the repository root, where the reference tree is available and
``make -C oracle ref`` has built the harness libraries:

    python tests/golden/make_golden.py

Each case stores its inputs, the reference's per-body outputs (single-threaded, so the
sums are reproducible), the reference's cells (begin, nbody, nchild, child, centre,
radius) and its M2L / P2P lists as visited by the reference recursion.  The steps_* cases
store the time-step pass of the top-level tree (get_steps = true): near-field pot / acc and
each body's accumulated 1 / tau^4, with a sink / source subset.  The emac_* cases store the
top tree's own get_force_and_potential: the low-order pre-pass (acc_old per body, min_acc per
cell) and the error-controlled MAC's lists and forces; the emac_jerks_* cases the same for the
jerks tree (its order-2 pre-pass with the FP32 vector near field, its one-sided MAC, and the
jerks).  The integ_* case stores the
reference integrator's diagnostics (kinetic / potential energy, centre of mass), three
compensated drifts and one split by time step.  The evolve_* case stores one do_evolve step
of the reference's HOLD block-time-step scheme with its own force evaluation (p = 8).

    python tests/golden/make_golden.py [--emac-jerks-only | --evolve-only | --integ-only | --emac-only |
                                        --steps-only]
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from taichi_collisional_b200 import ics  # noqa: E402

CASES = [
    # name, variant, generator, n, seed, p, theta, ncrit, shift seed
    ("top_plummer1k_p8", oracle.VARIANT_TOP, "plummer", 1024, 11, 8, 0.5, 32, 0),
    ("jerks_plummer1k_p8", oracle.VARIANT_JERKS, "plummer", 1024, 12, 8, 0.5, 32, 5),
    ("jerks_kroupa1500_p10", oracle.VARIANT_JERKS, "plummer_kroupa", 1500, 13, 10, 0.4, 32, 7),
    ("top_kroupa1500_p12", oracle.VARIANT_TOP, "plummer_kroupa", 1500, 14, 12, 0.4, 24, 0),
]


STEPS_CASES = [
    # name, generator, n, seed, p, theta, ncrit, dt_param, flags pattern
    ("steps_top_kroupa2k_p8", "plummer_kroupa", 2000, 21, 8, 0.5, 32, 0.025, True),
    ("steps_top_plummer40_p8", "plummer", 40, 22, 8, 0.5, 64, 0.01, False),
]


EMAC_CASES = [
    # name, generator, n, seed, p, ncrit, force_accuracy  (top tree, error-controlled MAC)
    ("emac_top_kroupa3k_p8", "plummer_kroupa", 3000, 31, 8, 32, 2.0e-7),
    ("emac_top_plummer2k_p12", "plummer", 2000, 32, 12, 64, 1.0e-8),
]


EMAC_JERKS_CASES = [
    # name, generator, n, seed, p, ncrit, force_accuracy, shift seed  (jerks tree, error-controlled MAC)
    ("emac_jerks_kroupa3k_p8", "plummer_kroupa", 3000, 51, 8, 32, 2.0e-8, 9),
    ("emac_jerks_plummer2k_p12", "plummer", 2000, 52, 12, 64, 2.0e-8, 10),
]


def make_emac_jerks(out_dir):
    """The jerks tree's own get_force_and_potential (low-order pre-pass, one-sided error MAC)."""
    for name, gen, n, seed, p, ncrit, fa, sseed in EMAC_JERKS_CASES:
        x, y, z, vx, vy, vz, m = getattr(ics, gen)(n, seed)
        r = oracle.ref_evaluate_high_jerks(x, y, z, m, vx, vy, vz, p=p, ncrit=ncrit, force_accuracy=fa, seed=sseed)
        cells = oracle.ref_cells(oracle.VARIANT_JERKS, p, r["ncell"], n)
        lists = oracle.ref_lists(oracle.VARIANT_JERKS, p)
        shift = oracle.ref_shift_uniforms(oracle.VARIANT_JERKS, p, sseed)
        np.savez_compressed(
            os.path.join(out_dir, name + ".npz"), p=p, ncrit=ncrit, force_accuracy=fa, shift_u=shift,
            x=x, y=y, z=z, vx=vx, vy=vy, vz=vz, m=m, ax=r["ax"], ay=r["ay"], az=r["az"], pot=r["pot"],
            jx=r["jx"], jy=r["jy"], jz=r["jz"], acc_old=r["acc_old"], min_acc=r["min_acc"],
            cell_begin=cells["begin"], cell_nbody=cells["nbody"], cell_nchild=cells["nchild"],
            cell_child=cells["child"], cell_X=cells["X"], cell_R=cells["R"],
            m2l_t=lists["m2l"][0], m2l_s=lists["m2l"][1], p2p_t=lists["p2p"][0], p2p_s=lists["p2p"][1])
        print(name, "cells", r["ncell"], "m2l", len(lists["m2l"][0]), "p2p", len(lists["p2p"][0]))


def make_emac(out_dir):
    for name, gen, n, seed, p, ncrit, fa in EMAC_CASES:
        x, y, z, vx, vy, vz, m = getattr(ics, gen)(n, seed)
        r = oracle.ref_evaluate_high(x, y, z, m, p=p, ncrit=ncrit, force_accuracy=fa)
        cells = oracle.ref_cells(oracle.VARIANT_TOP, p, r["ncell"], n)
        lists = oracle.ref_lists(oracle.VARIANT_TOP, p)
        np.savez_compressed(
            os.path.join(out_dir, name + ".npz"), p=p, ncrit=ncrit, force_accuracy=fa,
            x=x, y=y, z=z, m=m, ax=r["ax"], ay=r["ay"], az=r["az"], pot=r["pot"], acc_old=r["acc_old"],
            min_acc=r["min_acc"], cell_begin=cells["begin"], cell_nbody=cells["nbody"],
            cell_nchild=cells["nchild"], cell_child=cells["child"], cell_X=cells["X"], cell_R=cells["R"],
            m2l_t=lists["m2l"][0], m2l_s=lists["m2l"][1], p2p_t=lists["p2p"][0], p2p_s=lists["p2p"][1])
        print(name, "cells", r["ncell"], "m2l", len(lists["m2l"][0]), "p2p", len(lists["p2p"][0]))
    # the time-step pass through the error-controlled MAC, with a sink / source subset
    name, n, seed, p, ncrit, fa, dtp = "emac_steps_top_kroupa2k_p8", 2000, 33, 8, 32, 2.0e-7, 0.025
    x, y, z, vx, vy, vz, m = ics.plummer_kroupa(n, seed)
    fl = steps_flags(n)
    r = oracle.ref_evaluate_high_steps(x, y, z, m, vx, vy, vz, p=p, ncrit=ncrit, force_accuracy=fa, dt_param=dtp,
                                       flags=fl)
    np.savez_compressed(
        os.path.join(out_dir, name + ".npz"), p=p, ncrit=ncrit, force_accuracy=fa, dt_param=dtp,
        x=x, y=y, z=z, vx=vx, vy=vy, vz=vz, m=m, flags=fl, ax=r["ax"], ay=r["ay"], az=r["az"], pot=r["pot"],
        timestep=r["timestep"], acc_old=r["acc_old"])
    print(name, "cells", r["ncell"])


def steps_flags(n):
    """every third body a sink only, every fifth (from 1) a source only, the rest both"""
    fl = np.full(n, 3, np.uint8)
    fl[::3] = 1
    fl[1::5] = 2
    return fl


def make_steps(out_dir):
    for name, gen, n, seed, p, theta, ncrit, dtp, use_flags in STEPS_CASES:
        x, y, z, vx, vy, vz, m = getattr(ics, gen)(n, seed)
        fl = steps_flags(n) if use_flags else np.full(n, 3, np.uint8)
        r = oracle.ref_evaluate_steps(x, y, z, m, vx, vy, vz, p=p, theta=theta, ncrit=ncrit, dt_param=dtp,
                                      flags=fl)
        np.savez_compressed(
            os.path.join(out_dir, name + ".npz"), p=p, theta=theta, ncrit=ncrit, dt_param=dtp,
            x=x, y=y, z=z, vx=vx, vy=vy, vz=vz, m=m, flags=fl,
            ax=r["ax"], ay=r["ay"], az=r["az"], pot=r["pot"], timestep=r["timestep"])
        print(name, "cells", r["ncell"])


INTEG_CASE = ("integ_plummer_kroupa2k", "plummer_kroupa", 2048, 31, 1.0 / 64)


def make_integ(out_dir):
    name, gen, n, seed, dt = INTEG_CASE
    x, y, z, vx, vy, vz, m = getattr(ics, gen)(n, seed)
    pot = oracle.direct(x, y, z, m)["pot"]
    d = oracle.ref_system_diagnostics(m, x, y, z, vx, vy, vz, pot)
    diag = np.array([d["kinetic"], d["potential"], d["mass"], *d["cm_pos"], *d["cm_vel"]])
    st = (x, y, z, np.zeros(n), np.zeros(n), np.zeros(n))
    for _ in range(3):
        st = oracle.ref_drift(*st, vx, vy, vz, dt)
    # block time steps 2^-k (k = 3..9) from the body's speed, so the split has ties with dt
    speed = np.sqrt(vx * vx + vy * vy + vz * vz)
    ts = 2.0 ** -np.clip(np.round(3 + 6 * speed / speed.max()), 3, 9)
    perm, nf = oracle.ref_split(ts, dt)
    np.savez_compressed(os.path.join(out_dir, name + ".npz"), dt=dt, x=x, y=y, z=z, vx=vx, vy=vy, vz=vz, m=m,
                        pot=pot, diag=diag, drift_x=st[0], drift_y=st[1], drift_z=st[2], drift_ex=st[3],
                        drift_ey=st[4], drift_ez=st[5], ts=ts, split_perm=perm, split_nfast=nf)
    print(name, "kinetic", d["kinetic"], "potential", d["potential"], "fast", nf)


EVOLVE_CASE = ("evolve_hold_plummer_kroupa1k", "plummer_kroupa", 1024, 41, 64, 0.4, 2e-7, 0.025, 1.0 / 64)


def evolve_initial_state(gen, n, seed):
    x, y, z, vx, vy, vz, m = getattr(ics, gen)(n, seed)
    zero = np.zeros(n)
    return dict(x=x, y=y, z=z, vx=vx, vy=vy, vz=vz, m=m, ex=zero, ey=zero, ez=zero, timestep=zero, pot=zero,
                id=np.arange(n, dtype=np.int32))


def make_evolve(out_dir):
    name, gen, n, seed, nc, th, fa, dtp, dt = EVOLVE_CASE
    st0 = evolve_initial_state(gen, n, seed)
    st, simtime = oracle.ref_evolve_hold(st0, ncrit=nc, theta=th, force_accuracy=fa, dt_param=dtp, dt=dt)
    np.savez_compressed(os.path.join(out_dir, name + ".npz"), gen=gen, n=n, seed=seed, ncrit=nc, theta=th,
                        force_accuracy=fa, dt_param=dtp, dt=dt, simtime=simtime,
                        **{"out_" + k: v for k, v in st.items()})
    print(name, "simtime", simtime)


def main():
    out_dir = os.path.dirname(os.path.abspath(__file__))
    make_emac_jerks(out_dir)
    if "--emac-jerks-only" in sys.argv:
        return
    make_evolve(out_dir)
    if "--evolve-only" in sys.argv:
        return
    make_integ(out_dir)
    if "--integ-only" in sys.argv:
        return
    make_emac(out_dir)
    if "--emac-only" in sys.argv:
        return
    make_steps(out_dir)
    if "--steps-only" in sys.argv:
        return
    for name, variant, gen, n, seed, p, theta, ncrit, sseed in CASES:
        x, y, z, vx, vy, vz, m = getattr(ics, gen)(n, seed)
        r = oracle.ref_evaluate(x, y, z, m, vx, vy, vz, p=p, theta=theta, ncrit=ncrit, variant=variant,
                                seed=sseed, nthreads=1)
        cells = oracle.ref_cells(variant, p, r["ncell"], n)
        lists = oracle.ref_lists(variant, p)
        shift = oracle.ref_shift_uniforms(variant, p, sseed) if variant == oracle.VARIANT_JERKS else np.full(3, np.nan)
        np.savez_compressed(
            os.path.join(out_dir, name + ".npz"),
            variant=variant, p=p, theta=theta, ncrit=ncrit, shift_u=shift,
            x=x, y=y, z=z, vx=vx, vy=vy, vz=vz, m=m,
            ax=r["ax"], ay=r["ay"], az=r["az"], pot=r["pot"], jx=r["jx"], jy=r["jy"], jz=r["jz"],
            cell_begin=cells["begin"], cell_nbody=cells["nbody"], cell_nchild=cells["nchild"],
            cell_child=cells["child"], cell_X=cells["X"], cell_R=cells["R"], body_index=cells["index"],
            m2l_t=lists["m2l"][0], m2l_s=lists["m2l"][1], p2p_t=lists["p2p"][0], p2p_s=lists["p2p"][1])
        print(name, "cells", r["ncell"], "m2l", len(lists["m2l"][0]), "p2p", len(lists["p2p"][0]))


if __name__ == "__main__":
    main()
