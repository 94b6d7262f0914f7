"""CPU oracle for the FMM gravity evaluation -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this
package, and only as the checker / the timed CPU baseline.  The product
(``taichi_collisional_b200``) never imports it.

Two independent CPU implementations sit behind it:

* ``liboracle.so`` -- ``tc_oracle.c``, a plain-C FP64 restatement of the reference's
  theta-MAC force evaluation (tree build, Miniball centres, P2M/M2M, dual traversal,
  rotation M2L, L2L/L2P, P2P with jerks) plus an FP64 direct sum;
* ``_ref/libtcref_<tree>_p<P>_<isa>.so`` -- the reference's own headers compiled behind
  ``ref_harness.cpp`` (built here by ``oracle/Makefile``; the reference sources are not
  part of this repository).  These pin the restatement and give the "reference" CPU
  baseline.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
VARIANT_TOP, VARIANT_JERKS = 0, 1

_lib = None
_ref_libs = {}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_u8p = C.POINTER(C.c_ubyte)


class Params(C.Structure):
    _fields_ = [("p", C.c_int), ("ncrit", C.c_int), ("variant", C.c_int), ("use_shift", C.c_int),
                ("theta", C.c_double), ("shift_u", C.c_double * 3), ("direct_below", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("n_cells", C.c_longlong), ("n_leaves", C.c_longlong), ("n_m2l", C.c_longlong),
                ("n_p2p", C.c_longlong), ("n_p2p_inter", C.c_longlong), ("max_level", C.c_int)]


def _d(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def reference_dir():
    """The reference source tree: $TC_REFERENCE, else a `reference` directory beside the
    repository checkout; None when neither holds the reference's exafmm.h (the GPU host has
    only the prebuilt oracle/_ref libraries)."""
    cands = [os.environ.get("TC_REFERENCE"), os.path.join(HERE, "..", "..", "reference")]
    for c in cands:
        if c and os.path.isfile(os.path.join(c, "exafmm.h")):
            return os.path.abspath(c)
    return None


def build():
    """Compile liboracle.so (and, when the reference tree is present, oracle/_ref)."""
    subprocess.check_call(["make", "-s", "-C", HERE, "oracle"])
    if reference_dir():
        ref = "REF=" + reference_dir()
        subprocess.check_call(["make", "-s", "-j8", "-C", HERE, "ref", ref])
        # the reference's integrator over this repository's force evaluation needs the CUDA library
        if os.path.exists(os.path.join(HERE, "..", "taichi_collisional_b200", "libtaichi_b200.so")):
            subprocess.check_call(["make", "-s", "-j2", "-C", HERE, "ref-shim", ref])


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.check_call(["make", "-s", "-C", HERE, "oracle"])
        L = C.CDLL(path)
        L.tco_evaluate.argtypes = [C.POINTER(Params), C.c_int] + [_dp] * 7 + [_u8p] + [_dp] * 7 + [C.POINTER(Stats)]
        L.tco_evaluate.restype = C.c_int
        L.tco_evaluate_steps.argtypes = [C.POINTER(Params), C.c_double, C.c_int] + [_dp] * 7 + [_u8p] + [_dp] * 5 + \
            [C.POINTER(Stats)]
        L.tco_evaluate_steps.restype = C.c_int
        L.tco_last_ncell.restype = C.c_int
        L.tco_last_cells.argtypes = [_ip] * 5 + [_dp, _dp, _ip]
        L.tco_last_expansions.argtypes = [_dp] * 4
        L.tco_last_list.argtypes = [C.c_int, _ip, _ip]
        L.tco_last_list.restype = C.c_longlong
        L.tco_direct.argtypes = [C.c_int] + [_dp] * 7 + [C.c_int, _ip] + [_dp] * 7
        L.tco_init.argtypes = [C.c_int]
        L.tco_system_diagnostics.argtypes = [C.c_int] + [_dp] * 9
        L.tco_drift_compsum.argtypes = [C.c_int, _dp, _dp, _dp, C.c_double]
        L.tco_make_gnm.argtypes = [_dp, _dp, _dp, C.c_int]
        L.tco_swap_xz.argtypes = [_dp, C.c_int]
        L.tco_p2m.argtypes = [C.c_int, C.c_int] + [_dp] * 10
        L.tco_m2m.argtypes = [C.c_int] + [_dp] * 5
        L.tco_m2l_rotate.argtypes = [C.c_int] + [_dp] * 5
        L.tco_m2l_direct.argtypes = [C.c_int] + [_dp] * 3
        L.tco_l2l.argtypes = [C.c_int] + [_dp] * 5
        L.tco_l2p.argtypes = [C.c_int] + [_dp] * 5
        L.tco_miniball.argtypes = [C.c_int, _dp, _dp, _dp]
        L.tco_miniball.restype = C.c_int
        _lib = L
    return _lib


def evaluate(x, y, z, m, vx=None, vy=None, vz=None, *, p, theta, ncrit, variant=VARIANT_JERKS,
             shift_u=None, direct_below=0, flags=None):
    """Oracle force evaluation; returns dict(ax, ay, az, pot, jx, jy, jz, stats)."""
    L = lib()
    n = len(x)
    x, y, z, m = map(_f64, (x, y, z, m))
    vx, vy, vz = map(_f64, (vx, vy, vz))
    prm = Params(p=p, ncrit=ncrit, variant=variant, use_shift=int(shift_u is not None),
                 theta=theta, direct_below=direct_below)
    if shift_u is not None:
        for d in range(3):
            prm.shift_u[d] = float(shift_u[d])
    out = {k: np.zeros(n) for k in ("ax", "ay", "az", "pot", "jx", "jy", "jz")}
    st = Stats()
    fl = None if flags is None else np.ascontiguousarray(flags, dtype=np.uint8)
    rc = L.tco_evaluate(C.byref(prm), n, _d(x), _d(y), _d(z), _d(vx), _d(vy), _d(vz), _d(m),
                        None if fl is None else fl.ctypes.data_as(_u8p),
                        *[_d(out[k]) for k in ("ax", "ay", "az", "pot", "jx", "jy", "jz")], C.byref(st))
    if rc != 0:
        raise RuntimeError("oracle evaluate failed (%d)" % rc)
    out["stats"] = {f: getattr(st, f) for f, _ in Stats._fields_}
    return out


def evaluate_steps(x, y, z, m, vx, vy, vz, *, p, theta, ncrit, dt_param, flags=None):
    """Oracle time-step pass of the top-level tree (get_steps = true); returns dict(ax, ay,
    az, pot, timestep, stats), timestep = each body's sum of 1 / tau^4."""
    L = lib()
    n = len(x)
    x, y, z, m = map(_f64, (x, y, z, m))
    vx, vy, vz = map(_f64, (vx, vy, vz))
    prm = Params(p=p, ncrit=ncrit, variant=VARIANT_TOP, use_shift=0, theta=theta, direct_below=0)
    out = {k: np.zeros(n) for k in ("ax", "ay", "az", "pot", "timestep")}
    st = Stats()
    fl = None if flags is None else np.ascontiguousarray(flags, dtype=np.uint8)
    rc = L.tco_evaluate_steps(C.byref(prm), dt_param, n, _d(x), _d(y), _d(z), _d(vx), _d(vy), _d(vz), _d(m),
                              None if fl is None else fl.ctypes.data_as(_u8p),
                              *[_d(out[k]) for k in ("ax", "ay", "az", "pot", "timestep")], C.byref(st))
    if rc != 0:
        raise RuntimeError("oracle evaluate_steps failed (%d)" % rc)
    out["stats"] = {f: getattr(st, f) for f, _ in Stats._fields_}
    return out


def last_cells():
    L = lib()
    nc = L.tco_last_ncell()
    a = {k: np.zeros(nc, dtype=np.int32) for k in ("begin", "nbody", "nchild", "child", "level")}
    X = np.zeros((nc, 3))
    R = np.zeros(nc)
    L.tco_last_cells(*[a[k].ctypes.data_as(_ip) for k in ("begin", "nbody", "nchild", "child", "level")],
                     _d(X), _d(R), None)
    n = int(a["nbody"][0]) if nc else 0
    perm = np.zeros(n, dtype=np.int32)
    L.tco_last_cells(*[a[k].ctypes.data_as(_ip) for k in ("begin", "nbody", "nchild", "child", "level")],
                     _d(X), _d(R), perm.ctypes.data_as(_ip))
    a["X"], a["R"], a["perm"] = X, R, perm
    return a


def last_lists():
    L = lib()
    out = {}
    for kind, name in ((0, "m2l"), (1, "p2p")):
        cnt = L.tco_last_list(kind, None, None)
        t = np.zeros(cnt, dtype=np.int32)
        s = np.zeros(cnt, dtype=np.int32)
        L.tco_last_list(kind, t.ctypes.data_as(_ip), s.ctypes.data_as(_ip))
        out[name] = (t, s)
    return out


def direct(x, y, z, m, vx=None, vy=None, vz=None, targets=None):
    """FP64 direct summation at the given target indices (default: all)."""
    L = lib()
    n = len(x)
    x, y, z, m = map(_f64, (x, y, z, m))
    vx, vy, vz = map(_f64, (vx, vy, vz))
    tg = None if targets is None else np.ascontiguousarray(targets, dtype=np.int32)
    nt = n if tg is None else len(tg)
    out = {k: np.zeros(nt) for k in ("ax", "ay", "az", "pot", "jx", "jy", "jz")}
    L.tco_direct(n, _d(x), _d(y), _d(z), _d(vx), _d(vy), _d(vz), _d(m), nt,
                 None if tg is None else tg.ctypes.data_as(_ip),
                 *[_d(out[k]) for k in ("ax", "ay", "az", "pot", "jx", "jy", "jz")])
    return out


DIAG_KEYS = ("kinetic", "potential", "mass", "cm_pos", "cm_vel")


def _diag_dict(out):
    return {"kinetic": out[0], "potential": out[1], "mass": out[2], "cm_pos": tuple(out[3:6]),
            "cm_vel": tuple(out[6:9])}


def system_diagnostics(m, x, y, z, vx, vy, vz, pot):
    """The reference's system_kinetic_energy / system_potential_energy / system_center_of_mass
    (integrator.h:887-925), restated in C with long-double sums (tco_system_diagnostics)."""
    out = np.zeros(9)
    a = [_f64(v) for v in (m, x, y, z, vx, vy, vz, pot)]
    lib().tco_system_diagnostics(len(a[0]), *[_d(v) for v in a], _d(out))
    return _diag_dict(out)


def drift_compsum(s, e, v, dt):
    """drift with COMPSUM (integrator.h:42, :642-656) on one axis; returns new (s, e)."""
    s = np.array(s, dtype=np.float64)
    e = np.array(e, dtype=np.float64)
    v = _f64(v)
    lib().tco_drift_compsum(len(s), _d(s), _d(e), _d(v), float(dt))
    return s, e


def split_order(ts, dt):
    """The reference's split(dt, s, &slow, &fast) (integrator.h:591-640), restated: the order the
    bodies end in (ids) and the number of fast bodies.  Two pointers walk in from both ends and
    swap a slow body (timestep >= |dt|) found on the left with a fast one (timestep < |dt|)
    found on the right, so the k-th slow body inside the final fast prefix swaps with the k-th
    fast body, counted from the right, inside the final slow suffix; a single fast body is
    reported as none (fast.n = 1 -> 0)."""
    ts = np.asarray(ts, dtype=np.float64)
    n = len(ts)
    dt = abs(dt)
    fast = ts < dt
    nf = int(fast.sum())
    perm = np.arange(n)
    left = np.nonzero(~fast[:nf])[0]               # slow bodies in the fast prefix, left to right
    right = nf + np.nonzero(fast[nf:])[0][::-1]    # fast bodies in the slow suffix, right to left
    perm[left], perm[right] = right, left
    return perm, (0 if nf == 1 else nf)


# ----------------------------------------------------------------------------------------
# The reference's own code (oracle/_ref)
# ----------------------------------------------------------------------------------------
def _isa():
    try:
        with open("/proc/cpuinfo") as f:
            flags = f.read()
        return "avx512" if " avx512f " in flags and " avx512dq " in flags else "avx2"
    except OSError:
        return "avx2"


def ref_path(variant, p):
    tree = "jerks" if variant == VARIANT_JERKS else "top"
    return os.path.join(HERE, "_ref", "libtcref_%s_p%d_%s.so" % (tree, p, _isa()))


def ref_available(variant, p):
    return os.path.exists(ref_path(variant, p))


def ref_lib(variant, p):
    key = (variant, p)
    if key not in _ref_libs:
        L = C.CDLL(ref_path(variant, p))
        L.tcr_evaluate.argtypes = [C.c_int] + [_dp] * 7 + [_u8p, C.c_double, C.c_int, C.c_long, C.c_int] + [_dp] * 8
        L.tcr_evaluate.restype = C.c_int
        L.tcr_cells.argtypes = [_ip] * 4 + [_dp, _dp, _ip]
        L.tcr_expansions.argtypes = [_dp, _dp]
        L.tcr_list.argtypes = [C.c_int, _ip, _ip]
        L.tcr_list.restype = C.c_longlong
        L.tcr_shift_uniforms.argtypes = [C.c_long, _dp]
        if hasattr(L, "tcr_evaluate_high_jerks"):
            L.tcr_evaluate_high_jerks.argtypes = [C.c_int] + [_dp] * 7 + [_u8p, C.c_double, C.c_int, C.c_long,
                                                                          C.c_int] + [_dp] * 7
            L.tcr_evaluate_high_jerks.restype = C.c_int
            L.tcr_acc_old.argtypes = [_dp]
            L.tcr_min_acc.argtypes = [_dp, _dp]
        if hasattr(L, "tcr_evaluate_high"):
            L.tcr_evaluate_high.argtypes = [C.c_int] + [_dp] * 7 + [_u8p, C.c_double, C.c_int, C.c_int] + [_dp] * 4
            L.tcr_evaluate_high.restype = C.c_int
            L.tcr_evaluate_high_steps.argtypes = [C.c_int] + [_dp] * 7 + [_u8p, C.c_double, C.c_int, C.c_double,
                                                                          C.c_int] + [_dp] * 5
            L.tcr_evaluate_high_steps.restype = C.c_int
            L.tcr_acc_old.argtypes = [_dp]
            L.tcr_min_acc.argtypes = [_dp, _dp]
        if hasattr(L, "tcr_evaluate_steps"):
            L.tcr_evaluate_steps.argtypes = [C.c_int] + [_dp] * 7 + [_u8p, C.c_double, C.c_int, C.c_double,
                                                                     C.c_int] + [_dp] * 5
            L.tcr_evaluate_steps.restype = C.c_int
        _ref_libs[key] = L
    return _ref_libs[key]


def ref_shift_uniforms(variant, p, seed):
    u = np.zeros(3)
    ref_lib(variant, p).tcr_shift_uniforms(seed, _d(u))
    return u


def ref_evaluate(x, y, z, m, vx=None, vy=None, vz=None, *, p, theta, ncrit, variant=VARIANT_JERKS,
                 seed=1, nthreads=1, flags=None):
    """The reference's own theta-MAC evaluation.  nthreads=1 gives reproducible sums."""
    L = ref_lib(variant, p)
    n = len(x)
    x, y, z, m = map(_f64, (x, y, z, m))
    vx, vy, vz = map(_f64, (vx, vy, vz))
    out = {k: np.zeros(n) for k in ("ax", "ay", "az", "pot", "jx", "jy", "jz")}
    times = np.zeros(4)
    fl = None if flags is None else np.ascontiguousarray(flags, dtype=np.uint8)
    nc = L.tcr_evaluate(n, _d(x), _d(y), _d(z), _d(vx), _d(vy), _d(vz), _d(m),
                        None if fl is None else fl.ctypes.data_as(_u8p), theta, ncrit, seed, nthreads,
                        *[_d(out[k]) for k in ("ax", "ay", "az", "pot", "jx", "jy", "jz")], _d(times))
    out["ncell"] = nc
    out["times"] = times
    return out


def ref_evaluate_steps(x, y, z, m, vx, vy, vz, *, p, theta, ncrit, dt_param, nthreads=1, flags=None):
    """The reference's own time-step pass (top-level tree, horizontalPass with get_steps)."""
    L = ref_lib(VARIANT_TOP, p)
    n = len(x)
    x, y, z, m = map(_f64, (x, y, z, m))
    vx, vy, vz = map(_f64, (vx, vy, vz))
    out = {k: np.zeros(n) for k in ("ax", "ay", "az", "pot", "timestep")}
    fl = None if flags is None else np.ascontiguousarray(flags, dtype=np.uint8)
    nc = L.tcr_evaluate_steps(n, _d(x), _d(y), _d(z), _d(vx), _d(vy), _d(vz), _d(m),
                              None if fl is None else fl.ctypes.data_as(_u8p), theta, ncrit, dt_param, nthreads,
                              *[_d(out[k]) for k in ("ax", "ay", "az", "pot", "timestep")])
    out["ncell"] = nc
    return out


def ref_evaluate_high(x, y, z, m, *, p, ncrit, force_accuracy, nthreads=1, flags=None):
    """The top tree's own get_force_and_potential (integrator.h:459-562): low-order pre-pass,
    then the error-controlled MAC.  Also returns the pre-pass's per-body acc_old (caller order)
    and the per-cell min_acc and Pn of the reference's cells."""
    L = ref_lib(VARIANT_TOP, p)
    n = len(x)
    x, y, z, m = map(_f64, (x, y, z, m))
    out = {k: np.zeros(n) for k in ("ax", "ay", "az", "pot")}
    fl = None if flags is None else np.ascontiguousarray(flags, dtype=np.uint8)
    nc = L.tcr_evaluate_high(n, _d(x), _d(y), _d(z), None, None, None, _d(m),
                             None if fl is None else fl.ctypes.data_as(_u8p), force_accuracy, ncrit, nthreads,
                             *[_d(out[k]) for k in ("ax", "ay", "az", "pot")])
    out["ncell"] = nc
    out["acc_old"] = np.zeros(n)
    L.tcr_acc_old(_d(out["acc_old"]))
    out["min_acc"] = np.zeros(nc)
    out["pn"] = np.zeros((nc, p + 1))
    L.tcr_min_acc(_d(out["min_acc"]), _d(out["pn"]))
    return out


def ref_evaluate_high_jerks(x, y, z, m, vx, vy, vz, *, p, ncrit, force_accuracy, seed=1, nthreads=1, flags=None):
    """The jerks tree's own get_force_and_potential (taichi_with_jerks/integrator.h:308-432,
    without its direct branch): low-order pre-pass, then its one-sided error-controlled MAC.
    Returns the outputs, acc_old (caller order), per-cell min_acc and Pn."""
    L = ref_lib(VARIANT_JERKS, p)
    n = len(x)
    x, y, z, m = map(_f64, (x, y, z, m))
    vx, vy, vz = map(_f64, (vx, vy, vz))
    out = {k: np.zeros(n) for k in ("ax", "ay", "az", "pot", "jx", "jy", "jz")}
    fl = None if flags is None else np.ascontiguousarray(flags, dtype=np.uint8)
    nc = L.tcr_evaluate_high_jerks(n, _d(x), _d(y), _d(z), _d(vx), _d(vy), _d(vz), _d(m),
                                   None if fl is None else fl.ctypes.data_as(_u8p), force_accuracy, ncrit, seed,
                                   nthreads, *[_d(out[k]) for k in ("ax", "ay", "az", "pot", "jx", "jy", "jz")])
    out["ncell"] = nc
    out["acc_old"] = np.zeros(n)
    L.tcr_acc_old(_d(out["acc_old"]))
    out["min_acc"] = np.zeros(nc)
    out["pn"] = np.zeros((nc, p + 1))
    L.tcr_min_acc(_d(out["min_acc"]), _d(out["pn"]))
    return out


def ref_evaluate_high_steps(x, y, z, m, vx, vy, vz, *, p, ncrit, force_accuracy, dt_param, nthreads=1, flags=None):
    """The top tree's own get_force_and_potential(bodies, true): pre-pass, error-controlled MAC,
    time-step pass (near-field pot / acc and per-body sum of 1 / tau^4)."""
    L = ref_lib(VARIANT_TOP, p)
    n = len(x)
    x, y, z, m = map(_f64, (x, y, z, m))
    vx, vy, vz = map(_f64, (vx, vy, vz))
    out = {k: np.zeros(n) for k in ("ax", "ay", "az", "pot", "timestep")}
    fl = None if flags is None else np.ascontiguousarray(flags, dtype=np.uint8)
    nc = L.tcr_evaluate_high_steps(n, _d(x), _d(y), _d(z), _d(vx), _d(vy), _d(vz), _d(m),
                                   None if fl is None else fl.ctypes.data_as(_u8p), force_accuracy, ncrit, dt_param,
                                   nthreads, *[_d(out[k]) for k in ("ax", "ay", "az", "pot", "timestep")])
    out["ncell"] = nc
    out["acc_old"] = np.zeros(n)
    L.tcr_acc_old(_d(out["acc_old"]))
    return out


def ref_cells(variant, p, ncell, n):
    L = ref_lib(variant, p)
    a = {k: np.zeros(ncell, dtype=np.int32) for k in ("begin", "nbody", "nchild", "child")}
    X = np.zeros((ncell, 3))
    R = np.zeros(ncell)
    idx = np.zeros(n, dtype=np.int32)
    L.tcr_cells(*[a[k].ctypes.data_as(_ip) for k in ("begin", "nbody", "nchild", "child")], _d(X), _d(R),
                idx.ctypes.data_as(_ip))
    a["X"], a["R"], a["index"] = X, R, idx
    return a


def ref_lists(variant, p):
    L = ref_lib(variant, p)
    out = {}
    for kind, name in ((0, "m2l"), (1, "p2p")):
        cnt = L.tcr_list(kind, None, None)
        t = np.zeros(cnt, dtype=np.int32)
        s = np.zeros(cnt, dtype=np.int32)
        L.tcr_list(kind, t.ctypes.data_as(_ip), s.ctypes.data_as(_ip))
        out[name] = (t, s)
    return out


def integ_ref_path():
    return os.path.join(HERE, "_ref", "libtcref_integ_%s.so" % _isa())


def integ_ref_available():
    return os.path.exists(integ_ref_path())


def _integ_ref():
    key = "integ"
    if key not in _ref_libs:
        L = C.CDLL(integ_ref_path())
        L.tcr_system_diagnostics.argtypes = [C.c_int] + [_dp] * 9
        L.tcr_drift.argtypes = [C.c_int] + [_dp] * 9 + [C.c_double]
        L.tcr_split.argtypes = [C.c_int, _dp, C.c_double, _ip]
        L.tcr_split.restype = C.c_int
        _ref_libs[key] = L
    return _ref_libs[key]


def ref_system_diagnostics(m, x, y, z, vx, vy, vz, pot):
    """The reference's own diagnostics (oracle/_ref/libtcref_integ_*)."""
    out = np.zeros(9)
    a = [_f64(v) for v in (m, x, y, z, vx, vy, vz, pot)]
    _integ_ref().tcr_system_diagnostics(len(a[0]), *[_d(v) for v in a], _d(out))
    return _diag_dict(out)


def ref_drift(x, y, z, ex, ey, ez, vx, vy, vz, dt):
    """The reference's own drift (COMPSUM); returns new (x, y, z, ex, ey, ez)."""
    st = [np.array(a, dtype=np.float64) for a in (x, y, z, ex, ey, ez)]
    v = [_f64(a) for a in (vx, vy, vz)]
    _integ_ref().tcr_drift(len(st[0]), *[_d(a) for a in st], *[_d(a) for a in v], float(dt))
    return tuple(st)


def ref_split(ts, dt):
    """The reference's own split: (order of ids, fast.n)."""
    ts = _f64(ts)
    perm = np.zeros(len(ts), dtype=np.int32)
    nf = _integ_ref().tcr_split(len(ts), _d(ts), float(dt), perm.ctypes.data_as(_ip))
    return perm, nf


def integ_shim_path(gradient=False):
    return os.path.join(HERE, "_ref", "libtcref_integ_shim_%s%s.so" % ("grad_" if gradient else "", _isa()))


def _evolve_lib(shim, gradient=False):
    key = ("integ_shim_grad" if gradient else "integ_shim") if shim else "integ"
    if shim and key not in _ref_libs:
        _ref_libs[key] = C.CDLL(integ_shim_path(gradient))
    L = _ref_libs[key] if shim else _integ_ref()
    L.tcr_evolve_hold.argtypes = [C.c_int] + [_dp] * 12 + [_ip, C.c_int, C.c_double, C.c_double, C.c_double,
                                                           C.c_double]
    L.tcr_evolve_hold.restype = C.c_double
    return L


EVOLVE_KEYS = ("x", "y", "z", "ex", "ey", "ez", "vx", "vy", "vz", "m", "timestep", "pot")


def ref_evolve_hold(state, *, ncrit, theta, force_accuracy, dt_param, dt, shim=False):
    """One do_evolve step of the reference's HOLD scheme (evolve_split_hold_dkd) on a dict of
    arrays (EVOLVE_KEYS + "id"), with the reference's own force evaluation (p = 8), or -- shim=True
    -- with this repository's, through the C++ shim.  Returns (new state, simtime)."""
    st = {k: np.array(state[k], dtype=np.float64) for k in EVOLVE_KEYS}
    st["id"] = np.array(state["id"], dtype=np.int32)
    L = _evolve_lib(shim)
    t = L.tcr_evolve_hold(len(st["x"]), *[_d(st[k]) for k in EVOLVE_KEYS], st["id"].ctypes.data_as(_ip), ncrit,
                          theta, force_accuracy, dt_param, dt)
    return st, t


def ref_evolve_gradient(state, *, ncrit, theta, force_accuracy, dt_param, dt):
    """One do_evolve step of the reference's force-gradient scheme (evolve_split_omelyan, its
    GRADIENT / OUTPUTACC build) over this repository's force evaluation through the C++ shim.
    Returns (new state, simtime)."""
    st = {k: np.array(state[k], dtype=np.float64) for k in EVOLVE_KEYS}
    st["id"] = np.array(state["id"], dtype=np.int32)
    L = _evolve_lib(True, gradient=True)
    t = L.tcr_evolve_hold(len(st["x"]), *[_d(st[k]) for k in EVOLVE_KEYS], st["id"].ctypes.data_as(_ip), ncrit,
                          theta, force_accuracy, dt_param, dt)
    return st, t
