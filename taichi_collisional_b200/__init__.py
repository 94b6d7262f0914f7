"""taichi_collisional_b200 -- B200-native FMM gravity evaluation.

Python view of the C ABI in ``include/taichi_b200.h`` (``libtaichi_b200.so``, built in-tree
by ``taichi_collisional_b200.build``).  The entry point mirrors the reference's force
evaluation ``get_force_and_potential(Bodies&, bool)`` (integrator.h:459-562,
taichi_with_jerks/integrator.h:308-432): it takes positions, masses (and velocities for the
jerks tree) and returns acceleration, potential (p = +sum m/r) and jerk for every sink body,
in the caller's order.

There is no CPU fallback: if the CUDA library cannot be loaded the calls raise.
"""
import ctypes as C
import os

import numpy as np

from . import ics  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtaichi_b200.so")

VARIANT_TOP, VARIANT_JERKS = 0, 1
PREC_FP64, PREC_MIXED, PREC_MIXED_M2L = 0, 1, 2
MEM_HOST, MEM_DEVICE = 0, 1

STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "capacity exceeded", 4: "non-finite input",
          5: "tree depth limit reached", 6: "unsupported option", 7: "device-side wait timed out"}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_u8p = C.POINTER(C.c_ubyte)


class Params(C.Structure):
    _fields_ = [("p", C.c_int), ("ncrit", C.c_int), ("theta", C.c_double), ("variant", C.c_int),
                ("precision", C.c_int), ("use_shift", C.c_int), ("shift_u", C.c_double * 3),
                ("direct_below", C.c_int), ("device", C.c_int), ("selector", C.c_int),
                ("selector_tol", C.c_double), ("judge_n", C.c_int), ("judge_tol", C.c_double),
                ("judge_seed", C.c_ulonglong), ("softening", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("n_bodies", C.c_longlong), ("n_cells", C.c_longlong), ("n_leaves", C.c_longlong),
                ("n_m2l", C.c_longlong), ("n_p2p", C.c_longlong), ("n_p2p_inter", C.c_longlong),
                ("max_level", C.c_int), ("ms_total", C.c_double), ("ms_tree", C.c_double),
                ("ms_upward", C.c_double), ("ms_traverse", C.c_double), ("ms_m2l", C.c_double),
                ("ms_p2p", C.c_double), ("ms_downward", C.c_double), ("n_launches", C.c_longlong),
                ("flags", C.c_longlong), ("n_classes", C.c_int), ("class_order", C.c_int * 16),
                ("class_pairs", C.c_longlong * 16), ("m2l_flop_fraction", C.c_double), ("judge_rms", C.c_double),
                ("judge_redo", C.c_int)]


class TrainReport(C.Structure):
    _fields_ = [("samples", C.c_int), ("iters", C.c_int), ("n_classes", C.c_int), ("class_order", C.c_int * 6),
                ("train_loss", C.c_double), ("val_loss", C.c_double), ("seconds", C.c_double)]


EXPORTS = ["tc_default_params", "tc_create", "tc_destroy", "tc_set_stream", "tc_evaluate", "tc_get_stats",
           "tc_get_cells", "tc_get_lists", "tc_get_expansions", "tc_status_string", "tc_last_error_string",
           "tc_pmax", "tc_order_supported", "tc_kick_drift", "tc_probe_peak", "tc_evaluate_direct_noalloc",
           "tc_train_selector", "tc_get_selector_data", "tc_selector_nparam", "tc_get_selector_weights",
           "tc_set_selector_weights", "tc_mlp_loss_grad", "tc_mlp_predict", "tc_set_selector", "tc_tc_bins", "tc_direct_sums", "tc_evaluate_steps", "tc_set_graph", "tc_graph_ready", "tc_graph_note", "tc_set_error_mac", "tc_get_acc_old", "tc_hermite_predict", "tc_hermite_correct",
           "tc_system_diagnostics", "tc_drift_compensated", "tc_split_order", "tc_evolve_hold_dkd", "tc_evolve_omelyan", "tc_step_leapfrog",
           "tc_set_wait_limit"]
NOALLOC_MAX_N = 16384

_lib = None


class TaichiError(RuntimeError):
    pass


def load_library(path=LIB_PATH):
    """Load the CUDA library (raises if it is missing; there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise TaichiError("libtaichi_b200.so not built: run `python -m taichi_collisional_b200.build`")
    L = C.CDLL(path)
    L.tc_default_params.argtypes = [C.POINTER(Params)]
    L.tc_create.argtypes = [C.POINTER(Params), C.POINTER(C.c_void_p)]
    L.tc_create.restype = C.c_int
    L.tc_destroy.argtypes = [C.c_void_p]
    L.tc_destroy.restype = C.c_int
    L.tc_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    L.tc_set_stream.restype = C.c_int
    L.tc_set_graph.argtypes = [C.c_void_p, C.c_int]
    L.tc_set_graph.restype = C.c_int
    L.tc_graph_ready.argtypes = [C.c_void_p]
    L.tc_graph_ready.restype = C.c_int
    L.tc_graph_note.argtypes = [C.c_void_p]
    L.tc_graph_note.restype = C.c_char_p
    L.tc_hermite_predict.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 13 + [C.c_double]
    L.tc_hermite_predict.restype = C.c_int
    L.tc_hermite_correct.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 13 + [C.c_double]
    L.tc_hermite_correct.restype = C.c_int
    L.tc_set_wait_limit.argtypes = [C.c_void_p, C.c_longlong]
    L.tc_set_wait_limit.restype = C.c_int
    L.tc_step_leapfrog.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 14 + [C.c_double]
    L.tc_step_leapfrog.restype = C.c_int
    L.tc_set_error_mac.argtypes = [C.c_void_p, C.c_int, C.c_double]
    L.tc_set_error_mac.restype = C.c_int
    L.tc_get_acc_old.argtypes = [C.c_void_p, _dp]
    L.tc_get_acc_old.restype = C.c_int
    L.tc_evaluate.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 8 + [C.c_void_p] * 7 + [C.c_int]
    L.tc_evaluate.restype = C.c_int
    L.tc_get_stats.argtypes = [C.c_void_p, C.POINTER(Stats)]
    L.tc_get_stats.restype = C.c_int
    L.tc_get_cells.argtypes = [C.c_void_p] + [_ip] * 5 + [_dp, _dp, _ip]
    L.tc_get_cells.restype = C.c_int
    L.tc_get_lists.argtypes = [C.c_void_p, C.c_int, _ip, _ip]
    L.tc_get_lists.restype = C.c_int
    L.tc_get_expansions.argtypes = [C.c_void_p] + [_dp] * 4
    L.tc_get_expansions.restype = C.c_int
    L.tc_status_string.argtypes = [C.c_int]
    L.tc_status_string.restype = C.c_char_p
    L.tc_last_error_string.argtypes = [C.c_void_p]
    L.tc_last_error_string.restype = C.c_char_p
    L.tc_pmax.restype = C.c_int
    L.tc_order_supported.argtypes = [C.c_int]
    L.tc_order_supported.restype = C.c_int
    L.tc_kick_drift.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 9 + [C.c_double, C.c_double]
    L.tc_kick_drift.restype = C.c_int
    L.tc_system_diagnostics.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 8 + [C.POINTER(C.c_double)]
    L.tc_system_diagnostics.restype = C.c_int
    L.tc_drift_compensated.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 9 + [C.c_double]
    L.tc_drift_compensated.restype = C.c_int
    L.tc_split_order.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_double, C.c_void_p, C.POINTER(C.c_int)]
    L.tc_split_order.restype = C.c_int
    L.tc_evolve_hold_dkd.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 13 + [C.c_double, C.c_double,
                                                                                 C.POINTER(EvolveStats)]
    L.tc_evolve_hold_dkd.restype = C.c_int
    L.tc_evolve_omelyan.argtypes = L.tc_evolve_hold_dkd.argtypes
    L.tc_evolve_omelyan.restype = C.c_int
    L.tc_probe_peak.argtypes = [C.c_void_p, C.c_int]
    L.tc_probe_peak.restype = C.c_double
    L.tc_evaluate_direct_noalloc.argtypes = [C.c_int] + [C.c_void_p] * 8 + [C.c_void_p] * 7 + [C.c_int, C.c_void_p]
    L.tc_evaluate_direct_noalloc.restype = C.c_int
    _fp = C.POINTER(C.c_float)
    L.tc_train_selector.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 7 + [C.c_int, C.c_int, C.c_int,
                                                                               C.c_ulonglong, C.POINTER(TrainReport)]
    L.tc_train_selector.restype = C.c_int
    L.tc_get_selector_data.argtypes = [C.c_void_p, _fp, _fp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.tc_get_selector_data.restype = C.c_int
    L.tc_selector_nparam.argtypes = [C.c_void_p]
    L.tc_selector_nparam.restype = C.c_int
    L.tc_get_selector_weights.argtypes = [C.c_void_p, _fp, _fp]
    L.tc_get_selector_weights.restype = C.c_int
    L.tc_set_selector_weights.argtypes = [C.c_void_p, _fp, _fp]
    L.tc_set_selector_weights.restype = C.c_int
    L.tc_mlp_loss_grad.argtypes = [C.c_int, C.c_int, _fp, _fp, _fp, _fp, _fp, _fp]
    L.tc_mlp_loss_grad.restype = C.c_int
    L.tc_mlp_predict.argtypes = [C.c_int, C.c_int, _fp, _fp, _fp, _fp]
    L.tc_mlp_predict.restype = C.c_int
    L.tc_set_selector.argtypes = [C.c_void_p, C.c_int, C.c_double]
    L.tc_set_selector.restype = C.c_int
    L.tc_tc_bins.argtypes = [C.c_int, _fp, C.c_int]
    L.tc_tc_bins.restype = C.c_int
    L.tc_direct_sums.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 8 + [C.c_int, _ip, _dp, C.c_int]
    L.tc_direct_sums.restype = C.c_int
    L.tc_evaluate_steps.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 8 + [C.c_double] + [C.c_void_p] * 5 + \
        [C.c_int]
    L.tc_evaluate_steps.restype = C.c_int
    _lib = L
    return L


def default_params(**kw):
    L = load_library()
    prm = Params()
    L.tc_default_params(C.byref(prm))
    for k, v in kw.items():
        if k == "shift_u":
            if v is None:
                prm.use_shift = 0
            else:
                prm.use_shift = 1
                for d in range(3):
                    prm.shift_u[d] = float(v[d])
        else:
            setattr(prm, k, v)
    return prm


class EvolveStats(C.Structure):
    _fields_ = [("n_evaluations", C.c_int), ("n_direct", C.c_int), ("n_splits", C.c_int), ("max_level", C.c_int),
                ("simtime", C.c_double)]


EVOLVE_KEYS = ("x", "y", "z", "ex", "ey", "ez", "vx", "vy", "vz", "m", "timestep", "pot")


def _ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):  # torch tensor
        return C.c_void_p(a.data_ptr())
    return C.c_void_p(a.ctypes.data)


class Gravity:
    """A force-evaluation context (tc_create ... tc_destroy).

    ``evaluate`` is the replacement of ``get_force_and_potential(bodies, false)``.
    Inputs are numpy float64 arrays (host) or CUDA float64 torch tensors (device).
    """

    def __init__(self, p=12, ncrit=64, theta=0.4, variant=VARIANT_JERKS, precision=PREC_FP64, shift_u=None,
                 direct_below=-1, device=0, selector=0, selector_tol=1e-9, judge_n=0, judge_tol=0.0,
                 judge_seed=12345, softening=0.0):
        self._L = load_library()
        self.params = default_params(p=p, ncrit=ncrit, theta=theta, variant=variant, precision=precision,
                                     shift_u=shift_u, direct_below=direct_below, device=device, selector=selector,
                                     selector_tol=selector_tol, judge_n=judge_n, judge_tol=judge_tol,
                                     judge_seed=judge_seed, softening=softening)
        h = C.c_void_p()
        rc = self._L.tc_create(C.byref(self.params), C.byref(h))
        if rc != 0:
            raise TaichiError("tc_create failed: %s" % STATUS.get(rc, rc))
        self._h = h
        self.jerk = variant == VARIANT_JERKS

    def close(self):
        if getattr(self, "_h", None):
            self._L.tc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr):
        self._L.tc_set_stream(self._h, C.c_void_p(stream_ptr))

    def set_graph(self, on=True):
        """Run evaluate as one captured CUDA graph (tc_set_graph): the first call with a given set
        of buffers runs normally and captures; matching calls replay.  Host buffers must be
        pinned to be captured."""
        self._check(self._L.tc_set_graph(self._h, 1 if on else 0), "tc_set_graph")

    def graph_ready(self):
        """True when the next evaluate with the same buffers replays the captured graph."""
        return bool(self._L.tc_graph_ready(self._h))

    def set_error_mac(self, on=True, force_accuracy=2.0e-7):
        """The top tree's error-controlled MAC with the reference's low-order pre-pass
        (tc_set_error_mac)."""
        self._check(self._L.tc_set_error_mac(self._h, 1 if on else 0, force_accuracy), "tc_set_error_mac")

    def acc_old(self):
        """The pre-pass's per-body acceleration estimate of the last evaluation (caller order)."""
        a = np.zeros(int(self.stats()["n_bodies"]))
        self._check(self._L.tc_get_acc_old(self._h, a.ctypes.data_as(_dp)), "tc_get_acc_old")
        return a

    def graph_note(self):
        """Why the last capture was abandoned ('' when it succeeded)."""
        return self._L.tc_graph_note(self._h).decode()

    def _check(self, rc, what):
        if rc != 0:
            msg = self._L.tc_last_error_string(self._h).decode()
            raise TaichiError("%s: %s %s" % (what, STATUS.get(rc, rc), msg))

    def evaluate(self, x, y, z, m, vx=None, vy=None, vz=None, flags=None, out=None):
        """Returns dict ax, ay, az, pot (and jx, jy, jz with jerks) in the caller's order."""
        n = len(x)
        dev = hasattr(x, "data_ptr")
        if out is None:
            if dev:
                import torch
                out = {k: torch.empty(n, dtype=torch.float64, device=x.device) for k in
                       (("ax", "ay", "az", "pot", "jx", "jy", "jz") if self.jerk else ("ax", "ay", "az", "pot"))}
            else:
                out = {k: np.zeros(n) for k in
                       (("ax", "ay", "az", "pot", "jx", "jy", "jz") if self.jerk else ("ax", "ay", "az", "pot"))}
        if not dev:
            x, y, z, m = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, m))
            if vx is not None:
                vx, vy, vz = (np.ascontiguousarray(a, dtype=np.float64) for a in (vx, vy, vz))
            if flags is not None:
                flags = np.ascontiguousarray(flags, dtype=np.uint8)
        rc = self._L.tc_evaluate(self._h, n, _ptr(x), _ptr(y), _ptr(z), _ptr(vx), _ptr(vy), _ptr(vz), _ptr(m),
                                 _ptr(flags), _ptr(out["ax"]), _ptr(out["ay"]), _ptr(out["az"]), _ptr(out["pot"]),
                                 _ptr(out.get("jx")), _ptr(out.get("jy")), _ptr(out.get("jz")),
                                 MEM_DEVICE if dev else MEM_HOST)
        self._check(rc, "tc_evaluate")
        return out

    def evaluate_steps(self, x, y, z, m, vx, vy, vz, dt_param, flags=None):
        """The time-step pass of the top-level tree (get_force_and_potential(bodies, true)):
        dict ax, ay, az, pot (near field only, as in the reference) and timestep (each body's
        sum of 1 / tau^4), numpy or CUDA tensors like the inputs."""
        n = len(x)
        dev = hasattr(x, "data_ptr")
        if dev:
            import torch
            out = {k: torch.empty(n, dtype=torch.float64, device=x.device) for k in ("ax", "ay", "az", "pot", "timestep")}
        else:
            out = {k: np.zeros(n) for k in ("ax", "ay", "az", "pot", "timestep")}
            x, y, z, m, vx, vy, vz = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, m, vx, vy, vz))
            if flags is not None:
                flags = np.ascontiguousarray(flags, dtype=np.uint8)
        rc = self._L.tc_evaluate_steps(self._h, n, _ptr(x), _ptr(y), _ptr(z), _ptr(vx), _ptr(vy), _ptr(vz), _ptr(m),
                                       _ptr(flags), float(dt_param), _ptr(out["ax"]), _ptr(out["ay"]),
                                       _ptr(out["az"]), _ptr(out["pot"]), _ptr(out["timestep"]),
                                       MEM_DEVICE if dev else MEM_HOST)
        self._check(rc, "tc_evaluate_steps")
        return out

    def direct_sums(self, x, y, z, m, targets, vx=None, vy=None, vz=None, flags=None):
        """FP64 direct sums at the bodies `targets` (caller indices) over all bodies: a dict of
        pot, ax, ay, az, jx, jy, jz arrays (numpy), one entry per target.  Inputs are numpy
        (host) or CUDA torch tensors (device); used for accuracy statements."""
        n = len(x)
        dev = hasattr(x, "data_ptr")
        if not dev:
            x, y, z, m = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, m))
            if vx is not None:
                vx, vy, vz = (np.ascontiguousarray(a, dtype=np.float64) for a in (vx, vy, vz))
            if flags is not None:
                flags = np.ascontiguousarray(flags, dtype=np.uint8)
        t = np.ascontiguousarray(targets, dtype=np.int32)
        out = np.zeros((len(t), 7))
        rc = self._L.tc_direct_sums(self._h, n, _ptr(x), _ptr(y), _ptr(z), _ptr(vx), _ptr(vy), _ptr(vz), _ptr(m),
                                    _ptr(flags), len(t), t.ctypes.data_as(_ip), out.ctypes.data_as(_dp),
                                    MEM_DEVICE if dev else MEM_HOST)
        self._check(rc, "tc_direct_sums")
        return {k: out[:, i].copy() for i, k in enumerate(("pot", "ax", "ay", "az", "jx", "jy", "jz"))}

    def set_wait_limit(self, cycles):
        """Clock-cycle limit of the bounded device waits (tc_set_wait_limit; <= 0: default)."""
        self._check(self._L.tc_set_wait_limit(self._h, int(cycles)), "tc_set_wait_limit")

    def step_leapfrog(self, st, out, dt):
        """One kick-drift-kick step on CUDA tensors (tc_step_leapfrog): st holds x, y, z, vx, vy,
        vz, m; out holds ax, ay, az (the previous accelerations on entry), pot (and jx, jy, jz).
        With set_graph(True) the whole step replays as one CUDA graph."""
        rc = self._L.tc_step_leapfrog(self._h, len(st["x"]), *[_ptr(st[k]) for k in ("x", "y", "z", "vx", "vy", "vz",
                                                                                      "m")],
                                      *[_ptr(out.get(k)) for k in ("ax", "ay", "az", "pot", "jx", "jy", "jz")],
                                      float(dt))
        self._check(rc, "tc_step_leapfrog")

    def kick_drift(self, x, y, z, vx, vy, vz, ax, ay, az, dt_kick, dt_drift):
        """FP64 leapfrog update on CUDA tensors: v += a dt_kick; x += v dt_drift."""
        rc = self._L.tc_kick_drift(self._h, len(x), *[_ptr(a) for a in (x, y, z, vx, vy, vz, ax, ay, az)],
                                   float(dt_kick), float(dt_drift))
        self._check(rc, "tc_kick_drift")

    def system_diagnostics(self, m, x, y, z, vx, vy, vz, pot):
        """Kinetic and potential energy, total mass, centre of mass and its velocity of CUDA
        float64 tensors (tc_system_diagnostics; the reference's system_kinetic_energy,
        system_potential_energy, system_center_of_mass).  Returns a dict of floats."""
        out = (C.c_double * 9)()
        rc = self._L.tc_system_diagnostics(self._h, len(m), *[_ptr(a) for a in (m, x, y, z, vx, vy, vz, pot)], out)
        self._check(rc, "tc_system_diagnostics")
        return {"kinetic": out[0], "potential": out[1], "mass": out[2], "cm_pos": tuple(out[3:6]),
                "cm_vel": tuple(out[6:9])}

    def drift_compensated(self, x, y, z, ex, ey, ez, vx, vy, vz, dt):
        """Compensated drift x += v dt with running errors ex, ey, ez (tc_drift_compensated;
        the reference's drift with COMPSUM)."""
        rc = self._L.tc_drift_compensated(self._h, len(x), *[_ptr(a) for a in (x, y, z, ex, ey, ez, vx, vy, vz)],
                                          float(dt))
        self._check(rc, "tc_drift_compensated")

    def split_order(self, timestep, dt):
        """The reference's split by time step as a permutation (tc_split_order) of a CUDA float64
        tensor: returns (perm, nfast), perm an int32 CUDA tensor."""
        import torch
        perm = torch.empty(len(timestep), dtype=torch.int32, device=timestep.device)
        nf = C.c_int(0)
        rc = self._L.tc_split_order(self._h, len(timestep), _ptr(timestep), float(dt), _ptr(perm), C.byref(nf))
        self._check(rc, "tc_split_order")
        return perm, nf.value

    def evolve_hold_dkd(self, state, dt_param, dt):
        """One step dt of the reference's HOLD block-time-step scheme (tc_evolve_hold_dkd) on a
        dict of CUDA tensors: float64 EVOLVE_KEYS and int32 "id", permuted in place.  Returns the
        step's counts as a dict."""
        st = EvolveStats()
        rc = self._L.tc_evolve_hold_dkd(self._h, len(state["x"]), *[_ptr(state[k]) for k in EVOLVE_KEYS],
                                        _ptr(state["id"]), float(dt_param), float(dt), C.byref(st))
        self._check(rc, "tc_evolve_hold_dkd")
        return {k: getattr(st, k) for k, _ in EvolveStats._fields_}

    def evolve_omelyan(self, state, dt_param, dt):
        """One step dt of the reference's default force-gradient scheme (tc_evolve_omelyan), as
        evolve_hold_dkd."""
        st = EvolveStats()
        rc = self._L.tc_evolve_omelyan(self._h, len(state["x"]), *[_ptr(state[k]) for k in EVOLVE_KEYS],
                                       _ptr(state["id"]), float(dt_param), float(dt), C.byref(st))
        self._check(rc, "tc_evolve_omelyan")
        return {k: getattr(st, k) for k, _ in EvolveStats._fields_}

    def hermite_predict(self, x, y, z, vx, vy, vz, a, save, dt):
        """Hermite 4th-order predictor on CUDA tensors (tc_hermite_predict); `a` is the dict of
        ax, ay, az, jx, jy, jz at t, `save` a CUDA float64 tensor of 12 n."""
        rc = self._L.tc_hermite_predict(self._h, len(x), *[_ptr(v) for v in (x, y, z, vx, vy, vz)],
                                        *[_ptr(a[k]) for k in ("ax", "ay", "az", "jx", "jy", "jz")], _ptr(save),
                                        float(dt))
        self._check(rc, "tc_hermite_predict")

    def hermite_correct(self, x, y, z, vx, vy, vz, a, save, dt):
        """Hermite 4th-order corrector with a (ax..jz) evaluated at the predicted state."""
        rc = self._L.tc_hermite_correct(self._h, len(x), *[_ptr(v) for v in (x, y, z, vx, vy, vz)],
                                        *[_ptr(a[k]) for k in ("ax", "ay", "az", "jx", "jy", "jz")], _ptr(save),
                                        float(dt))
        self._check(rc, "tc_hermite_correct")

    def probe_peak(self, kind):
        """Measured FMA throughput of this GPU in GFLOP/s (0: FP64, 1: FP32)."""
        return self._L.tc_probe_peak(self._h, kind)

    def train_selector(self, x, y, z, m, vx=None, vy=None, vz=None, nsamples=16384, iters=2000, seed=1):
        """Fit the learned order selector on pairs of this input (tc_train_selector)."""
        dev = hasattr(x, "data_ptr")
        if not dev:
            x, y, z, m = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, m))
            if vx is not None:
                vx, vy, vz = (np.ascontiguousarray(a, dtype=np.float64) for a in (vx, vy, vz))
        rep = TrainReport()
        rc = self._L.tc_train_selector(self._h, len(x), _ptr(x), _ptr(y), _ptr(z), _ptr(vx), _ptr(vy), _ptr(vz),
                                       _ptr(m), MEM_DEVICE if dev else MEM_HOST, int(nsamples), int(iters),
                                       int(seed), C.byref(rep))
        self._check(rc, "tc_train_selector")
        out = {f: getattr(rep, f) for f, _ in TrainReport._fields_}
        out["class_order"] = list(rep.class_order)[:rep.n_classes]
        return out

    def selector_data(self):
        n, nc = C.c_int(), C.c_int()
        self._L.tc_get_selector_data(self._h, None, None, C.byref(n), C.byref(nc))
        f = np.zeros((n.value, 8), dtype=np.float32)
        lab = np.zeros((n.value, nc.value), dtype=np.float32)
        fp = C.POINTER(C.c_float)
        self._L.tc_get_selector_data(self._h, f.ctypes.data_as(fp), lab.ctypes.data_as(fp), C.byref(n), C.byref(nc))
        return f, lab

    def selector_weights(self):
        npar = self._L.tc_selector_nparam(self._h)
        w = np.zeros(npar, dtype=np.float32)
        norm = np.zeros(17, dtype=np.float32)
        fp = C.POINTER(C.c_float)
        self._check(self._L.tc_get_selector_weights(self._h, w.ctypes.data_as(fp), norm.ctypes.data_as(fp)),
                    "tc_get_selector_weights")
        return w, norm

    def set_selector_weights(self, w, norm):
        fp = C.POINTER(C.c_float)
        w = np.ascontiguousarray(w, dtype=np.float32)
        norm = np.ascontiguousarray(norm, dtype=np.float32)
        self._check(self._L.tc_set_selector_weights(self._h, w.ctypes.data_as(fp), norm.ctypes.data_as(fp)),
                    "tc_set_selector_weights")

    def set_selector(self, selector, tol):
        """Switch the far-field order selector of this context (0 fixed, 1 analytic, 2 learned)."""
        self._check(self._L.tc_set_selector(self._h, int(selector), float(tol)), "tc_set_selector")
        self.params.selector = selector
        self.params.selector_tol = tol

    def stats(self):
        st = Stats()
        self._L.tc_get_stats(self._h, C.byref(st))
        out = {f: getattr(st, f) for f, _ in Stats._fields_}
        out["class_order"] = list(st.class_order)[:st.n_classes]
        out["class_pairs"] = list(st.class_pairs)[:st.n_classes]
        return out

    def cells(self):
        st = self.stats()
        nc, n = int(st["n_cells"]), int(st["n_bodies"])
        a = {k: np.zeros(nc, dtype=np.int32) for k in ("begin", "nbody", "nchild", "child", "level")}
        X = np.zeros((nc, 3))
        R = np.zeros(nc)
        perm = np.zeros(n, dtype=np.int32)
        rc = self._L.tc_get_cells(self._h, *[a[k].ctypes.data_as(_ip) for k in ("begin", "nbody", "nchild", "child",
                                                                                  "level")],
                                  X.ctypes.data_as(_dp), R.ctypes.data_as(_dp), perm.ctypes.data_as(_ip))
        self._check(rc, "tc_get_cells")
        a["X"], a["R"], a["perm"] = X, R, perm
        return a

    def lists(self):
        st = self.stats()
        out = {}
        for kind, name, cnt in ((0, "m2l", st["n_m2l"]), (1, "p2p", st["n_p2p"])):
            t = np.zeros(cnt, dtype=np.int32)
            s = np.zeros(cnt, dtype=np.int32)
            rc = self._L.tc_get_lists(self._h, kind, t.ctypes.data_as(_ip), s.ctypes.data_as(_ip))
            self._check(rc, "tc_get_lists")
            out[name] = (t, s)
        return out

    def expansions(self):
        st = self.stats()
        nt = (self.params.p + 1) ** 2
        nc = int(st["n_cells"])
        M, L = np.zeros((nc, nt)), np.zeros((nc, nt))
        Md = np.zeros((nc, nt)) if self.jerk else None
        Ld = np.zeros((nc, nt)) if self.jerk else None
        rc = self._L.tc_get_expansions(self._h, M.ctypes.data_as(_dp), None if Md is None else Md.ctypes.data_as(_dp),
                                       L.ctypes.data_as(_dp), None if Ld is None else Ld.ctypes.data_as(_dp))
        self._check(rc, "tc_get_expansions")
        return M, Md, L, Ld


def tc_bins(q):
    """Constant matrices of the tensor-core far field at order q: (hi, lo) arrays of shape
    (bins, 256) in the kernel's layout (see include/taichi_b200.h, tc_tc_bins)."""
    L = load_library()
    n = L.tc_tc_bins(q, None, 0)
    if n < 0:
        raise TaichiError("no tensor-core plan for order %d" % q)
    buf = np.zeros(n, dtype=np.float32)
    L.tc_tc_bins(q, buf.ctypes.data_as(C.POINTER(C.c_float)), n)
    return buf[: n // 2].reshape(-1, 256), buf[n // 2:].reshape(-1, 256)


def evaluate_direct_noalloc(x, y, z, m, vx=None, vy=None, vz=None, flags=None, out=None, stream=0):
    """Direct sum without any device allocation by the library (tc_evaluate_direct_noalloc).

    For callers that cannot allocate device memory; CUDA float64 tensors in and out, at most
    NOALLOC_MAX_N bodies.  The library's working storage is a fixed static device array, so
    calls that overlap on the GPU race.  Returns the output dict (queued on ``stream``)."""
    import torch
    L = load_library()
    n = len(x)
    jerk = vx is not None
    if out is None:
        keys = ("ax", "ay", "az", "pot", "jx", "jy", "jz") if jerk else ("ax", "ay", "az", "pot")
        out = {k: torch.empty(n, dtype=torch.float64, device=x.device) for k in keys}
    rc = L.tc_evaluate_direct_noalloc(n, _ptr(x), _ptr(y), _ptr(z), _ptr(vx), _ptr(vy), _ptr(vz), _ptr(m),
                                      _ptr(flags), _ptr(out["ax"]), _ptr(out["ay"]), _ptr(out["az"]),
                                      _ptr(out["pot"]), _ptr(out.get("jx")), _ptr(out.get("jy")),
                                      _ptr(out.get("jz")), int(jerk), C.c_void_p(stream))
    if rc != 0:
        raise TaichiError("tc_evaluate_direct_noalloc: %s" % STATUS.get(rc, rc))
    return out


def get_force_and_potential(x, y, z, m, vx=None, vy=None, vz=None, flags=None, **params):
    """One-shot helper: create a context, evaluate, destroy."""
    g = Gravity(**params)
    try:
        return g.evaluate(x, y, z, m, vx, vy, vz, flags)
    finally:
        g.close()
