"""ctypes binding of the C ABI declared in include/qv.h (libqvort_b200.so).

This is the Python face of the same entry points the Fortran driver binds
through ISO_C_BINDING.  Arrays cross as numpy buffers: positions and
velocities (n, 3) float64 C-contiguous (= Fortran x(3,n)), links (n,) int32
with 1-based indices and 0 for an empty slot.  A failing call raises
QvError carrying the status code and qv_last_error()'s message.

There is no fallback: importing this module loads the CUDA library, and a
missing or unloadable library raises at import time.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libqvort_b200.so"

QV_OK = 0
QV_ERR_ARG = -1
QV_ERR_CUDA = -2
QV_ERR_SINGULAR = -3
QV_ERR_TREE_DEPTH = -4
QV_ERR_STATE = -5
QV_ERR_NOMEM = -6
QV_ERR_UNSUPPORTED = -7
QV_ERR_NAN = -8
QV_ERR_NOALLOC_LIMIT = -9
QV_NOALLOC_MAX_POINTS = 16384
QV_MAX_DEPTH = 64

BC = {"open": 0, "periodic": 1, "openx": 2, "openxy": 3}
VELOCITY = {"Off": 0, "LIA": 1, "BS": 2, "Tree": 3}
PREC = {"fp64": 0, "mixed": 1}


class QvParams(C.Structure):
    _fields_ = [
        ("quant_circ", C.c_double),
        ("corea", C.c_double),
        ("box_size", C.c_double),
        ("delta", C.c_double),
        ("dt", C.c_double),
        ("tree_theta", C.c_double),
        ("boundary", C.c_int),
        ("velocity", C.c_int),
        ("deriv_order", C.c_int),
        ("tree_extra_correction", C.c_int),
        ("fixed_lia_beta", C.c_int),
        ("precision", C.c_int),
        ("runge_kutta", C.c_int),
        ("recon_shots", C.c_int),
        ("line_ops", C.c_int),
    ]


class QvRun(C.Structure):
    _fields_ = [
        ("p", QvParams),
        ("nsteps", C.c_int),
        ("shots", C.c_int),
        ("pcount", C.c_int),
        ("readin_var_file", C.c_int),
        ("switch_off_recon", C.c_int),
        ("initf", C.c_char * 32),
    ]


class QvState(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("x", "u", "u1", "u2", "u3", "infront", "behind",
                                          "closest", "closestd")]


class QvRestart(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("x", "u", "u1", "u2", "u3", "u_li", "u_bs", "gi", "gb",
                                          "gii", "gbb", "closestd", "infront", "behind",
                                          "closest")]


RESTART_VEC = ("x", "u", "u1", "u2", "u3", "u_li", "u_bs", "gi", "gb", "gii", "gbb")
RESTART_INT = ("infront", "behind", "closest")


class QvError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"qv error {code}: {msg}")
        self.code = code


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is not built; run `python -m qvort_b200.build` (nvcc, sm_100a)")
    return C.CDLL(str(LIB_PATH))


_lib = _load()

_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)

_SIGS = {
    "qv_default_params": [C.POINTER(QvParams)],
    "qv_create": [C.POINTER(QvParams), _P, C.POINTER(_P)],
    "qv_destroy": [_P],
    "qv_set_params": [_P, C.POINTER(QvParams)],
    "qv_set_points": [_P, C.c_int, _P, _P, _P],
    "qv_set_points_device": [_P, C.c_int, _P, _P, _P],
    "qv_set_history": [_P, _P, _P, _P],
    "qv_get_history": [_P, _P, _P, _P],
    "qv_set_closest": [_P, _P],
    "qv_get_points": [_P, _P, _P],
    "qv_get_closest": [_P, _P, _P],
    "qv_device_arrays": [_P, _P, _P, _P, _P],
    "qv_ghosts": [_P],
    "qv_get_ghosts": [_P, _P, _P, _P, _P],
    "qv_build_tree": [_P],
    "qv_tree_info": [_P, _I, _I],
    "qv_tree_export": [_P, C.c_int, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    "qv_velocity": [_P, _P, _P, _P, C.POINTER(C.c_longlong)],
    "qv_step_ab": [_P],
    "qv_step_rk3": [_P],
    "qv_enforce_periodic": [_P],
    "qv_closest": [_P, _P, _P],
    "qv_energy": [_P, _D],
    "qv_step": [_P, C.c_int],
    "qv_set_state": [_P, C.c_int, C.POINTER(QvState)],
    "qv_get_state": [_P, C.c_int, C.POINTER(QvState), _I],
    "qv_step_exchange": [_P, C.c_int, C.c_int, C.POINTER(QvState), C.c_int, C.POINTER(QvState), _I],
    "qv_steps": [_P, C.c_int, C.c_int],
    "qv_sync": [_P],
    "qv_profile": [_P, C.c_int],
    "qv_phase_times": [_P, _P, C.c_int],
    "qv_counters": [_P, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                    C.POINTER(C.c_longlong)],
    "qv_probe_fp32": [_P, _D],
    "qv_test_stage_timeout": [C.c_int],
    "qv_test_root_speculation": [C.c_int, C.c_double],
    "qv_test_late_level1": [C.c_int],
    "qv_root_undecided": [_P, _I],
    "qv_velocity_direct_noalloc": [C.POINTER(QvParams), C.c_int, _P, _P, _P, _P, _P],
    "qv_velocity_device": [_P, _P],
    "qv_velocity_vjp": [_P, _P, _P],
    "qv_energy_grad": [_P, _P, _D, _P, _P],
    "qv_ab_step_device": [_P, C.c_int, _P, _P, _P, _P, _P, _P],
    "qv_ab_vjp_device": [_P, C.c_int, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    "qv_field_velocity": [_P, C.c_int, _P, C.c_int, _P, _P],
    "qv_field_velocity_tree": [_P, C.c_int, _P, _P, C.POINTER(C.c_longlong)],
    "qv_read_run_file": [C.c_char_p, C.POINTER(QvRun)],
    "qv_read_var_file": [C.c_char_p, C.c_int, _I, _D, _P, _P, _P],
    "qv_write_var_file": [C.c_char_p, C.c_int, C.c_double, _P, _P, _P],
    "qv_write_restart_file": [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_double, _P],
    "qv_read_restart_file": [C.c_char_p, C.c_int, _I, _I, _I, _D, _P],
    "qv_dump": [_P, C.c_char_p, C.c_int, C.c_int, C.c_double],
    "qv_restore": [_P, C.c_char_p, _I, _I, _D],
    "qv_write_snapshot": [_P, C.c_char_p, C.c_double],
    "qv_setup_loops": [C.c_char_p, C.c_int, C.c_double, _P, _P, _P],
    "qv_pinsert": [_P, _I],
    "qv_premove": [_P, _I],
    "qv_point_count": [_P, _I],
    "qv_precon": [_P, _I],
    "qv_get_links": [_P, _P, _P],
    "qv_batch_create": [C.POINTER(QvParams), C.c_int, _P, _P, _P, _P, C.POINTER(_P)],
    "qv_batch_set_points": [_P, _P, _P, _P],
    "qv_batch_velocity": [_P, _P],
    "qv_batch_step": [_P, C.c_int],
    "qv_batch_get_points": [_P, _P, _P],
    "qv_batch_tune": [_P, C.c_int, _P, C.POINTER(C.c_float)],
    "qv_batch_set_config": [_P, C.c_int, C.c_int, C.c_int],
    "qv_batch_stats": [_P, _P, _I, _P],
}
for _name, _args in _SIGS.items():
    _f = getattr(_lib, _name)
    _f.argtypes = _args
    _f.restype = C.c_int
_lib.qv_last_error.argtypes = [_P]
_lib.qv_last_error.restype = C.c_char_p
_lib.qv_batch_last_error.argtypes = [_P]
_lib.qv_batch_last_error.restype = C.c_char_p
_lib.qv_batch_destroy.argtypes = [_P]
_lib.qv_batch_destroy.restype = None

EXPORTED = tuple(_SIGS) + ("qv_last_error", "qv_batch_last_error", "qv_batch_destroy")


def lib() -> C.CDLL:
    return _lib


def default_params(**kw) -> QvParams:
    p = QvParams()
    _lib.qv_default_params(C.byref(p))
    for k, v in kw.items():
        if k == "boundary" and isinstance(v, str):
            v = BC[v]
        elif k == "velocity" and isinstance(v, str):
            v = VELOCITY[v]
        elif k == "precision" and isinstance(v, str):
            v = PREC[v]
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f64(a, n=None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    if n is not None:
        a = a.reshape(n, 3)
    return a


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


class Context:
    """One filament system on the device (a qv_ctx)."""

    def __init__(self, params: QvParams | None = None, stream: int | None = None, **kw):
        self.params = params if params is not None else default_params(**kw)
        h = C.c_void_p()
        self._check(_lib.qv_create(C.byref(self.params), stream, C.byref(h)), None)
        self._h = h
        self.n = 0

    def _check(self, rc: int, h=-1):
        if rc < 0:
            hh = self._h if h == -1 else h
            msg = _lib.qv_last_error(hh).decode() if hh else "qv_create failed"
            raise QvError(rc, msg)
        return rc

    def close(self):
        if getattr(self, "_h", None):
            _lib.qv_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- state
    def set_params(self, params: QvParams):
        self._check(_lib.qv_set_params(self._h, C.byref(params)))
        self.params = params

    def set_points(self, x, infront, behind):
        x = _f64(x)
        n = x.shape[0]
        inf, beh = _i32(infront), _i32(behind)
        assert inf.shape == (n,) and beh.shape == (n,)
        self._check(_lib.qv_set_points(self._h, n, _ptr(x), _ptr(inf), _ptr(beh)))
        self.n = n

    def set_points_device(self, n: int, x_ptr: int, inf_ptr: int, beh_ptr: int):
        self._check(_lib.qv_set_points_device(self._h, n, x_ptr, inf_ptr, beh_ptr))
        self.n = n

    @staticmethod
    def _state(arrays) -> QvState:
        return QvState(*[None if arrays.get(k) is None else _ptr(arrays[k])
                         for k, _ in QvState._fields_])

    def set_state(self, n: int, **arrays):
        """One upload of x, infront, behind (required), u1..u3, closest (optional;
        host arrays of at least n entries, contiguous)."""
        self._check(_lib.qv_set_state(self._h, n, C.byref(self._state(arrays))))
        self.n = n

    def get_state(self, cap: int, **arrays) -> int:
        """One download into the given host arrays (capacity cap slots); returns
        the slot count in use."""
        m = C.c_int()
        self._check(_lib.qv_get_state(self._h, cap, C.byref(self._state(arrays)), C.byref(m)))
        self.n = m.value
        return m.value

    def step_exchange(self, itime: int, n: int, cap: int, inp: dict, out: dict) -> int:
        """One step with the host copy of the state: set_state(n, **inp), step,
        get_state(cap, **out) in one call (inp and out may share arrays); the
        copies overlap the step where the data allows.  Returns the slot count."""
        m = C.c_int()
        self._check(_lib.qv_step_exchange(self._h, itime, n, C.byref(self._state(inp)), cap,
                                          C.byref(self._state(out)), C.byref(m)))
        self.n = m.value
        return m.value

    def set_history(self, u1=None, u2=None, u3=None):
        arrs = [None if u is None else _f64(u, self.n) for u in (u1, u2, u3)]
        self._check(_lib.qv_set_history(self._h, *[_ptr(a) for a in arrs]))

    def get_history(self, *bufs):
        out = list(bufs) if bufs else [np.empty((self.n, 3)) for _ in range(3)]
        self._check(_lib.qv_get_history(self._h, *[_ptr(a) for a in out]))
        return out

    def set_closest(self, closest):
        c = _i32(closest)
        self._check(_lib.qv_set_closest(self._h, _ptr(c)))

    def get_points(self, x=None, u=None):
        x = np.empty((self.n, 3)) if x is None else x
        u = np.empty((self.n, 3)) if u is None else u
        self._check(_lib.qv_get_points(self._h, _ptr(x), _ptr(u)))
        return x, u

    def get_closest(self, closest=None, closestd=None):
        cl = np.empty(self.n, np.int32) if closest is None else closest
        cd = np.empty(self.n) if closestd is None else closestd
        self._check(_lib.qv_get_closest(self._h, _ptr(cl), _ptr(cd)))
        return cl, cd

    def device_arrays(self):
        px, pu, pi, pb = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
        self._check(_lib.qv_device_arrays(self._h, C.byref(px), C.byref(pu), C.byref(pi),
                                          C.byref(pb)))
        return px.value, pu.value, pi.value, pb.value

    # ---- path entry points
    def ghosts(self):
        self._check(_lib.qv_ghosts(self._h))

    def get_ghosts(self):
        out = [np.empty((self.n, 3)) for _ in range(4)]
        self._check(_lib.qv_get_ghosts(self._h, *[_ptr(a) for a in out]))
        return out

    def build_tree(self):
        self._check(_lib.qv_build_tree(self._h))

    def tree_info(self):
        a, b = C.c_int(), C.c_int()
        self._check(_lib.qv_tree_info(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def tree_export(self):
        m, _ = self.tree_info()
        parent = np.empty(m, np.int32)
        digit = np.empty(m, np.int32)
        depth = np.empty(m, np.int32)
        pos = np.empty((m, 3))
        width = np.empty(m)
        pcount = np.empty(m, np.int32)
        cent = np.empty((m, 3))
        circ = np.empty((m, 3))
        cij = np.empty((m, 9))
        first = np.empty(m, np.int32)
        arrs = [parent, digit, depth, pos, width, pcount, cent, circ, cij, first]
        self._check(_lib.qv_tree_export(self._h, m, *[_ptr(a) for a in arrs]))
        return dict(parent=parent, digit=digit, depth=depth, pos=pos, width=width,
                    pcount=pcount, cent=cent, circ=circ, Cij=cij, first=first)

    def velocity(self, want_parts: bool = True):
        u = np.empty((self.n, 3))
        uli = np.empty((self.n, 3)) if want_parts else None
        ubs = np.empty((self.n, 3)) if want_parts else None
        ev = C.c_longlong()
        self._check(_lib.qv_velocity(self._h, _ptr(u), _ptr(uli), _ptr(ubs), C.byref(ev)))
        return u, uli, ubs, ev.value

    def step_ab(self):
        self._check(_lib.qv_step_ab(self._h))

    def step_rk3(self):
        self._check(_lib.qv_step_rk3(self._h))

    def enforce_periodic(self):
        self._check(_lib.qv_enforce_periodic(self._h))

    def closest(self):
        cl = np.empty(self.n, np.int32)
        cd = np.empty(self.n)
        self._check(_lib.qv_closest(self._h, _ptr(cl), _ptr(cd)))
        return cl, cd

    def energy(self) -> float:
        e = C.c_double()
        self._check(_lib.qv_energy(self._h, C.byref(e)))
        return e.value

    def pinsert(self) -> int:
        k = C.c_int()
        self._check(_lib.qv_pinsert(self._h, C.byref(k)))
        self._sync_count()
        return k.value

    def precon(self) -> int:
        k = C.c_int()
        self._check(_lib.qv_precon(self._h, C.byref(k)))
        return k.value

    def premove(self) -> int:
        k = C.c_int()
        self._check(_lib.qv_premove(self._h, C.byref(k)))
        return k.value

    def get_links(self, inf=None, beh=None):
        inf = np.empty(self.n, np.int32) if inf is None else inf
        beh = np.empty(self.n, np.int32) if beh is None else beh
        self._check(_lib.qv_get_links(self._h, _ptr(inf), _ptr(beh)))
        return inf, beh

    def _sync_count(self):
        m = C.c_int()
        self._check(_lib.qv_point_count(self._h, C.byref(m)))
        self.n = m.value
        return self.n

    def step(self, itime: int = 1):
        self._check(_lib.qv_step(self._h, itime))
        if self.params.line_ops:
            self._sync_count()

    def steps(self, itime0: int, nsteps: int):
        self._check(_lib.qv_steps(self._h, itime0, nsteps))
        if self.params.line_ops:
            self._sync_count()

    def dump(self, path, itime: int, t: float, recon_count: int = 0):
        self._check(_lib.qv_dump(self._h, str(path).encode(), recon_count, itime, t))

    def restore(self, path):
        """Returns (itime, t, recon_count) of the file; the state is loaded."""
        rcn, it, t = C.c_int(), C.c_int(), C.c_double()
        self._check(_lib.qv_restore(self._h, str(path).encode(), C.byref(rcn), C.byref(it),
                                    C.byref(t)))
        self._sync_count()
        return it.value, t.value, rcn.value

    def root_undecided(self) -> int:
        k = C.c_int()
        self._check(_lib.qv_root_undecided(self._h, C.byref(k)))
        return k.value

    def write_snapshot(self, path, t: float):
        self._check(_lib.qv_write_snapshot(self._h, str(path).encode(), t))

    def sync(self):
        self._check(_lib.qv_sync(self._h))

    # ---- derivatives (device pointers)
    def velocity_device(self, u_ptr: int):
        self._check(_lib.qv_velocity_device(self._h, u_ptr))

    def velocity_vjp(self, ubar_ptr: int, xbar_ptr: int):
        self._check(_lib.qv_velocity_vjp(self._h, ubar_ptr, xbar_ptr))

    def energy_grad(self, u_ptr: int, xbar_ptr: int, ubar_ptr: int) -> float:
        e = C.c_double()
        self._check(_lib.qv_energy_grad(self._h, u_ptr, C.byref(e), xbar_ptr, ubar_ptr))
        return e.value

    def ab_step_device(self, x_ptr: int, u_ptr: int, u1_ptr: int, u2_ptr: int, u3_ptr: int,
                       xo_ptr: int):
        self._check(_lib.qv_ab_step_device(self._h, self.n, x_ptr, u_ptr, u1_ptr, u2_ptr, u3_ptr,
                                           xo_ptr))

    def ab_vjp_device(self, u1_ptr: int, u2_ptr: int, u3_ptr: int, xob_ptr: int, xb_ptr: int,
                      ub_ptr: int, u1b_ptr: int, u2b_ptr: int, u3b_ptr: int):
        self._check(_lib.qv_ab_vjp_device(self._h, self.n, u1_ptr, u2_ptr, u3_ptr, xob_ptr, xb_ptr,
                                          ub_ptr, u1b_ptr, u2b_ptr, u3b_ptr))

    def field_velocity_tree(self, pts):
        """tree_walk_general at the given points (the mesh_velocity Tree arm)."""
        pts = _f64(pts).reshape(-1, 3)
        u = np.empty_like(pts)
        ev = C.c_longlong()
        self._check(_lib.qv_field_velocity_tree(self._h, pts.shape[0], _ptr(pts), _ptr(u),
                                                C.byref(ev)))
        return u, ev.value

    def field_velocity(self, pts, grad_images: bool = False):
        pts = _f64(pts).reshape(-1, 3)
        m = pts.shape[0]
        u = np.empty((m, 3))
        du = np.empty((m, 3, 3))
        self._check(_lib.qv_field_velocity(self._h, m, _ptr(pts), int(grad_images), _ptr(u),
                                           _ptr(du)))
        return u, du

    # ---- instrumentation
    PHASES = ("ghosts", "build", "local", "nonlocal", "update", "search", "wrap",
              "build_levels", "build_moments", "line", "walk_kernel")

    def profile(self, enable: bool = True):
        self._check(_lib.qv_profile(self._h, int(enable)))

    def phase_times(self, reset: bool = True) -> dict:
        ms = np.zeros(len(self.PHASES))
        self._check(_lib.qv_phase_times(self._h, _ptr(ms), int(reset)))
        return dict(zip(self.PHASES, ms.tolist()))

    def counters(self):
        a, b, c = C.c_longlong(), C.c_longlong(), C.c_longlong()
        self._check(_lib.qv_counters(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return dict(launches=a.value, leaf_evals=b.value, far_evals=c.value)


def read_run_file(path) -> QvRun:
    r = QvRun()
    rc = _lib.qv_read_run_file(str(path).encode(), C.byref(r))
    if rc < 0:
        raise QvError(rc, f"cannot read {path}")
    return r


def read_var_file(path):
    n, t = C.c_int(), C.c_double()
    rc = _lib.qv_read_var_file(str(path).encode(), 0, C.byref(n), C.byref(t), None, None, None)
    if rc < 0:
        raise QvError(rc, f"cannot read {path}")
    x = np.empty((n.value, 3))
    inf = np.empty(n.value, np.int32)
    beh = np.empty(n.value, np.int32)
    rc = _lib.qv_read_var_file(str(path).encode(), n.value, C.byref(n), C.byref(t), _ptr(x),
                               _ptr(inf), _ptr(beh))
    if rc < 0:
        raise QvError(rc, f"cannot read {path}")
    return t.value, x, inf, beh


def write_var_file(path, t, x, infront, u=None):
    x = _f64(x)
    inf = _i32(infront)
    uu = None if u is None else _f64(u)
    rc = _lib.qv_write_var_file(str(path).encode(), x.shape[0], t, _ptr(x), _ptr(inf), _ptr(uu))
    if rc < 0:
        raise QvError(rc, f"cannot write {path}")


def write_restart_file(path, t: float, itime: int, recon_count: int = 0, **fields):
    """data_dump's var.dat from host arrays (x, infront, behind required)."""
    arrs = {k: (_f64(v) if k in RESTART_VEC or k == "closestd" else _i32(v))
            for k, v in fields.items() if v is not None}
    n = arrs["x"].shape[0]
    r = QvRestart(*[_ptr(arrs.get(k)) for k, _ in QvRestart._fields_])
    rc = _lib.qv_write_restart_file(str(path).encode(), n, recon_count, itime, t, C.byref(r))
    if rc < 0:
        raise QvError(rc, f"cannot write {path}")


def read_restart_file(path):
    """data_restore's read of var.dat: (t, itime, recon_count, fields)."""
    n, rcn, it, t = C.c_int(), C.c_int(), C.c_int(), C.c_double()
    rc = _lib.qv_read_restart_file(str(path).encode(), 0, C.byref(n), C.byref(rcn), C.byref(it),
                                   C.byref(t), None)
    if rc < 0:
        raise QvError(rc, f"cannot read {path}")
    m = n.value
    arrs = {k: np.empty((m, 3)) for k in RESTART_VEC}
    arrs["closestd"] = np.empty(m)
    arrs.update({k: np.empty(m, np.int32) for k in RESTART_INT})
    r = QvRestart(*[_ptr(arrs[k]) for k, _ in QvRestart._fields_])
    rc = _lib.qv_read_restart_file(str(path).encode(), m, C.byref(n), C.byref(rcn), C.byref(it),
                                   C.byref(t), C.byref(r))
    if rc < 0:
        raise QvError(rc, f"{path} is not a restart file of this layout")
    return t.value, it.value, rcn.value, arrs


def setup_loops(initf: str, pcount: int, delta: float):
    x = np.empty((pcount, 3))
    inf = np.empty(pcount, np.int32)
    beh = np.empty(pcount, np.int32)
    rc = _lib.qv_setup_loops(initf.encode(), pcount, delta, _ptr(x), _ptr(inf), _ptr(beh))
    if rc < 0:
        raise QvError(rc, f"initf {initf} is outside this path")
    return x, inf, beh


def test_stage_timeout(enable: bool) -> None:
    """Test hook: every direct-sum source-tile wait reports that it ran out
    (the copies still land and are drained); False restores normal waits."""
    _lib.qv_test_stage_timeout(int(bool(enable)))


def test_late_level1(mode: int = -1) -> None:
    """Test hook: -1 by build size (default), 0 never, 1 always pack the big
    root children of a mixed Tree build late (the walk adds their far-field
    terms after its launch)."""
    rc = _lib.qv_test_late_level1(int(mode))
    if rc < 0:
        raise QvError(rc, "bad late level-1 setting")


def test_root_speculation(mode: int = -1, bound_scale: float = 1.0) -> None:
    """Test hook: -1 by tree size (default), 0 never, 1 always start from the
    root centroid's estimate; bound_scale widens the estimate's bound."""
    rc = _lib.qv_test_root_speculation(int(mode), float(bound_scale))
    if rc < 0:
        raise QvError(rc, "bad root speculation setting")


def probe_fp32(stream: int | None = None) -> float:
    """Measured FP32 FMA throughput of the current device, TFLOP/s."""
    t = C.c_double()
    rc = _lib.qv_probe_fp32(stream, C.byref(t))
    if rc < 0:
        raise QvError(rc, "qv_probe_fp32 failed")
    return t.value


class Batch:
    """Independent open systems advanced together (a qv_batch).

    systems: list of (x (n, 3), infront, behind) with each system's own 1-based
    links; method[s] "BS" or "Tree"; dt[s] per system."""

    def __init__(self, params: QvParams, systems, method, dt, stream: int | None = None):
        self.params = params
        self.sizes = [len(sx[0]) for sx in systems]
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)]).astype(np.int32)
        meth = np.array([VELOCITY[m] if isinstance(m, str) else int(m) for m in method], np.int32)
        dts = np.asarray(dt, np.float64)
        h = C.c_void_p()
        rc = _lib.qv_batch_create(C.byref(params), len(systems), _ptr(self.offsets), _ptr(meth),
                                  _ptr(dts), stream, C.byref(h))
        if rc < 0:
            raise QvError(rc, "qv_batch_create failed")
        self._h = h
        self.ntot = int(self.offsets[-1])
        x = _f64(np.concatenate([sx[0] for sx in systems]))
        inf = _i32(np.concatenate([sx[1] for sx in systems]))
        beh = _i32(np.concatenate([sx[2] for sx in systems]))
        self._check(_lib.qv_batch_set_points(self._h, _ptr(x), _ptr(inf), _ptr(beh)))

    def _check(self, rc: int):
        if rc < 0:
            raise QvError(rc, _lib.qv_batch_last_error(self._h).decode())
        return rc

    def close(self):
        if getattr(self, "_h", None):
            _lib.qv_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def split(self, a: np.ndarray):
        return [a[self.offsets[s]:self.offsets[s + 1]] for s in range(len(self.sizes))]

    def velocity(self) -> np.ndarray:
        u = np.empty((self.ntot, 3))
        self._check(_lib.qv_batch_velocity(self._h, _ptr(u)))
        return u

    def step(self, nsteps: int = 1):
        self._check(_lib.qv_batch_step(self._h, int(nsteps)))

    def get_points(self):
        x = np.empty((self.ntot, 3))
        u = np.empty((self.ntot, 3))
        self._check(_lib.qv_batch_get_points(self._h, _ptr(x), _ptr(u)))
        return x, u

    def tune(self, reps: int = 3):
        cfg = np.zeros(3, np.int32)
        ms = C.c_float()
        self._check(_lib.qv_batch_tune(self._h, reps, _ptr(cfg), C.byref(ms)))
        return dict(warps_per_block=int(cfg[0]), blocks_per_sm=int(cfg[1]), order=int(cfg[2]),
                    work_ms=ms.value)

    def set_config(self, warps_per_block: int, blocks_per_sm: int, order: int):
        self._check(_lib.qv_batch_set_config(self._h, warps_per_block, blocks_per_sm, order))

    def stats(self) -> dict:
        ev = np.zeros(2, np.int64)
        g = C.c_int()
        cfg = np.zeros(8, np.int32)
        self._check(_lib.qv_batch_stats(self._h, _ptr(ev), C.byref(g), _ptr(cfg)))
        keys = ("warps_per_block", "blocks_per_sm", "order", "stack", "items", "tree_systems",
                "depth", "launches")
        return dict(leaf_evals=int(ev[0]), far_evals=int(ev[1]), graph=bool(g.value),
                    **{k: int(v) for k, v in zip(keys, cfg)})
