"""ctypes binding of the CPU oracle (oracle/qv_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, never by the qvort_b200 package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libqv_oracle.so"


def build() -> Path:
    src = HERE / "qv_oracle.c"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE), "-s"], check=True)
    return LIB


class QoParams(C.Structure):
    _fields_ = [
        ("quant_circ", C.c_double), ("corea", C.c_double), ("box_size", C.c_double),
        ("delta", C.c_double), ("dt", C.c_double), ("tree_theta", C.c_double),
        ("boundary", C.c_int), ("velocity", C.c_int), ("deriv_order", C.c_int),
        ("tree_extra_correction", C.c_int), ("fixed_lia_beta", C.c_int),
    ]


_BC = {"open": 0, "periodic": 1, "openx": 2, "openxy": 3}
_VEL = {"Off": 0, "LIA": 1, "BS": 2, "Tree": 3}


def params(**kw) -> QoParams:
    p = QoParams()
    p.quant_circ = kw.get("quant_circ", 9.97e-4)
    p.corea = kw.get("corea", 8.244023e-9)
    p.box_size = kw.get("box_size", 0.1)
    p.delta = kw.get("delta", 5e-4)
    p.dt = kw.get("dt", 1e-7)
    p.tree_theta = kw.get("tree_theta", 0.0)
    b = kw.get("boundary", "open")
    p.boundary = _BC[b] if isinstance(b, str) else b
    v = kw.get("velocity", "BS")
    p.velocity = _VEL[v] if isinstance(v, str) else v
    p.deriv_order = kw.get("deriv_order", 2)
    p.tree_extra_correction = kw.get("tree_extra_correction", 1)
    p.fixed_lia_beta = kw.get("fixed_lia_beta", 0)
    return p


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(str(LIB))
        P = C.POINTER(QoParams)
        v = C.c_void_p
        _lib.qo_ghosts.argtypes = [P, C.c_int, v, v, v, v, v, v, v]
        _lib.qo_enforce_periodic.argtypes = [P, C.c_int, v, v]
        _lib.qo_tree_build.argtypes = [P, C.c_int, v, v, v]
        _lib.qo_tree_build.restype = C.c_void_p
        _lib.qo_tree_free.argtypes = [v]
        _lib.qo_tree_status.argtypes = [v]
        _lib.qo_tree_maxdepth.argtypes = [v]
        _lib.qo_tree_count.argtypes = [v]
        _lib.qo_tree_export.argtypes = [v, C.c_int] + [v] * 10
        _lib.qo_velocity.argtypes = [P, C.c_int, v, v, v, v, v, v, v, v, C.c_int, v, v, v, v,
                                     C.POINTER(C.c_longlong), C.c_int]
        _lib.qo_pmotion_ab.argtypes = [C.c_double, C.c_int, v, v, v, v, v, v]
        _lib.qo_pclose_tree.argtypes = [v, C.c_int, v, v, v, v, v, C.c_int]
        _lib.qo_pclose.argtypes = [C.c_int, v, v, v, v, v]
        _lib.qo_energy.argtypes = [P, C.c_int, v, v, v, v, v, v, v]
        _lib.qo_energy.restype = C.c_double
        _lib.qo_step.argtypes = [P, C.c_int, v, v, v, v, v, v, v, v, v, v, v, C.c_int, v, v,
                                 C.POINTER(C.c_longlong), C.c_int]
        _lib.qo_dt_max.argtypes = [P]
        _lib.qo_dt_max.restype = C.c_double
        _lib.qo_set_depth_cap.argtypes = [C.c_int]
        _lib.qo_pinsert.argtypes = [P, C.POINTER(C.c_int), C.c_int, C.POINTER(QoState)]
        _lib.qo_premove.argtypes = [P, C.c_int, C.POINTER(QoState)]
        _lib.qo_precon.argtypes = [P, C.c_int, C.POINTER(QoState)]
        _lib.qo_field_velocity_tree.argtypes = [P, v, C.c_int, v, v]
        _lib.qo_field_velocity_tree.restype = C.c_longlong
        _lib.qo_field_velocity.argtypes = [P, C.c_int, v, v, v, C.c_int, v, v]
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def ghosts(p: QoParams, x, inf, beh):
    x, inf, beh = _f(x), _i(inf), _i(beh)
    n = x.shape[0]
    g = [np.zeros((n, 3)) for _ in range(4)]
    lib().qo_ghosts(C.byref(p), n, _p(x), _p(inf), _p(beh), *[_p(a) for a in g])
    return g


class Tree:
    def __init__(self, p: QoParams, x, gi, inf):
        self.x, self.gi, self.inf = _f(x), _f(gi), _i(inf)
        self.h = lib().qo_tree_build(C.byref(p), self.x.shape[0], _p(self.x), _p(self.gi),
                                     _p(self.inf))

    @property
    def status(self) -> int:
        return lib().qo_tree_status(self.h)

    def export(self) -> dict:
        m = lib().qo_tree_count(self.h)
        out = dict(parent=np.empty(m, np.int32), digit=np.empty(m, np.int32),
                   depth=np.empty(m, np.int32), pos=np.empty((m, 3)), width=np.empty(m),
                   pcount=np.empty(m, np.int32), cent=np.empty((m, 3)), circ=np.empty((m, 3)),
                   Cij=np.empty((m, 9)), first=np.empty(m, np.int32))
        keys = ["parent", "digit", "depth", "pos", "width", "pcount", "cent", "circ", "Cij",
                "first"]
        lib().qo_tree_export(self.h, m, *[_p(out[k]) for k in keys])
        return out

    def close(self):
        if self.h:
            lib().qo_tree_free(self.h)
            self.h = None

    def __del__(self):
        self.close()


def velocity(p: QoParams, x, inf, beh, g, tree: Tree | None = None, targets=None,
             nthreads: int = 1):
    x, inf, beh = _f(x), _i(inf), _i(beh)
    g = [_f(a) for a in g]
    n = x.shape[0]
    tg = None if targets is None else _i(targets)
    nt = n if tg is None else tg.shape[0]
    u = np.zeros((nt, 3))
    uli = np.zeros((nt, 3))
    ubs = np.zeros((nt, 3))
    ev = C.c_longlong()
    st = lib().qo_velocity(C.byref(p), n, _p(x), _p(inf), _p(beh), *[_p(a) for a in g],
                           tree.h if tree is not None else None, nt, _p(tg), _p(u), _p(uli),
                           _p(ubs), C.byref(ev), nthreads)
    return u, uli, ubs, ev.value, st


def pmotion_ab(dt, x, u, u1, u2, u3, inf):
    x, u = _f(x).copy(), _f(u)
    u1, u2, u3 = _f(u1).copy(), _f(u2).copy(), _f(u3).copy()
    lib().qo_pmotion_ab(dt, x.shape[0], _p(x), _p(u), _p(u1), _p(u2), _p(u3), _p(_i(inf)))
    return x, u1, u2, u3


def pclose_tree(tree: Tree, x, inf, beh, closest, nthreads: int = 1):
    x, inf, beh = _f(x), _i(inf), _i(beh)
    cl = _i(closest).copy()
    cd = np.zeros(x.shape[0])
    lib().qo_pclose_tree(tree.h, x.shape[0], _p(x), _p(inf), _p(beh), _p(cl), _p(cd), nthreads)
    return cl, cd


def pclose(x, inf, beh, closest, closestd=None):
    x, inf, beh = _f(x), _i(inf), _i(beh)
    cl = _i(closest).copy()
    cd = np.zeros(x.shape[0]) if closestd is None else _f(closestd).copy()
    lib().qo_pclose(x.shape[0], _p(x), _p(inf), _p(beh), _p(cl), _p(cd))
    return cl, cd


def energy(p: QoParams, x, u, inf, g) -> float:
    x, u, inf = _f(x), _f(u), _i(inf)
    g = [_f(a) for a in g]
    return lib().qo_energy(C.byref(p), x.shape[0], _p(x), _p(u), _p(inf), *[_p(a) for a in g])


class State:
    """The oracle's copy of f(:) for whole steps (qo_step)."""

    def __init__(self, p: QoParams, x, inf, beh):
        self.p = p
        self.x = _f(x).copy()
        self.inf, self.beh = _i(inf), _i(beh)
        n = self.x.shape[0]
        self.u = np.zeros((n, 3))
        self.u1 = np.zeros((n, 3))
        self.u2 = np.zeros((n, 3))
        self.u3 = np.zeros((n, 3))
        self.g = [np.zeros((n, 3)) for _ in range(4)]
        self.closest = np.zeros(n, np.int32)
        self.closestd = np.zeros(n)
        self.evals = 0

    def step(self, runge_kutta: bool = False, search: bool = True, nthreads: int = 1) -> int:
        ev = C.c_longlong()
        st = lib().qo_step(C.byref(self.p), self.x.shape[0], _p(self.x), _p(self.inf),
                           _p(self.beh), _p(self.u), _p(self.u1), _p(self.u2), _p(self.u3),
                           *[_p(a) for a in self.g], int(runge_kutta),
                           _p(self.closest) if search else None,
                           _p(self.closestd) if search else None, C.byref(ev), nthreads)
        self.evals = ev.value
        return st


class QoState(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("x", "u", "u1", "u2", "u3", "gi", "gb", "gii", "gbb",
                                          "u_li", "u_bs", "closestd", "infront", "behind",
                                          "closest")]


LINE_FIELDS = {"x": 3, "u": 3, "u1": 3, "u2": 3, "u3": 3, "gi": 3, "gb": 3, "gii": 3, "gbb": 3,
               "u_li": 3, "u_bs": 3, "closestd": 1, "infront": 0, "behind": 0, "closest": 0}


def line_state(n: int, cap: int, **arrays):
    """Arrays of cap slots for pinsert/premove, the first n filled from `arrays`
    (missing fields zero)."""
    st = {}
    for k, w in LINE_FIELDS.items():
        if w == 0:
            a = np.zeros(cap, np.int32)
        elif w == 1:
            a = np.zeros(cap)
        else:
            a = np.zeros((cap, 3))
        if k in arrays:
            a[:n] = arrays[k]
        st[k] = a
    return st


def _qostate(st) -> QoState:
    return QoState(*[st[k].ctypes.data_as(C.c_void_p) for k in LINE_FIELDS])


def pinsert(p: QoParams, n: int, st) -> tuple[int, int]:
    """pinsert on the state dict in place; returns (new pcount, points inserted)."""
    cap = st["x"].shape[0]
    pc = C.c_int(n)
    k = lib().qo_pinsert(C.byref(p), C.byref(pc), cap, C.byref(_qostate(st)))
    if k < 0:
        raise RuntimeError("pinsert needs more than cap slots")
    return pc.value, k


def premove(p: QoParams, n: int, st) -> int:
    """premove on the state dict in place; returns the points removed."""
    return lib().qo_premove(C.byref(p), n, C.byref(_qostate(st)))


def precon(p: QoParams, n: int, st) -> int:
    """precon_original on the state dict in place; returns the reconnections."""
    return lib().qo_precon(C.byref(p), n, C.byref(_qostate(st)))


class Loop:
    """The reference's whole time-loop body (src/run.f90:41-93) on the oracle's
    copy of f(:), with the line operations:

      ghostp; construct_tree; pmotion; pinsert; every recon_shots steps
      pclose_tree on the tree built before the move (pclose when
      tree_theta = 0), precon_original, premove; ghostp; enforce_periodic.

    line_ops: 0 = none, 1 = pinsert and premove, 2 = also precon (the
    reference's default loop, switch_off_recon F).  Arrays hold `cap` slots;
    `n` is pcount.  Points inserted this step are searched as targets but
    cannot be found as partners (the tree predates them), as in the reference.
    """

    def __init__(self, p: QoParams, x, inf, beh, cap: int | None = None, line_ops: int = 2,
                 recon_shots: int = 1, nthreads: int = 1):
        x = _f(x)
        self.p = p
        self.n = x.shape[0]
        self.cap = cap or 2 * self.n + 64
        self.st = line_state(self.n, self.cap, x=x, infront=_i(inf), behind=_i(beh))
        self.line_ops = line_ops
        self.recon_shots = recon_shots
        self.nthreads = nthreads
        self.evals = 0
        self.counts = {}

    def _ghosts(self):
        n, s = self.n, self.st
        g = ghosts(self.p, s["x"][:n], s["infront"][:n], s["behind"][:n])
        for k, a in zip(("gi", "gb", "gii", "gbb"), g):
            s[k][:n] = a

    def step(self, itime: int) -> int:
        p, s = self.p, self.st
        n = self.n
        self._ghosts()                                            # run.f90:41
        tree = None
        if p.tree_theta > 0:                                      # run.f90:43
            tree = Tree(p, s["x"][:n], s["gi"][:n], s["infront"][:n])
            if tree.status:
                return -2
        g = [s[k][:n] for k in ("gi", "gb", "gii", "gbb")]       # run.f90:50 pmotion
        u, uli, ubs, ev, st = velocity(p, s["x"][:n], s["infront"][:n], s["behind"][:n], g, tree,
                                       nthreads=self.nthreads)
        if st:
            return st
        self.evals = ev
        act = s["infront"][:n] != 0
        s["u"][:n][act], s["u_li"][:n][act], s["u_bs"][:n][act] = u[act], uli[act], ubs[act]
        xn, h1, h2, h3 = pmotion_ab(p.dt, s["x"][:n], s["u"][:n], s["u1"][:n], s["u2"][:n],
                                    s["u3"][:n], s["infront"][:n])
        s["x"][:n], s["u1"][:n], s["u2"][:n], s["u3"][:n] = xn, h1, h2, h3
        self.counts = {"inserted": 0, "reconnected": 0, "removed": 0}
        if self.line_ops:                                         # run.f90:61
            self.n, self.counts["inserted"] = pinsert(p, self.n, s)
            n = self.n
        if itime % self.recon_shots == 0:                         # run.f90:63-72
            if tree is not None:
                cl, cd = pclose_tree(tree, s["x"][:n], s["infront"][:n], s["behind"][:n],
                                     s["closest"][:n], self.nthreads)
            else:
                cl, cd = pclose(s["x"][:n], s["infront"][:n], s["behind"][:n], s["closest"][:n],
                                s["closestd"][:n])
            s["closest"][:n], s["closestd"][:n] = cl, cd
            if self.line_ops == 2:
                self.counts["reconnected"] = precon(p, n, s)
            if self.line_ops:
                self.counts["removed"] = premove(p, n, s)
        if tree is not None:
            tree.close()
        self._ghosts()                                            # run.f90:75
        if p.boundary in (1, 2, 3):                               # run.f90:82-93
            lib().qo_enforce_periodic(C.byref(p), n, _p(s["x"]), _p(s["infront"]))
        return 0

    def state(self) -> dict:
        n = self.n
        return {k: v[:n].copy() for k, v in self.st.items()}


def field_velocity_tree(p: QoParams, tree, pts):
    """tree_walk_general at the points (the Tree arm of mesh_velocity)."""
    pts = _f(pts).reshape(-1, 3)
    u = np.zeros_like(pts)
    ev = lib().qo_field_velocity_tree(C.byref(p), tree.h, pts.shape[0], _p(pts), _p(u))
    return u, ev


def field_velocity(p: QoParams, x, inf, gi, pts):
    """biot_savart_general with the boundary's images at the points (the BS arm
    of mesh_velocity)."""
    x, inf, gi = _f(x), _i(inf), _f(gi)
    pts = _f(pts).reshape(-1, 3)
    u = np.zeros_like(pts)
    lib().qo_field_velocity(C.byref(p), x.shape[0], _p(x), _p(gi), _p(inf), pts.shape[0],
                            _p(pts), _p(u))
    return u


def dt_max(p: QoParams) -> float:
    return lib().qo_dt_max(C.byref(p))
