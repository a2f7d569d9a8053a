"""ctypes wrapper of the CPU oracle (oracle/libvx_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvx_oracle.so")

PREC_FP64, PREC_REF = 0, 1
BIRTH_REF, BIRTH_FILE, BIRTH_HALF_PANEL = 0, 1, 2


class Params(C.Structure):
    _fields_ = [
        ("dt", C.c_double), ("nu", C.c_double), ("rho", C.c_double),
        ("vinf_x", C.c_double), ("vinf_y", C.c_double),
        ("eps", C.c_double),
        ("r_col_diff_sign", C.c_double), ("r_col_same_sign", C.c_double),
        ("max_ve_g", C.c_double),
        ("x_min", C.c_double), ("x_max", C.c_double), ("y_min", C.c_double), ("y_max", C.c_double),
        ("prof_x_min", C.c_double), ("prof_x_max", C.c_double),
        ("prof_y_min", C.c_double), ("prof_y_max", C.c_double),
        ("rc_x", C.c_double), ("rc_y", C.c_double),
        ("drop_eps", C.c_double),
        ("n_of_points", C.c_int64), ("n_col", C.c_int64),
        ("birth_mode", C.c_int32), ("prec", C.c_int32),
    ]


class State(C.Structure):
    _fields_ = [
        ("cap", C.c_int64), ("n", C.c_int64),
        ("x", C.c_void_p), ("y", C.c_void_p), ("g", C.c_void_p),
        ("vx", C.c_void_p), ("vy", C.c_void_p), ("d", C.c_void_p),
        ("dg", C.c_double), ("fx", C.c_double), ("fy", C.c_double), ("m", C.c_double),
    ]


_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        _lib.vxo_collapse.restype = C.c_int64
        _lib.vxo_compact.restype = C.c_int64
        _lib.vxo_step.restype = C.c_int64
        _lib.vxo_compact.argtypes = [C.c_void_p] * 3 + [C.c_int64, C.c_double]
        _lib.vxo_hitting.restype = C.c_int
    return _lib


def _p(a):
    """Pointer to a numpy array's data.  The caller must keep `a` referenced
    until the C call returns (never pass a temporary)."""
    return C.c_void_p(a.ctypes.data) if a is not None else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def make_params(**kw) -> Params:
    p = Params()
    defaults = dict(dt=0.005, nu=1e-3, rho=1.0, vinf_x=1.0, vinf_y=0.0, eps=0.0157,
                    r_col_diff_sign=0.0, r_col_same_sign=0.3, max_ve_g=1e30,
                    x_min=-2.0, x_max=10.0, y_min=-10.0, y_max=10.0,
                    prof_x_min=-0.5, prof_x_max=0.5, prof_y_min=-0.5, prof_y_max=0.5,
                    rc_x=0.0, rc_y=0.0, drop_eps=1e-12, n_of_points=20, n_col=2,
                    birth_mode=BIRTH_REF, prec=PREC_FP64)
    defaults.update(kw)
    for k, v in defaults.items():
        setattr(p, k, v)
    return p


def panel_matrix(pan):
    P = len(pan)
    L = np.zeros((P + 1, P + 1))
    M = np.zeros((P + 1, P + 1))
    rc = lib().vxo_panel_matrix(_p(pan), C.c_int64(P), _p(L), _p(M))
    if rc:
        raise RuntimeError("singular panel system")
    return L, M


def birth_rhs(p, pan, x, y, g):
    R = np.zeros(len(pan))
    x, y, g = _f64(x), _f64(y), _f64(g)
    lib().vxo_birth_rhs(C.byref(p), _p(pan), C.c_int64(len(pan)), _p(x), _p(y), _p(g),
                        C.c_int64(len(x)), _p(R))
    return R


def birth_gamma(Minv, R, dg):
    P = len(R)
    gam = np.zeros(P)
    Minv, R = _f64(Minv), _f64(R)
    lib().vxo_birth_gamma(C.c_int64(P), _p(Minv), _p(R), C.c_double(dg), _p(gam))
    return gam


def birth_place(p, pan, gamma):
    P = len(pan)
    x, y, g = np.zeros(P), np.zeros(P), np.zeros(P)
    gamma = _f64(gamma)
    lib().vxo_birth_place(C.byref(p), _p(pan), C.c_int64(P), _p(gamma), _p(x), _p(y), _p(g))
    return x, y, g


def velocity(p, x, y, g, n, s=None):
    """Targets [0,n); 3-nearest over [0,s) (default round32(n))."""
    if s is None:
        s = (n + 31) // 32 * 32
    x, y, g = _f64(x), _f64(y), _f64(g)
    assert len(x) >= s
    vx, vy, d = np.zeros(n), np.zeros(n), np.zeros(n)
    lib().vxo_velocity(C.byref(p), _p(x), _p(y), _p(g), C.c_int64(n), C.c_int64(s),
                       _p(vx), _p(vy), _p(d))
    return vx, vy, d


def diffusion(p, x, y, g, n, d, vx, vy):
    vx, vy = _f64(vx).copy(), _f64(vy).copy()
    x, y, g, d = _f64(x), _f64(y), _f64(g), _f64(d)
    lib().vxo_diffusion(C.byref(p), _p(x), _p(y), _p(g), C.c_int64(n), _p(d), _p(vx), _p(vy))
    return vx, vy


def diffusion_sums(p, x, y, g, n, d):
    """(I1, A1) of every target: the diffusion sum and its magnitude sum."""
    x, y, g, d = _f64(x), _f64(y), _f64(g), _f64(d)
    I1, A1 = np.zeros(n), np.zeros(n)
    lib().vxo_diffusion_sums(C.byref(p), _p(x), _p(y), _p(g), C.c_int64(n), _p(d), _p(I1), _p(A1))
    return I1, A1


def wall_diffusion(p, pan, x, y, n, d, vx, vy):
    vx, vy = _f64(vx).copy(), _f64(vy).copy()
    x, y, d = _f64(x), _f64(y), _f64(d)
    lib().vxo_wall_diffusion(C.byref(p), _p(pan), C.c_int64(len(pan)), _p(x), _p(y),
                             C.c_int64(n), _p(d), _p(vx), _p(vy))
    return vx, vy


def advect(p, pan, x, y, g, vx, vy, n, n_new):
    x, y, g = _f64(x).copy(), _f64(y).copy(), _f64(g).copy()
    t = np.zeros((4, n))
    vx, vy = _f64(vx), _f64(vy)
    lib().vxo_advect(C.byref(p), _p(pan), C.c_int64(len(pan)), _p(x), _p(y), _p(g),
                     _p(vx), _p(vy), C.c_int64(n), C.c_int64(n_new),
                     _p(t[0]), _p(t[1]), _p(t[2]), _p(t[3]))
    return x, y, g, t


def sums(p, t):
    n = t.shape[1]
    t = np.ascontiguousarray(t)
    out = (C.c_double * 4)()
    lib().vxo_sums(C.byref(p), C.c_int64(n), _p(t[0]), _p(t[1]), _p(t[2]), _p(t[3]),
                   C.byref(out, 0), C.byref(out, 8), C.byref(out, 16), C.byref(out, 24))
    return tuple(out)


def compact(x, y, g, n, drop_eps=1e-12):
    x, y, g = _f64(x).copy(), _f64(y).copy(), _f64(g).copy()
    m = lib().vxo_compact(_p(x), _p(y), _p(g), C.c_int64(n), C.c_double(drop_eps))
    return x, y, g, int(m)


def collapse_col(p, pas, x, y, g, n):
    col = np.zeros(n, dtype=np.int32)
    x, y, g = _f64(x), _f64(y), _f64(g)
    lib().vxo_collapse_col(C.byref(p), C.c_int(pas), _p(x), _p(y), _p(g), C.c_int64(n), _p(col))
    return col


def collapse_merge(pas, x, y, g, n, col):
    x, y, g = _f64(x).copy(), _f64(y).copy(), _f64(g).copy()
    col = np.ascontiguousarray(col, dtype=np.int32).copy()
    lib().vxo_collapse_merge(C.c_int(pas), _p(x), _p(y), _p(g), C.c_int64(n), _p(col))
    return x, y, g


def collapse(p, pas, x, y, g, n):
    x, y, g = _f64(x).copy(), _f64(y).copy(), _f64(g).copy()
    col = np.zeros(max(n, 1), dtype=np.int32)
    m = lib().vxo_collapse(C.byref(p), C.c_int(pas), _p(x), _p(y), _p(g), C.c_int64(n), _p(col))
    return x, y, g, int(m)


def probe(p, x, y, g, n, px, py):
    px, py = _f64(px), _f64(py)
    vx, vy = np.zeros(len(px)), np.zeros(len(px))
    x, y, g = _f64(x), _f64(y), _f64(g)
    lib().vxo_probe(C.byref(p), _p(x), _p(y), _p(g), C.c_int64(n),
                    _p(px), _p(py), C.c_int64(len(px)), _p(vx), _p(vy))
    return vx, vy


def fill_tail(x, y, g, start, stop):
    lib().vxo_fill_tail(_p(x), _p(y), _p(g), C.c_int64(start), C.c_int64(stop))


class OracleSim:
    """Whole-step oracle: a particle store with the reference's padded tail."""

    def __init__(self, params: Params, pan, Minv, cap: int = 8192):
        self.p = params
        self.pan = np.ascontiguousarray(pan)
        self.P = len(pan)
        self.Minv = np.ascontiguousarray(Minv, dtype=np.float64)
        self.cap = 0
        self.arr = {k: np.zeros(0) for k in ("x", "y", "g", "vx", "vy", "d")}
        self.n = 0
        self.dg = self.fx = self.fy = self.m = 0.0
        self._grow(cap)

    def _grow(self, cap):
        old = self.cap
        for k in self.arr:
            a = np.zeros(cap)
            a[:old] = self.arr[k][:old]
            self.arr[k] = a
        fill_tail(self.arr["x"], self.arr["y"], self.arr["g"], old, cap)
        self.cap = cap

    def load(self, x, y, g):
        n = len(x)
        need = (n + self.P + 31) // 32 * 32 + 32
        if need > self.cap:
            self._grow(need)
        self.arr["x"][:n], self.arr["y"][:n], self.arr["g"][:n] = x, y, g
        self.n = n

    def step(self):
        need = (self.n + self.P + 31) // 32 * 32 + 32
        if need > self.cap:
            self._grow(max(need, self.cap + 8192))
        st = State(self.cap, self.n, *[self.arr[k].ctypes.data for k in ("x", "y", "g", "vx", "vy", "d")],
                   self.dg, self.fx, self.fy, self.m)
        lib().vxo_step(C.byref(self.p), _p(self.pan), C.c_int64(self.P), _p(self.Minv), C.byref(st))
        self.n, self.dg, self.fx, self.fy, self.m = st.n, st.dg, st.fx, st.fy, st.m
        return self.n

    def particles(self):
        n = self.n
        return self.arr["x"][:n].copy(), self.arr["y"][:n].copy(), self.arr["g"][:n].copy()
