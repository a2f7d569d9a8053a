"""Driver for the reference's own build in oracle/_ref/libvortex_ref.so.

TEST INFRASTRUCTURE ONLY.  Calls the reference's unit_1.cuh entry points
(include/unit_1.cuh:15-55) the way its src/main.c step loop does
(src/main.c:652-785), to pin the CPU oracle and to record golden vectors.
matr_creation is host code and runs anywhere; vort_creation/Speed/Step need a
GPU.  The reference's AoS records (NO_TREE build): Vortex = 3 doubles
(x, y, G), PVortex = 2 doubles, tPanel = 120 bytes.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libvortex_ref.so")

_lib = None
_libc = C.CDLL(None)
_libc.free.argtypes = [C.c_void_p]


def available() -> bool:
    return os.path.exists(REF_LIB)


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(REF_LIB)
        _lib.matr_creation.restype = C.c_void_p
        _lib.matr_creation.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t]
        _lib.vxref_conf_set.argtypes = [C.c_char_p, C.c_double]
        _lib.vxref_malloc.restype = C.c_void_p
        _lib.vxref_malloc.argtypes = [C.c_size_t]
        _lib.vxref_free.argtypes = [C.c_void_p]
        _lib.vxref_h2d.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        _lib.vxref_d2h.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        _lib.vort_creation.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_size_t,
                                       C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.Speed.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p,
                               C.c_double, C.c_void_p]
        _lib.Step.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_size_t), C.c_size_t,
                              C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.velocity_control.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p,
                                          C.c_void_p, C.c_size_t]
        assert _lib.vxref_sizeof_vortex() == 24 and _lib.vxref_sizeof_panel() == 120
    return _lib


def round32(v: int) -> int:
    return (v + 31) // 32 * 32


def padded_panels(pan: np.ndarray) -> np.ndarray:
    P = len(pan)
    out = np.zeros(round32(P), dtype=pan.dtype)
    out[:P] = pan
    return out


def matr_creation(pan: np.ndarray) -> np.ndarray:
    """Reference panel matrix (src/unit_1.cu:256-402): returns the padded
    (P32+1)^2 row-major inverse.  The reference writes L.txt/M.txt into the
    working directory, so it runs inside a temporary directory."""
    P = len(pan)
    P32 = round32(P)
    pp = padded_panels(pan)
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as td:
        os.chdir(td)
        try:
            ptr = lib().matr_creation(pp.ctypes.data, P, P32)
        finally:
            os.chdir(cwd)
    if not ptr:
        raise RuntimeError("reference matr_creation failed")
    S = P32 + 1
    M = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_double)), shape=(S * S,)).copy()
    _libc.free(ptr)
    return M.reshape(S, S)


class RefRun:
    """Runs the reference step loop on the GPU (src/main.c:652-785) with the
    device arrays pre-sized so incr_vort_quant is never needed; the never-
    written tail holds far-away G=0 fillers (like randomize_tail)."""

    def __init__(self, pan, conf: dict, cap: int):
        L = lib()
        self.P = len(pan)
        self.P32 = round32(self.P)
        self.cap = cap
        L.vxref_conf_reset()
        for k, v in conf.items():
            if L.vxref_conf_set(k.encode(), float(v)):
                raise KeyError(k)
        L.vxref_conf_set(b"birth_quant", float(self.P))
        if L.init_device_conf_values():
            raise RuntimeError("init_device_conf_values failed")
        M = matr_creation(pan)
        self.nu = conf["viscosity"]
        S = self.P32 + 1
        self.d_pos = L.vxref_malloc(cap * 24)
        self.d_vel = L.vxref_malloc(cap * 16)
        self.d_d = L.vxref_malloc(cap * 8)
        self.d_M = L.vxref_malloc(S * S * 8)
        self.d_pan = L.vxref_malloc(self.P32 * 120)
        self.d_vinf = L.vxref_malloc(16)
        self.d_dg = L.vxref_malloc(8)
        self.d_F = L.vxref_malloc(16)
        self.d_Mom = L.vxref_malloc(8)
        pos = np.zeros((cap, 3))
        pos[:, 0] = 4.0e5 + np.arange(cap)
        pos[:, 1] = 4.0e5 + np.arange(cap)
        self._h2d(self.d_pos, pos)
        self._h2d(self.d_M, np.ascontiguousarray(M))
        self._h2d(self.d_pan, padded_panels(pan))
        self._h2d(self.d_vinf, np.array([conf["v_inf_x"], conf["v_inf_y"]]))
        self.n = 0

    @staticmethod
    def _h2d(dst, arr):
        arr = np.ascontiguousarray(arr)
        if lib().vxref_h2d(dst, arr.ctypes.data, arr.nbytes):
            raise RuntimeError("h2d")

    @staticmethod
    def _d2h(src, shape, dtype=np.float64):
        out = np.zeros(shape, dtype=dtype)
        if lib().vxref_d2h(out.ctypes.data, src, out.nbytes):
            raise RuntimeError("d2h")
        return out

    def load(self, x, y, g):
        n = len(x)
        pos = np.stack([x, y, g], axis=1)
        self._h2d(self.d_pos, pos)
        self.n = n

    def state(self, upto):
        return self._d2h(self.d_pos, (upto, 3))

    def scalars(self):
        dg = self._d2h(self.d_dg, (1,))[0]
        F = self._d2h(self.d_F, (2,))
        Mm = self._d2h(self.d_Mom, (1,))[0]
        return dg, F[0], F[1], Mm

    def step(self, record=None):
        """One step; when record is a dict, the state after each stage is stored."""
        L = lib()
        P, P32 = self.P, self.P32
        s = round32(self.n + P)
        assert s + 32 <= self.cap
        if record is not None:
            record["pre_pos"] = self.state(s)
            record["pre_n"] = self.n
            record["pre_dg"] = self.scalars()[0]
        if L.vort_creation(self.d_pos, self.d_vinf, P, P32, self.n, self.d_M, self.d_dg, self.d_pan):
            raise RuntimeError("vort_creation")
        self.n += P
        if record is not None:
            record["born_pos"] = self.state(s)
        if L.Speed(self.d_pos, self.d_vinf, s, self.d_vel, self.d_d, self.nu, self.d_pan):
            raise RuntimeError("Speed")
        if record is not None:
            record["vel"] = self._d2h(self.d_vel, (s, 2))
            record["d"] = self._d2h(self.d_d, (s,))
        z = np.zeros(2)
        self._h2d(self.d_F, z)
        self._h2d(self.d_dg, z[:1])
        self._h2d(self.d_Mom, z[:1])
        n = C.c_size_t(self.n)
        if L.Step(self.d_pos, self.d_vel, C.byref(n), s, self.d_dg, self.d_F, self.d_Mom, self.d_pan):
            raise RuntimeError("Step")
        self.n = n.value
        if record is not None:
            record["post_pos"] = self.state(s)
            record["post_n"] = self.n
            record["post_scalars"] = np.array(self.scalars())
        return self.n

    def probe(self, px, py):
        L = lib()
        npb = len(px)
        cp = np.zeros((npb, 3))
        cp[:, 0], cp[:, 1] = px, py
        d_cp = L.vxref_malloc(npb * 24)
        d_v = L.vxref_malloc(round32(npb) * 16)
        self._h2d(d_cp, cp)
        if L.velocity_control(self.d_pos, self.d_vinf, self.n, d_cp, d_v, npb):
            raise RuntimeError("velocity_control")
        v = self._d2h(d_v, (npb, 2))
        L.vxref_free(d_cp)
        L.vxref_free(d_v)
        return v

    def close(self):
        L = lib()
        for p in (self.d_pos, self.d_vel, self.d_d, self.d_M, self.d_pan, self.d_vinf,
                  self.d_dg, self.d_F, self.d_Mom):
            L.vxref_free(p)
