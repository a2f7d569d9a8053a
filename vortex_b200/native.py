"""ctypes binding of libvortex_b200.so (include/vortex_b200.h).

The library is the product; this module only marshals numpy arrays through
its C ABI.  Importing it on a machine without the built library raises: there
is no fallback path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .profiles import PANEL_DTYPE

HERE = os.path.dirname(os.path.abspath(__file__))
# the in-tree build; VORTEX_B200_LIB names another build of the same sources
# (a variant built with VX_NVCC_DEFS, for measuring it side by side)
LIB_PATH = os.environ.get("VORTEX_B200_LIB") or os.path.join(HERE, "libvortex_b200.so")

PREC_FP64, PREC_FP32 = 0, 1
BIRTH_REF, BIRTH_FILE, BIRTH_HALF_PANEL = 0, 1, 2
STAGE = dict(birth=1, velocity=2, diffusion=4, wall=8, advect=16, compact=32,
             collapse1=64, collapse2=128, all=0xFF)


class Conf(C.Structure):
    _fields_ = [
        ("steps", C.c_int64), ("saving_step", C.c_int64), ("inc_step", C.c_int64),
        ("n_of_points", C.c_int64), ("n_col", C.c_int64), ("v_inf_incr_steps", C.c_int64),
        ("tree_depth", C.c_int64),
        ("dt", C.c_double), ("viscosity", C.c_double), ("rho", C.c_double),
        ("v_inf_x", C.c_double), ("v_inf_y", C.c_double),
        ("x_max", C.c_double), ("x_min", C.c_double), ("y_max", C.c_double), ("y_min", C.c_double),
        ("ve_size", C.c_double), ("h_col_x", C.c_double), ("h_col_y", C.c_double),
        ("rc_x", C.c_double), ("rc_y", C.c_double),
        ("r_col_diff_sign", C.c_double), ("r_col_same_sign", C.c_double), ("max_ve_g", C.c_double),
        ("rel_t", C.c_double), ("theta", C.c_double),
        ("matrix_load", C.c_int32), ("steady_flow", C.c_int32), ("log_level", C.c_int32),
        ("no_log_buf", C.c_int32),
        ("pr_file", C.c_char * 256), ("timings_file", C.c_char * 256), ("kadr_file", C.c_char * 256),
        ("second_points_file", C.c_char * 256), ("log_file", C.c_char * 256),
        ("precision", C.c_int32), ("birth_offset_mode", C.c_int32),
        ("drop_eps", C.c_double), ("diff_cutoff", C.c_double),
        ("n_probes_grid", C.c_int32), ("pad1_", C.c_int32), ("probe_box", C.c_double * 4),
        ("fmm", C.c_int32), ("gj_pivot", C.c_int32), ("fmm_leaf", C.c_int32), ("fmm_p", C.c_int32),
    ]


class VxError(RuntimeError):
    pass


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise VxError(f"{LIB_PATH} is missing: build it with `python -m vortex_b200.build`")
        _lib = C.CDLL(LIB_PATH)
        _lib.vx_last_error.restype = C.c_char_p
        _lib.vx_status_str.restype = C.c_char_p
        _lib.vx_get_stream.restype = C.c_void_p
        _lib.vx_get_stream.argtypes = [C.c_void_p]
        _lib.vx_batch_stream.restype = C.c_void_p
        _lib.vx_batch_stream.argtypes = [C.c_void_p]
        for name in ("vx_create",):
            getattr(_lib, name).argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_void_p]
    return _lib


def _check(rc, what=""):
    if rc != 0:
        L = lib()
        raise VxError(f"{what}: {L.vx_status_str(rc).decode()} ({L.vx_last_error().decode()})")


def _p(a):
    return C.c_void_p(a.ctypes.data)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def default_conf(**kw) -> Conf:
    c = Conf()
    _check(lib().vx_conf_default(C.byref(c)), "vx_conf_default")
    base = dict(steps=400, saving_step=50, inc_step=8192, n_of_points=20, n_col=2, v_inf_incr_steps=0,
                dt=0.005, viscosity=1e-3, rho=1.0, v_inf_x=1.0, v_inf_y=0.0,
                x_max=10.0, x_min=-2.0, y_max=10.0, y_min=-10.0, ve_size=0.0157,
                rc_x=0.0, rc_y=0.0, r_col_diff_sign=0.0, r_col_same_sign=0.3, max_ve_g=1e30)
    base.update(kw)
    for k, v in base.items():
        if isinstance(v, str):
            v = v.encode()
        setattr(c, k, v)
    return c


def measure_peak(device: int = 0, fp64: bool = False, mode: int | None = None) -> float:
    """TFLOP/s of the FP32 (or FP64) FMA pipe; mode 3: 1e12 rsqrt + ex2 units/s."""
    t = C.c_double(0)
    m = int(fp64) if mode is None else mode
    _check(lib().vx_measure_peak(C.c_int(device), C.c_int(m), C.byref(t)), "vx_measure_peak")
    return t.value


def read_conf(path: str, conf: Conf | None = None) -> Conf:
    c = conf if conf is not None else default_conf()
    _check(lib().vx_conf_read(path.encode(), C.byref(c)), "vx_conf_read")
    return c


def read_profile(path: str) -> np.ndarray:
    P = C.c_int64(0)
    _check(lib().vx_profile_read(path.encode(), None, C.c_int64(0), C.byref(P)), "vx_profile_read")
    pan = np.zeros(P.value, dtype=PANEL_DTYPE)
    _check(lib().vx_profile_read(path.encode(), _p(pan), C.c_int64(P.value), C.byref(P)), "vx_profile_read")
    return pan


class Sim:
    """One body resident on a GPU (vx_sim)."""

    def __init__(self, conf: Conf, panels: np.ndarray, device: int = 0):
        self.conf = conf
        self.pan = np.ascontiguousarray(panels, dtype=PANEL_DTYPE)
        self.P = len(self.pan)
        self.h = C.c_void_p()
        _check(lib().vx_create(C.byref(conf), _p(self.pan), C.c_int64(self.P), C.c_int(device),
                               C.byref(self.h)), "vx_create")

    def close(self):
        if self.h:
            lib().vx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- state -----------------------------------------------------------
    def set_particles(self, x, y, g):
        x, y, g = _f64(x), _f64(y), _f64(g)
        _check(lib().vx_set_particles(self.h, _p(x), _p(y), _p(g), C.c_int64(len(x))), "vx_set_particles")

    def set_slots(self, x, y, g, n):
        x, y, g = _f64(x), _f64(y), _f64(g)
        _check(lib().vx_set_slots(self.h, _p(x), _p(y), _p(g), C.c_int64(len(x)), C.c_int64(n)), "vx_set_slots")

    def get_slots(self, count):
        x, y, g = np.zeros(count), np.zeros(count), np.zeros(count)
        _check(lib().vx_get_slots(self.h, _p(x), _p(y), _p(g), C.c_int64(count)), "vx_get_slots")
        return x, y, g

    def set_velocity(self, vx=None, vy=None, d=None):
        n = len(vx) if vx is not None else len(d)
        arrs = [None if a is None else _f64(a) for a in (vx, vy, d)]
        ptrs = [None if a is None else _p(a) for a in arrs]
        _check(lib().vx_set_velocity(self.h, *ptrs, C.c_int64(n)), "vx_set_velocity")

    def count(self) -> int:
        n = C.c_int64(0)
        _check(lib().vx_get_count(self.h, C.byref(n)), "vx_get_count")
        return n.value

    def particles(self):
        n = self.count()
        x, y, g = np.zeros(n), np.zeros(n), np.zeros(n)
        m = C.c_int64(0)
        _check(lib().vx_get_particles(self.h, _p(x), _p(y), _p(g), C.c_int64(n), C.byref(m)), "vx_get_particles")
        return x, y, g

    def particles_into(self, x, y, g) -> int:
        """Live particles copied into caller arrays (float64, contiguous,
        large enough; pinned host memory makes the copies fastest)."""
        m = C.c_int64(0)
        _check(lib().vx_get_particles(self.h, _p(x), _p(y), _p(g), C.c_int64(min(len(x), len(y), len(g))),
                                      C.byref(m)), "vx_get_particles")
        return m.value

    def velocity(self):
        n = self.count()
        vx, vy, d = np.zeros(n), np.zeros(n), np.zeros(n)
        _check(lib().vx_get_velocity(self.h, _p(vx), _p(vy), _p(d), C.c_int64(n)), "vx_get_velocity")
        return vx, vy, d

    def forces(self):
        o = np.zeros(4)
        _check(lib().vx_get_forces(self.h, _p(o)), "vx_get_forces")
        return o

    def state(self):
        o = np.zeros(9)
        _check(lib().vx_get_state(self.h, _p(o)), "vx_get_state")
        return dict(n=int(o[0]), n0=int(o[1]), step=int(o[2]), vinf=(o[3], o[4]), dg=o[5],
                    fx=o[6], fy=o[7], m=o[8])

    def matrix(self):
        M = np.zeros((self.P + 1, self.P + 1))
        _check(lib().vx_get_matrix(self.h, _p(M)), "vx_get_matrix")
        return M

    def set_dg(self, dg):
        _check(lib().vx_set_dg(self.h, C.c_double(dg)), "vx_set_dg")

    def set_vinf(self, vx, vy):
        _check(lib().vx_set_vinf(self.h, C.c_double(vx), C.c_double(vy)), "vx_set_vinf")

    def set_step_index(self, k):
        _check(lib().vx_set_step_index(self.h, C.c_int64(k)), "vx_set_step_index")

    # --- running -----------------------------------------------------------
    def step(self, nsteps: int = 1):
        _check(lib().vx_step(self.h, C.c_int64(nsteps)), "vx_step")

    def stage(self, *names):
        mask = 0
        for nm in names:
            mask |= STAGE[nm]
        _check(lib().vx_stage(self.h, C.c_uint(mask)), "vx_stage")

    def sync(self):
        _check(lib().vx_sync(self.h), "vx_sync")

    def probe(self, px, py):
        px, py = _f64(px), _f64(py)
        vx, vy = np.zeros(len(px)), np.zeros(len(px))
        _check(lib().vx_probe(self.h, _p(px), _p(py), C.c_int64(len(px)), _p(vx), _p(vy)), "vx_probe")
        return vx, vy

    def checkpoint_save(self, path: str):
        _check(lib().vx_checkpoint_save(self.h, os.fsencode(path)), "vx_checkpoint_save")

    def checkpoint_load(self, path: str):
        _check(lib().vx_checkpoint_load(self.h, os.fsencode(path)), "vx_checkpoint_load")

    def move_points(self, x, y, g, u, v):
        """Tracer points moved one step with velocities (u, v); returns new
        (x, y, g), g = 0 for points absorbed by the wall or the window."""
        x, y, g = _f64(x).copy(), _f64(y).copy(), _f64(g).copy()
        u, v = _f64(u), _f64(v)
        _check(lib().vx_move_points(self.h, _p(x), _p(y), _p(g), _p(u), _p(v), C.c_int64(len(x))),
               "vx_move_points")
        return x, y, g

    def set_graph(self, on: bool):
        _check(lib().vx_set_graph(self.h, C.c_int(int(on))), "vx_set_graph")

    def set_timing(self, on: bool):
        _check(lib().vx_set_timing(self.h, C.c_int(int(on))), "vx_set_timing")

    def timing(self):
        """ms per stage: birth, velocity, diffusion, wall, step, bs_pair, diff_pair, total."""
        o = np.zeros(8)
        _check(lib().vx_get_timing(self.h, _p(o)), "vx_get_timing")
        return o

    def pair_counts(self, clear: bool = False):
        """(near-field pairs, diffusion pairs) executed by the bulk form."""
        o = np.zeros(2)
        _check(lib().vx_get_pair_counts(self.h, _p(o), C.c_int(int(clear))), "vx_get_pair_counts")
        return o

    def tree_info(self) -> dict:
        """Quadtree depth / leaf side / 3-nearest fallbacks and neighbour-grid
        geometry of the last bulk-form pass."""
        o = np.zeros(6)
        _check(lib().vx_get_tree_info(self.h, _p(o)), "vx_get_tree_info")
        return {"fmm_level": int(o[0]), "leaf_side": o[1], "nn3_redone": int(o[2]), "cell_side": o[3],
                "cells_x": int(o[4]), "cells_y": int(o[5])}

    def launches(self) -> int:
        n = C.c_int64(0)
        _check(lib().vx_get_launch_count(self.h, C.byref(n)), "vx_get_launch_count")
        return n.value

    def stream(self) -> int:
        return lib().vx_get_stream(self.h) or 0

    def set_fmm(self, fmm: bool, leaf: int = 8, p: int = None):
        _check(lib().vx_set_fmm(self.h, C.c_int(int(fmm)), C.c_int(int(leaf))), "vx_set_fmm")
        if p is not None:
            _check(lib().vx_set_fmm_order(self.h, C.c_int(int(p))), "vx_set_fmm_order")

    def kernel_times(self, nsteps: int = 3) -> dict:
        """{kernel name: (total ms, launches)} over nsteps instrumented steps
        (an event pair around every launch)."""
        cap = 512
        names = C.create_string_buffer(64 * cap)
        ms = np.zeros(cap)
        cnt = np.zeros(cap, dtype=np.int64)
        nk = C.c_int64(0)
        _check(lib().vx_kernel_times(self.h, C.c_int64(nsteps), names, C.c_int64(len(names)), _p(ms), _p(cnt),
                                     C.c_int64(cap), C.byref(nk)), "vx_kernel_times")
        nm = names.value.decode().split("\n")
        k = min(nk.value, cap)
        return {nm[i]: (float(ms[i]), int(cnt[i])) for i in range(k)}

    def device_bytes(self) -> int:
        b = C.c_int64(0)
        _check(lib().vx_get_device_bytes(self.h, C.byref(b)), "vx_get_device_bytes")
        return b.value


def estimate_bytes(conf: Conf, P: int, n_max: int, device: int = 0) -> int:
    """Device bytes a body with P panels holds once it reaches n_max vortices."""
    b = C.c_int64(0)
    _check(lib().vx_estimate_bytes(C.byref(conf), C.c_int64(P), C.c_int64(n_max), C.c_int(device),
                                   C.byref(b)), "vx_estimate_bytes")
    return b.value


def step_many(sims, nsteps: int = 1):
    """Advance several bodies together (their kernels overlap); asynchronous."""
    arr = (C.c_void_p * len(sims))(*[s.h.value for s in sims])
    _check(lib().vx_step_many(arr, C.c_int(len(sims)), C.c_int64(nsteps)), "vx_step_many")


_rt = None


def cudart():
    """The CUDA runtime the library itself links (for events and streams)."""
    global _rt
    if _rt is None:
        lib()
        _rt = C.CDLL("libcudart.so.12")
        _rt.cudaEventCreate.argtypes = [C.POINTER(C.c_void_p)]
        _rt.cudaEventRecord.argtypes = [C.c_void_p, C.c_void_p]
        _rt.cudaEventSynchronize.argtypes = [C.c_void_p]
        _rt.cudaEventElapsedTime.argtypes = [C.POINTER(C.c_float), C.c_void_p, C.c_void_p]
        _rt.cudaEventDestroy.argtypes = [C.c_void_p]
        _rt.cudaStreamWaitEvent.argtypes = [C.c_void_p, C.c_void_p, C.c_uint]
    return _rt


class Event:
    """A CUDA event with timing (device time between two records)."""

    def __init__(self):
        self.e = C.c_void_p()
        if cudart().cudaEventCreate(C.byref(self.e)) != 0:
            raise VxError("cudaEventCreate failed")

    def record(self, stream: int = 0):
        if cudart().cudaEventRecord(self.e, C.c_void_p(stream)) != 0:
            raise VxError("cudaEventRecord failed")

    def synchronize(self):
        if cudart().cudaEventSynchronize(self.e) != 0:
            raise VxError("cudaEventSynchronize failed")

    def elapsed_ms(self, end: "Event") -> float:
        end.synchronize()
        t = C.c_float(0.0)
        if cudart().cudaEventElapsedTime(C.byref(t), self.e, end.e) != 0:
            raise VxError("cudaEventElapsedTime failed")
        return float(t.value)

    def __del__(self):
        try:
            if self.e:
                cudart().cudaEventDestroy(self.e)
        except Exception:
            pass


def wait_event(stream: int, ev: Event):
    if cudart().cudaStreamWaitEvent(C.c_void_p(stream), ev.e, 0) != 0:
        raise VxError("cudaStreamWaitEvent failed")


class Batch:
    """Bodies of one device advanced together (vx_batch): one launch per
    kernel of the step for all bodies, the batched step one CUDA graph."""

    def __init__(self, sims):
        self.sims = list(sims)
        arr = (C.c_void_p * len(self.sims))(*[s.h.value for s in self.sims])
        self.h = C.c_void_p()
        _check(lib().vx_batch_create(arr, C.c_int(len(self.sims)), C.byref(self.h)), "vx_batch_create")

    def step(self, nsteps: int = 1):
        _check(lib().vx_batch_step(self.h, C.c_int64(nsteps)), "vx_batch_step")

    def add(self, sim):
        _check(lib().vx_batch_add(self.h, sim.h), "vx_batch_add")
        self.sims.append(sim)

    def remove(self, sim):
        _check(lib().vx_batch_remove(self.h, sim.h), "vx_batch_remove")
        self.sims.remove(sim)

    def last_results(self) -> dict:
        """{sim handle value: (count, d_g, Fx, Fy, M)} after the last batched step."""
        cap = max(len(self.sims), 1) + 64
        mem = (C.c_void_p * cap)()
        out = np.zeros(5 * cap)
        cnt = C.c_int(0)
        _check(lib().vx_batch_last_results(self.h, mem, _p(out), C.c_int(cap), C.byref(cnt)),
               "vx_batch_last_results")
        return {mem[i]: tuple(out[5 * i:5 * i + 5]) for i in range(min(cnt.value, cap))}

    def sync(self):
        _check(lib().vx_batch_sync(self.h), "vx_batch_sync")

    def stream(self) -> int:
        return lib().vx_batch_stream(self.h) or 0

    def info(self) -> dict:
        o = np.zeros(6)
        _check(lib().vx_batch_info(self.h, _p(o)), "vx_batch_info")
        t = np.zeros(8)
        _check(lib().vx_batch_host_times(self.h, _p(t)), "vx_batch_host_times")
        return {"steps": int(o[0]), "kernels": int(o[1]), "kernels_per_step": int(o[2]), "rebuilds": int(o[3]),
                "graph_instantiations": int(o[4]), "bodies": int(o[5]),
                "host_grow_ms_max": float(t[0]), "host_grow_ms_total": float(t[1]),
                "host_refresh_ms_max": float(t[2]), "host_refresh_ms_total": float(t[3]),
                "host_phase_ms_max": {"record": float(t[4]), "merge": float(t[5]), "upload": float(t[6]),
                                      "graph": float(t[7])}}

    def close(self):
        if self.h:
            lib().vx_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Server:
    """Continuous-batching request loop over resident bodies (vx_server)."""

    STATES = ("queued", "resident", "done", "failed")

    def __init__(self, budget_bytes: int, max_active: int = 64, device: int = 0):
        self.h = C.c_void_p()
        _check(lib().vx_server_create(C.c_int(device), C.c_int64(int(budget_bytes)), C.c_int(max_active),
                                      C.byref(self.h)), "vx_server_create")

    def close(self):
        if self.h:
            lib().vx_server_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, conf: Conf, panels, x, y, g, nsteps: int) -> int:
        pan = np.ascontiguousarray(panels, dtype=PANEL_DTYPE)
        x, y, g = _f64(x), _f64(y), _f64(g)
        rid = C.c_int64(0)
        _check(lib().vx_server_submit(self.h, C.byref(conf), _p(pan), C.c_int64(len(pan)), _p(x), _p(y), _p(g),
                                      C.c_int64(len(x)), C.c_int64(nsteps), C.byref(rid)), "vx_server_submit")
        return rid.value

    def set_batched(self, on: bool):
        _check(lib().vx_server_set_batched(self.h, C.c_int(int(on))), "vx_server_set_batched")

    def tick(self):
        """One scheduling round; returns (resident, queued) after it."""
        a, q = C.c_int64(0), C.c_int64(0)
        _check(lib().vx_server_tick(self.h, C.byref(a), C.byref(q)), "vx_server_tick")
        return a.value, q.value

    def result(self, rid: int, cap_steps: int = 0):
        st, done, nf = C.c_int(0), C.c_int64(0), C.c_int64(0)
        _check(lib().vx_server_result(self.h, C.c_int64(rid), C.byref(st), C.byref(done), None, C.c_int64(0),
                                      C.byref(nf)), "vx_server_result")
        k = min(cap_steps, done.value) if cap_steps else done.value
        f = np.zeros((max(k, 1), 4))
        if k:
            _check(lib().vx_server_result(self.h, C.c_int64(rid), C.byref(st), C.byref(done), _p(f),
                                          C.c_int64(k), C.byref(nf)), "vx_server_result")
        out = {"state": self.STATES[st.value], "steps": done.value, "forces": f[:k], "n_final": nf.value}
        if out["state"] == "failed":
            buf = C.create_string_buffer(512)
            _check(lib().vx_server_failure(self.h, C.c_int64(rid), buf, C.c_int64(512)), "vx_server_failure")
            out["error"] = buf.value.decode(errors="replace")
        return out

    def stats(self) -> dict:
        o = np.zeros(10)
        _check(lib().vx_server_stats(self.h, _p(o)), "vx_server_stats")
        return {"finished": int(o[0]), "step_ms_p50": o[1], "step_ms_p99": o[2], "ttc_s_p50": o[3],
                "ttc_s_p99": o[4], "mean_resident": o[5], "body_steps": int(o[6]), "particle_steps": o[7],
                "bytes_reserved": int(o[8]), "ticks": int(o[9])}
