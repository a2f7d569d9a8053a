"""The reference's own entry points (include/unit_1.cuh), as exported by
libvortex_b200.so, replayed on the reference's recorded states.

Each golden step (tests/golden/ref_*.npz, recorded from the reference's CUDA
build) is fed through vort_creation / Speed / Step / velocity_control on AoS
device arrays exactly as the reference's src/main.c passes them:
  * birth: positions exact, strengths within 1e-10 of the FP64 oracle and
    1e-5 of the reference (which sums its right-hand side in FP32), or, where
    the reference's FP32 sums depart further from FP64 (its 1000-panel
    circle: up to 2e-3 of the largest strength), no further from the
    reference than the FP64 oracle is;
  * Speed: d bit-exact and velocity within 1e-12 of the FP64 oracle, within
    2e-3 of the reference;
  * Step on the reference's own velocities: the reference's count, identical
    strengths, positions within 2 ulp, d_g/F/M within 1e-12;
  * velocity_control: within 5e-6 of the reference's FP32 probe, or no
    further from it than the FP64 oracle's probe is.
"""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.test_ref_golden_cpu import CASES, load, params
from vortex_b200 import native as N

pytestmark = pytest.mark.gpu


class VxuConf(C.Structure):
    _fields_ = [
        ("steps", C.c_size_t), ("saving_step", C.c_size_t), ("dt", C.c_double), ("inc_step", C.c_size_t),
        ("viscosity", C.c_double), ("rho", C.c_double), ("v_inf_x", C.c_double), ("v_inf_y", C.c_double),
        ("n_of_points", C.c_size_t), ("x_max", C.c_double), ("x_min", C.c_double), ("y_max", C.c_double),
        ("y_min", C.c_double), ("profile_x_min", C.c_double), ("profile_x_max", C.c_double),
        ("profile_y_min", C.c_double), ("profile_y_max", C.c_double), ("ve_size", C.c_double),
        ("n_col", C.c_size_t), ("h_col_x", C.c_double), ("h_col_y", C.c_double), ("rc_x", C.c_double),
        ("rc_y", C.c_double), ("pr_file", C.c_char * 256), ("birth_quant", C.c_size_t),
        ("r_col_diff_sign", C.c_double), ("r_col_same_sign", C.c_double), ("matrix_load", C.c_uint8),
        ("v_inf_incr_steps", C.c_size_t), ("max_ve_g", C.c_double), ("log_file", C.c_char * 256),
        ("config_file", C.c_char * 256), ("log_level", C.c_uint8), ("timings_file", C.c_char * 256),
        ("kadr_file", C.c_char * 256), ("second_points_file", C.c_char * 256), ("rel_t", C.c_double),
        ("steady_flow", C.c_uint8), ("no_log_buf", C.c_uint8),
    ]


assert C.sizeof(VxuConf) == 1792

_rt = None


def rt():
    global _rt
    if _rt is None:
        _rt = C.CDLL("libcudart.so.12")
        _rt.cudaMalloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
        _rt.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
        _rt.cudaFree.argtypes = [C.c_void_p]
    return _rt


class Dev:
    """A device buffer owned by the test (cudart, no framework)."""

    def __init__(self, nbytes):
        self.p = C.c_void_p()
        assert rt().cudaMalloc(C.byref(self.p), max(nbytes, 8)) == 0
        self.nbytes = nbytes

    def put(self, arr):
        arr = np.ascontiguousarray(arr)
        assert arr.nbytes <= self.nbytes
        assert rt().cudaMemcpy(self.p, arr.ctypes.data, arr.nbytes, 1) == 0

    def get(self, shape, dtype=np.float64):
        out = np.zeros(shape, dtype)
        assert rt().cudaMemcpy(out.ctypes.data, self.p, out.nbytes, 2) == 0
        return out

    def __del__(self):
        try:
            rt().cudaFree(self.p)
        except Exception:
            pass


def setup_conf(c, P):
    L = N.lib()
    conf = VxuConf.in_dll(L, "conf")
    C.memset(C.addressof(conf), 0, C.sizeof(conf))
    for k in ("dt", "viscosity", "rho", "v_inf_x", "v_inf_y", "x_max", "x_min", "y_max", "y_min",
              "profile_x_min", "profile_x_max", "profile_y_min", "profile_y_max", "ve_size", "rc_x", "rc_y",
              "r_col_diff_sign", "r_col_same_sign", "max_ve_g"):
        setattr(conf, k, float(c[k]))
    conf.n_of_points = int(c["n_of_points"])
    conf.n_col = int(c["n_col"])
    conf.inc_step = 8192
    conf.birth_quant = P
    assert L.init_device_conf_values() == 0
    return conf


def round32(v):
    return (v + 31) // 32 * 32


@pytest.mark.parametrize("name,k", CASES)
def test_unit1_entry_points_replay_reference(name, k):
    z, c, pan = load(name)
    L = N.lib()
    P = len(pan)
    P32 = round32(P)
    setup_conf(c, P)
    p64 = params(c, O.PREC_FP64)
    # panel system through matr_creation (host array in, padded host matrix out)
    pp = np.zeros(P32, dtype=pan.dtype)
    pp[:P] = pan
    L.matr_creation.restype = C.c_void_p
    cwd = os.getcwd()
    os.chdir(os.environ.get("TMPDIR", "/tmp"))
    try:
        mptr = L.matr_creation(C.c_void_p(pp.ctypes.data), C.c_size_t(P), C.c_size_t(P32))
    finally:
        os.chdir(cwd)
    assert mptr
    S1 = P32 + 1
    M = np.ctypeslib.as_array(C.cast(mptr, C.POINTER(C.c_double)), shape=(S1 * S1,)).copy().reshape(S1, S1)
    C.CDLL(None).free(C.c_void_p(mptr))
    _, Mo = O.panel_matrix(pan)
    assert np.abs(M[:P + 1, :P + 1] - Mo).max() < 1e-11 * np.abs(Mo).max()
    assert not M[P + 1:].any() and not M[:, P + 1:].any()

    pre, n0, dg = z[f"s{k}_pre_pos"], int(z[f"s{k}_pre_n"]), float(z[f"s{k}_pre_dg"])
    born_ref, vel_ref, d_ref = z[f"s{k}_born_pos"], z[f"s{k}_vel"], z[f"s{k}_d"]
    s = len(born_ref)
    cap = s + 64
    pos = Dev(cap * 24)
    buf = np.zeros((cap, 3))
    buf[:, 0] = buf[:, 1] = 4e5 + np.arange(cap)
    buf[:s] = pre
    pos.put(buf)
    vel = Dev(cap * 16)
    dd = Dev(cap * 8)
    vinf = Dev(16)
    vinf.put(np.array([c["v_inf_x"], c["v_inf_y"]]))
    ddg = Dev(8)
    ddg.put(np.array([dg]))
    mdev = Dev(S1 * S1 * 8)
    mdev.put(M)
    pdev = Dev(P32 * 120)
    pdev.put(pp)
    vp = C.c_void_p
    # --- vort_creation
    assert L.vort_creation(pos.p, vinf.p, C.c_size_t(P), C.c_size_t(P32), C.c_size_t(n0), mdev.p, ddg.p, pdev.p) == 0
    born = pos.get((cap, 3))
    n = n0 + P
    R = O.birth_rhs(p64, pan, pre[:n0, 0].copy(), pre[:n0, 1].copy(), pre[:n0, 2].copy())
    bx, by, bg = O.birth_place(p64, pan, O.birth_gamma(Mo, R, dg))
    assert np.array_equal(born[n0:n, 0], bx) and np.array_equal(born[n0:n, 1], by)
    assert np.abs(born[n0:n, 2] - bg).max() <= 1e-10 * np.abs(bg).max()
    # the reference sums its right-hand side in FP32
    ref_gap = np.abs(bg - born_ref[n0:n, 2]).max()
    assert np.abs(born[n0:n, 2] - born_ref[n0:n, 2]).max() <= max(1e-5 * np.abs(bg).max(),
                                                                  ref_gap + 1e-10 * np.abs(bg).max())
    # --- Speed on the reference's post-birth state
    buf[:s] = born_ref
    pos.put(buf)
    assert L.Speed(pos.p, vinf.p, C.c_size_t(s), vel.p, dd.p, C.c_double(c["viscosity"]), pdev.p) == 0
    v = vel.get((cap, 2))
    d = dd.get(cap)
    xs, ys, gs = born_ref[:, 0].copy(), born_ref[:, 1].copy(), born_ref[:, 2].copy()
    ovx, ovy, od = O.velocity(p64, xs, ys, gs, s, s)
    ovx, ovy = O.diffusion(p64, xs, ys, gs, s, od, ovx, ovy)
    ovx, ovy = O.wall_diffusion(p64, pan, xs, ys, s, od, ovx, ovy)
    assert np.array_equal(d[:s], od)
    assert max(np.abs(v[:s, 0] - ovx).max(), np.abs(v[:s, 1] - ovy).max()) < 1e-11
    assert max(np.abs(v[:n] - vel_ref[:n]).max(), 0) < 2e-3
    # --- Step on the reference's own velocities
    vel.put(np.concatenate([vel_ref, np.zeros((cap - s, 2))]))
    F = Dev(16)
    F.put(np.zeros(2))
    Mm = Dev(8)
    Mm.put(np.zeros(1))
    nn = C.c_size_t(n)
    assert L.Step(pos.p, vel.p, C.byref(nn), C.c_size_t(s), ddg.p, F.p, Mm.p, pdev.p) == 0
    assert nn.value == int(z[f"s{k}_post_n"])
    post = pos.get((s, 3))
    ref = z[f"s{k}_post_pos"]
    assert np.array_equal(post[:, 2], ref[:, 2])
    ulp = np.spacing(np.maximum(np.abs(ref[:, :2]), 1e-300))
    assert np.all(np.abs(post[:, :2] - ref[:, :2]) <= 2 * ulp)
    got = [ddg.get(1)[0], *F.get(2), Mm.get(1)[0]]
    for a, b in zip(got, z[f"s{k}_post_scalars"]):
        assert abs(a - b) <= 1e-12 * max(1.0, abs(b))
    # --- velocity_control at the reference's 500 control points
    cp = np.zeros((500, 3))
    cp[:, 0] = -0.15
    cp[:, 1] = 0.01 + 0.002 * np.arange(500)
    cpd = Dev(500 * 24)
    cpd.put(cp)
    vout = Dev(512 * 16)
    assert L.velocity_control(pos.p, vinf.p, C.c_size_t(nn.value), cpd.p, vout.p, C.c_size_t(500)) == 0
    pv = vout.get((500, 2))
    # the reference's probe sums in FP32: within 5e-6 of it, or (its
    # 1000-panel circle, 3200 vortices) no further than the FP64 oracle's
    # probe of the same state is
    post_pos = pos.get((cap, 3))[:nn.value]
    ox, oy = O.probe(p64, post_pos[:, 0].copy(), post_pos[:, 1].copy(), post_pos[:, 2].copy(), nn.value,
                     cp[:, 0].copy(), cp[:, 1].copy())
    gap = np.abs(np.stack([ox, oy], 1) - z[f"s{k}_probe"]).max()
    assert np.abs(pv - z[f"s{k}_probe"]).max() < max(5e-6, 1.01 * gap + 1e-12)
    L.vxu_launch_count.restype = C.c_int64
    assert L.vxu_launch_count() > 0


def test_unit1_speed_fp32_bulk_form():
    """VORTEX_B200_PRECISION=fp32 switches the unit_1 entry points to the
    FP32-bulk form: Speed on a recorded reference state gives the 3-nearest
    distance within 1e-6 relative of the FP64 oracle, velocities within the
    2e-3 the reference's own FP32 build is held to, median relative error
    below 1e-4; unsetting it restores the plain form."""
    name, k = CASES[0]
    z, c, pan = load(name)
    L = N.lib()
    P = len(pan)
    P32 = round32(P)
    p64 = params(c, O.PREC_FP64)
    born_ref = z[f"s{k}_born_pos"]
    s = len(born_ref)
    cap = s + 64
    pp = np.zeros(P32, dtype=pan.dtype)
    pp[:P] = pan
    pdev = Dev(P32 * 120)
    pdev.put(pp)
    vinf = Dev(16)
    vinf.put(np.array([c["v_inf_x"], c["v_inf_y"]]))
    buf = np.zeros((cap, 3))
    buf[:, 0] = buf[:, 1] = 4e5 + np.arange(cap)
    buf[:s] = born_ref
    pos, vel, dd = Dev(cap * 24), Dev(cap * 16), Dev(cap * 8)
    pos.put(buf)
    saved = os.environ.get("VORTEX_B200_PRECISION")
    os.environ["VORTEX_B200_PRECISION"] = "fp32"
    try:
        setup_conf(c, P)
        assert L.Speed(pos.p, vinf.p, C.c_size_t(s), vel.p, dd.p, C.c_double(c["viscosity"]), pdev.p) == 0
    finally:
        if saved is None:
            os.environ.pop("VORTEX_B200_PRECISION", None)
        else:
            os.environ["VORTEX_B200_PRECISION"] = saved
        setup_conf(c, P)
    v = vel.get((cap, 2))[:s]
    d = dd.get(cap)[:s]
    xs, ys, gs = born_ref[:, 0].copy(), born_ref[:, 1].copy(), born_ref[:, 2].copy()
    ovx, ovy, od = O.velocity(p64, xs, ys, gs, s, s)
    ovx, ovy = O.diffusion(p64, xs, ys, gs, s, od, ovx, ovy)
    ovx, ovy = O.wall_diffusion(p64, pan, xs, ys, s, od, ovx, ovy)
    assert np.abs(d - od).max() <= 1e-6 * od.max()
    dv = np.hypot(v[:, 0] - ovx, v[:, 1] - ovy)
    err = dv / np.maximum(np.hypot(ovx, ovy), 1e-30)
    # the near-wall diffusion quotient is ill-conditioned: the reference's own
    # FP32 build is held to 2e-3 of the FP64 oracle on these states
    assert dv.max() <= 2e-3 and np.median(err) <= 1e-4, (dv.max(), np.percentile(err, [50, 99]))
