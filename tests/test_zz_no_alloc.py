"""velocity_control_noalloc, the allocation-free variant of velocity_control
(include/vortex_b200_unit1.h), against velocity_control itself through the
C ABI, on two calls in a row with different sizes so that anything the first
call leaves in the shared scratch would show in the second.

Both run the plain FP64 form with the same source split, so the tolerance is
the one the unit_1 tests use for FP64 against FP64: 1e-12 relative.
"""
import ctypes as C
import math
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from tests.test_unit1_gpu import Dev, VxuConf
from vortex_b200 import native as N

pytestmark = pytest.mark.gpu

MAX_POINTS = 4096


def _setup(L):
    conf = VxuConf.in_dll(L, "conf")
    C.memset(C.addressof(conf), 0, C.sizeof(conf))
    conf.dt, conf.viscosity, conf.rho = 0.002, 5e-4, 1.0
    conf.v_inf_x = 1.0
    conf.x_min, conf.x_max, conf.y_min, conf.y_max = -2.0, 10.0, -10.0, 10.0
    conf.ve_size = 2 * math.pi * 0.5 / 1000
    conf.r_col_same_sign, conf.max_ve_g = 0.3, 1e30
    conf.n_of_points, conf.n_col, conf.birth_quant, conf.inc_step = 20, 2, 32, 8192
    assert L.init_device_conf_values() == 0


def _bind(L):
    for name in ("velocity_control", "velocity_control_noalloc"):
        f = getattr(L, name)
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_size_t]
        f.restype = C.c_int


def test_noalloc_matches_velocity_control_on_consecutive_calls():
    saved = os.environ.pop("VORTEX_B200_PRECISION", None)
    try:
        L = N.lib()
        _setup(L)
        _bind(L)
        rng = np.random.default_rng(7)
        for call, (n, npts) in enumerate([(20000, 3000), (7000, 700)]):
            pos = np.zeros((n, 3))
            pos[:, 0] = rng.uniform(0.55, 3.0, n)
            pos[:, 1] = rng.uniform(-1.0, 1.0, n)
            pos[:, 2] = rng.normal(0.0, 1e-3, n)
            cp = np.zeros((npts, 3))
            cp[:, 0] = rng.uniform(0.0, 3.5, npts)
            cp[:, 1] = rng.uniform(-1.2, 1.2, npts)
            cp[: npts // 10, :2] = pos[: npts // 10, :2]    # control points on vortices (core smoothing)
            d_pos, d_cp, d_vinf = Dev(pos.nbytes), Dev(cp.nbytes), Dev(16)
            d_pos.put(pos)
            d_cp.put(cp)
            d_vinf.put(np.array([1.0, 0.1 * call]))
            d_a, d_b = Dev(npts * 16), Dev(npts * 16)
            assert L.velocity_control(d_pos.p, d_vinf.p, n, d_cp.p, d_a.p, npts) == 0
            assert L.velocity_control_noalloc(d_pos.p, d_vinf.p, n, d_cp.p, d_b.p, npts) == 0
            a, b = d_a.get((npts, 2)), d_b.get((npts, 2))
            scale = max(1.0, float(np.abs(a).max()))
            assert np.abs(a - b).max() <= 1e-12 * scale, (call, np.abs(a - b).max())
            assert np.abs(b[:, 0] - 1.0).max() > 0.0   # the vortices act
        # beyond the stated maximum: rejected before anything is launched
        big = Dev((MAX_POINTS + 1) * 24)
        out = Dev((MAX_POINTS + 1) * 16)
        assert L.velocity_control_noalloc(d_pos.p, d_vinf.p, n, big.p, out.p, MAX_POINTS + 1) == 2
    finally:
        if saved is not None:
            os.environ["VORTEX_B200_PRECISION"] = saved


# Run in a fresh process with every module of the library loaded when the
# context is created (CUDA_MODULE_LOADING=EAGER), so that the 4 MiB array is
# already resident and lazy module loading cannot be mistaken for an
# allocation.  The first call on the device and a second one must leave the
# device's free memory exactly as it was.
_FRESH = textwrap.dedent("""
    import ctypes as C, sys
    import numpy as np
    sys.path.insert(0, {root!r})
    from tests.test_zz_no_alloc import _setup, _bind
    from tests.test_unit1_gpu import Dev, rt
    from vortex_b200 import native as N
    L = N.lib()
    assert rt().cudaFree(C.c_void_p(0)) == 0
    _setup(L)
    _bind(L)
    rng = np.random.default_rng(3)
    n, npts = 30000, 4096
    pos = np.zeros((n, 3))
    pos[:, 0] = rng.uniform(0.55, 3.0, n)
    pos[:, 1] = rng.uniform(-1.0, 1.0, n)
    pos[:, 2] = rng.normal(0.0, 1e-3, n)
    cp = np.zeros((npts, 3))
    cp[:, 0] = rng.uniform(0.0, 3.5, npts)
    cp[:, 1] = rng.uniform(-1.2, 1.2, npts)
    d_pos, d_cp, d_vinf, d_out = Dev(pos.nbytes), Dev(cp.nbytes), Dev(16), Dev(npts * 16)
    d_pos.put(pos); d_cp.put(cp); d_vinf.put(np.array([1.0, 0.0]))
    free, total = C.c_size_t(), C.c_size_t()
    def free_bytes():
        assert rt().cudaDeviceSynchronize() == 0
        assert rt().cudaMemGetInfo(C.byref(free), C.byref(total)) == 0
        return free.value
    f0 = free_bytes()
    assert L.velocity_control_noalloc(d_pos.p, d_vinf.p, n, d_cp.p, d_out.p, npts) == 0   # first call
    f1 = free_bytes()
    assert L.velocity_control_noalloc(d_pos.p, d_vinf.p, n, d_cp.p, d_out.p, npts) == 0
    f2 = free_bytes()
    print("free bytes", f0, f1, f2)
    assert f0 == f1 == f2, (f0, f1, f2)
    assert np.isfinite(d_out.get((npts, 2))).all()
""")


def test_noalloc_allocates_nothing_from_the_first_call():
    root = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
    env = dict(os.environ, CUDA_MODULE_LOADING="EAGER")
    env.pop("VORTEX_B200_PRECISION", None)
    r = subprocess.run([sys.executable, "-c", _FRESH.format(root=root)], env=env, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
