"""Drop-in check: the reference's own host driver (its src/main.c, unchanged)
linked against libvortex_b200.so instead of its src/unit_1.cu + src/kernel.cu
(oracle/_ref/vortex_linkswap, built by oracle/build_ref.sh) runs the same
.conf/profile/restart-frame inputs as the reference's whole program
(oracle/_ref/vortex_ref) and writes the same output files with agreeing
contents.

Both runs restart from a Kadr frame (kadr_file): the reference's
randomize_tail (src/unit_1.cu:488-509) has no return statement, so the fresh
start path, which checks that value through incr_vort_quant, aborts the
reference's own program; the restart path ignores it.  inc_step is large
enough that no growth happens during the run.

The reference computes its pair sums in FP32 and this library in FP64, so
the comparison allows FP32-level differences: panel matrix files (printed to
6 decimals) and the first saved frame agree to 2e-6, the force history to
1 % of its scale over the first steps (a force is a difference of impulses,
so FP32 rounding shows up there first), particle counts to 3 %.
"""
import math
import os
import subprocess

import numpy as np
import pytest

from vortex_b200 import profiles

pytestmark = pytest.mark.gpu
ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
REF = os.path.join(ROOT, "oracle", "_ref", "vortex_ref")
SWAP = os.path.join(ROOT, "oracle", "_ref", "vortex_linkswap")

CONF = """steps 12
saving_step 6
dt 0.005
inc_step 65536
pr_file circle200.txt
viscosity 0.001
rho 1.0
v_inf_x 1.0
v_inf_y 0.0
v_inf_incr_steps 00
n_of_points 20
x_max 10.0
x_min -2.0
y_max 10
y_min -10
ve_size {eps}
n_col 2
r_col_diff_sign 0.5
r_col_same_sign 0.3
max_ve_g 0.05
rc_x 0.0
rc_y 0.0
matrix_load 0
timings_file output/timings.txt
kadr_file Kadr000012.txt
"""


def start_frame(path, n=3000, seed=5):
    """A restart frame in the reference's Kadr format (src/main.c:175-188)."""
    rng = np.random.default_rng(seed)
    th = rng.uniform(0, 2 * math.pi, n)
    r = 0.5 + 0.004 + rng.exponential(0.06, n)
    x, y = r * np.cos(th), r * np.sin(th)
    g = rng.normal(0, 2e-3, n)
    with open(path, "w") as fh:
        fh.write(f"{n}\n")
        for i in range(n):
            fh.write(f"{i} 0.008000 {x[i]:f} {y[i]:f} 0.000000 0.000000 0.000000 {g[i]:f}\n")


def run(exe, wd, inc=65536):
    os.makedirs(wd, exist_ok=True)
    profiles.write_profile(os.path.join(wd, "circle200.txt"), profiles.circle(200))
    with open(os.path.join(wd, "run.conf"), "w") as fh:
        fh.write(CONF.format(eps=2 * math.pi * 0.5 / 200).replace("inc_step 65536", f"inc_step {inc}"))
    start_frame(os.path.join(wd, "Kadr000012.txt"))
    r = subprocess.run([exe, "-c", "run.conf", "-l", "1"], cwd=wd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


def counts(wd):
    out = {}
    for line in open(os.path.join(wd, "output", "timings.txt")):
        parts = line.split("\t")
        out[int(parts[0])] = int(parts[1].split("=")[1])
    return out


def numbers(path):
    return np.array(open(path).read().split(), dtype=float)


@pytest.mark.skipif(not (os.path.exists(REF) and os.path.exists(SWAP)), reason="oracle/_ref binaries not built")
def test_reference_driver_runs_on_this_library(tmp_path):
    a, b = str(tmp_path / "ref"), str(tmp_path / "swap")
    run(REF, a)
    run(SWAP, b)
    for f in ("L.txt", "M.txt", os.path.join("output", "kadrs", "Kadr000012.txt")):
        fa, fb = numbers(os.path.join(a, f)), numbers(os.path.join(b, f))
        assert fa.shape == fb.shape, f
        assert np.abs(fa - fb).max() <= 2e-6, f
    Fa = np.loadtxt(os.path.join(a, "output", "F_p.txt"))
    Fb = np.loadtxt(os.path.join(b, "output", "F_p.txt"))
    assert Fa.shape == Fb.shape and np.array_equal(Fa[:, 0], Fb[:, 0])
    scale = np.abs(Fa[1:6, 1:3]).max()
    assert scale > 0
    assert np.abs(Fa[1:6, 1:3] - Fb[1:6, 1:3]).max() <= 1e-2 * scale
    ca, cb = counts(a), counts(b)
    assert ca.keys() == cb.keys() and len(ca) >= 12
    for k in ca:
        assert abs(ca[k] - cb[k]) <= 0.03 * ca[k] + 2
    for f in ("Kadr000018.txt", "Kadr000024.txt"):
        assert os.path.exists(os.path.join(b, "output", "kadrs", f))
    assert os.path.exists(os.path.join(b, "output", "vels", "contr_Vel000018.txt"))


@pytest.mark.skipif(not os.path.exists(SWAP), reason="oracle/_ref binaries not built")
def test_reference_driver_grows_the_store_through_this_library(tmp_path):
    """The reference's driver with inc_step 512: its step loop calls
    incr_vort_quant (allocate_arrays, randomize_tail) whenever the padded
    count outgrows the store, here on the first step and several times
    after (3000 restart vortices, 200 born per step).  Growth keeps every
    slot and fills the new tail far from every vortex, so the run writes
    the same frames, forces and counts, to the last printed digit, as the
    run whose store never grows (inc_step 65536).  (The reference's own
    randomize_tail returns no value, which its driver takes as a failure at
    the first growth, so only the library is run here.)"""
    a, b = str(tmp_path / "big"), str(tmp_path / "grow")
    run(SWAP, a, inc=65536)
    run(SWAP, b, inc=512)
    for f in ("M.txt", os.path.join("output", "kadrs", "Kadr000018.txt"),
              os.path.join("output", "kadrs", "Kadr000024.txt"), os.path.join("output", "F_p.txt")):
        fa, fb = numbers(os.path.join(a, f)), numbers(os.path.join(b, f))
        assert fa.shape == fb.shape and np.array_equal(fa, fb), f
    assert counts(a) == counts(b)
