"""The command-line driver (vortex_b200/bin/vortex, built from
vortex_b200/csrc/vortex_cli.cpp) with the reference program's interface.

* Restart from a Kadr frame, against the reference's own whole program
  (oracle/_ref/vortex_ref) on the same .conf and frame: the same output files
  with the tolerances of the link-swap test (the reference sums its pairs in
  FP32, this library in FP64): matrix files and the first frame to 2e-6, the
  force history's first steps to 1 % of its scale, counts to 3 %.
* Fresh start (which the reference's own program cannot do): the counts in
  the timings file and the last frame match the native API stepping the same
  configuration; matrix_load 1 reads back the M.txt the first run wrote.
"""
import math
import os
import subprocess

import numpy as np
import pytest

from tests.test_linkswap_gpu import CONF, REF, counts, numbers, start_frame
from vortex_b200 import native as N
from vortex_b200 import profiles

pytestmark = pytest.mark.gpu
ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
CLI = os.path.join(ROOT, "vortex_b200", "bin", "vortex")
EPS = 2 * math.pi * 0.5 / 200


def run_cli(wd, conf_text, frame=True):
    os.makedirs(wd, exist_ok=True)
    profiles.write_profile(os.path.join(wd, "circle200.txt"), profiles.circle(200))
    with open(os.path.join(wd, "run.conf"), "w") as fh:
        fh.write(conf_text)
    if frame:
        start_frame(os.path.join(wd, "Kadr000012.txt"))
    r = subprocess.run([CLI, "-c", "run.conf", "-l", "1"], cwd=wd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


@pytest.mark.skipif(not os.path.exists(CLI), reason="CLI not built")
@pytest.mark.skipif(not os.path.exists(REF), reason="oracle/_ref/vortex_ref not built")
def test_cli_restart_matches_reference_program(tmp_path):
    a, b = str(tmp_path / "ref"), str(tmp_path / "cli")
    conf = CONF.format(eps=EPS)
    run_cli(b, conf)
    os.makedirs(a, exist_ok=True)
    profiles.write_profile(os.path.join(a, "circle200.txt"), profiles.circle(200))
    with open(os.path.join(a, "run.conf"), "w") as fh:
        fh.write(conf)
    start_frame(os.path.join(a, "Kadr000012.txt"))
    r = subprocess.run([REF, "-c", "run.conf", "-l", "1"], cwd=a, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0
    for f in ("L.txt", "M.txt", os.path.join("output", "kadrs", "Kadr000012.txt")):
        fa, fb = numbers(os.path.join(a, f)), numbers(os.path.join(b, f))
        assert fa.shape == fb.shape, f
        assert np.abs(fa - fb).max() <= 2e-6, f
    Fa = np.loadtxt(os.path.join(a, "output", "F_p.txt"))
    Fb = np.loadtxt(os.path.join(b, "output", "F_p.txt"))
    assert Fa.shape == Fb.shape and np.array_equal(Fa[:, 0], Fb[:, 0])
    scale = np.abs(Fa[1:6, 1:3]).max()
    assert np.abs(Fa[1:6, 1:3] - Fb[1:6, 1:3]).max() <= 1e-2 * scale
    ca, cb = counts(a), counts(b)
    assert ca.keys() == cb.keys() and len(ca) >= 12
    for k in ca:
        assert abs(ca[k] - cb[k]) <= 0.03 * ca[k] + 2
    for f in ("Kadr000018.txt", "Kadr000024.txt"):
        assert os.path.exists(os.path.join(b, "output", "kadrs", f))
    vel = np.loadtxt(os.path.join(b, "output", "vels", "contr_Vel000018.txt"))
    assert vel.shape == (500 * 6, 5) and np.abs(vel[:, 3]).max() > 0


@pytest.mark.skipif(not os.path.exists(CLI), reason="CLI not built")
def test_cli_fresh_start_matches_native_api(tmp_path):
    conf = CONF.format(eps=EPS).replace("kadr_file Kadr000012.txt\n", "")
    wd = str(tmp_path / "fresh")
    run_cli(wd, conf, frame=False)
    c = counts(wd)
    assert sorted(c) == list(range(13))
    # the same configuration through the native API
    cf = N.read_conf(os.path.join(wd, "run.conf"))
    pan = N.read_profile(os.path.join(wd, "circle200.txt"))
    sim = N.Sim(cf, pan)
    for k in range(12):
        sim.step(1)
        if k + 1 < 12:
            # the timings line of step k+1 is written after that step's birth
            assert c[k + 1] == sim.count() + len(pan)
    n = sim.count()
    assert c[12] == n
    frame = np.loadtxt(os.path.join(wd, "output", "kadrs", "Kadr000012.txt"), skiprows=1)
    x, y, g = sim.particles()
    assert frame.shape == (n, 8)
    assert np.abs(frame[:, 2] - x).max() <= 1e-6 and np.abs(frame[:, 3] - y).max() <= 1e-6
    assert np.abs(frame[:, 7] - g).max() <= 1e-6
    F = np.loadtxt(os.path.join(wd, "output", "F_p.txt"))
    f = sim.forces()
    assert F.shape == (13, 4) and np.abs(F[-1, 1:] - f[1:]).max() <= 1e-6 * max(1.0, np.abs(f[1:]).max())
    sim.close()
    # matrix_load 1 reads the M.txt written above (6 decimals): the run goes
    # through and tracks the generated one closely
    conf2 = conf.replace("matrix_load 0", "matrix_load 1")
    with open(os.path.join(wd, "run.conf"), "w") as fh:
        fh.write(conf2)
    r = subprocess.run([CLI, "-c", "run.conf", "-l", "1"], cwd=wd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    c2 = counts(wd)
    assert abs(c2[12] - c[12]) <= 0.02 * c[12]
