"""Record golden vectors from the reference's own CUDA build.

Runs the reference's vort_creation / Speed / Step (built unmodified from the
reference sources into oracle/_ref/libvortex_ref.so by oracle/build_ref.sh)
on a GPU, the way its src/main.c step loop calls them, and stores the state
around each stage for a few steps:

    python tests/golden/make_ref_goldens.py --out tests/golden

Workloads: the 200-panel circle of radius 0.5 (generated by
vortex_b200.profiles.circle), core radius = panel length, U = (1, 0),
nu = 1e-3, dt = 0.005, with the reference's own birth placement and 1e-12
removal threshold; "cfg1" has same-sign collapse only (ratio 0.3), "mixed"
also merges opposite signs (ratio 0.5) and caps merged strength at 0.05;
"krug1000" is the 1000-panel circle of the cylinder benchmark (the layout of
the reference's profiles/Profile_file_krug_1000.txt), nu = 5e-4, dt = 0.002,
same-sign collapse only.
Per recorded step k the file holds pre_pos, born_pos, vel, d, post_pos
(slots [0, s), s = n rounded up to 32 after birth), pre/post counts and the
post-step (d_g, Fx, Fy, M), plus probe velocities at 500 points.
"""
from __future__ import annotations

import argparse
import math
import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

from oracle import refdrv  # noqa: E402
from vortex_b200 import profiles  # noqa: E402

BASE = dict(dt=0.005, viscosity=1e-3, rho=1.0, v_inf_x=1.0, v_inf_y=0.0, x_min=-2.0, x_max=10.0,
            y_min=-10.0, y_max=10.0, n_of_points=20, n_col=2, rc_x=0.0, rc_y=0.0,
            inc_step=8192)
RUNS = {   # panels, conf overrides, steps, recorded steps
    "cfg1": (200, dict(r_col_diff_sign=0.0, r_col_same_sign=0.3, max_ve_g=1e30), 30, (1, 4, 30)),
    "mixed": (200, dict(r_col_diff_sign=0.5, r_col_same_sign=0.3, max_ve_g=0.05), 20, (2, 20)),
    "krug1000": (1000, dict(dt=0.002, viscosity=5e-4, r_col_diff_sign=0.0, r_col_same_sign=0.3, max_ve_g=1e30),
                 6, (2, 6)),
}


def run(name, out_dir):
    P, extra, steps, rec = RUNS[name]
    pan = profiles.circle(P)
    conf = dict(BASE, ve_size=2 * math.pi * 0.5 / P, **extra)
    bb = profiles.profile_bbox(pan, (conf["x_min"], conf["x_max"], conf["y_min"], conf["y_max"]))
    conf.update(profile_x_min=bb[0], profile_x_max=bb[1], profile_y_min=bb[2], profile_y_max=bb[3])
    cap = refdrv.round32(P * steps + P) + 256
    r = refdrv.RefRun(pan, conf, cap)
    out = {"conf_keys": np.array(list(conf.keys())), "conf_vals": np.array(list(conf.values()), dtype=float),
           "panels": pan.view(np.uint8)}
    py = 0.01 + 0.002 * np.arange(500)
    px = np.full(500, -0.15)
    for k in range(1, steps + 1):
        rd = {} if k in rec else None
        r.step(rd)
        if rd is not None:
            for key, val in rd.items():
                out[f"s{k}_{key}"] = np.asarray(val)
            out[f"s{k}_probe"] = r.probe(px, py)
        print(name, "step", k, "n", r.n, flush=True)
    r.close()
    path = os.path.join(out_dir, f"ref_{name}.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    ap.add_argument("--runs", default="cfg1,mixed")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    for nm in a.runs.split(","):
        run(nm, a.out)
