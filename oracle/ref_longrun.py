"""The reference's own program on the cylinder configuration from an
impulsive start: the vortex count over the run.

TEST INFRASTRUCTURE ONLY.  Runs oracle/_ref/vortex_ref (the reference's
src/main.c + src/unit_1.cu + src/kernel.cu, built with -DNO_TREE by
oracle/build_ref.sh) with the configuration of the 1000-panel cylinder at
Re 2000, dt 0.002 (core radius = panel length, same-sign collapse within
0.3 eps, window [-2, 10] x [-10, 10]; src/main.c:60-110 reads these keys),
started from a restart frame that holds one vortex of zero strength outside
the window (killed at the first step, and adding exactly zero to every sum
before that), and reads the count it logs every step in its timings
file (src/main.c:689, "<step>\tN = <count>\t...").  The count is the
checker for the library's own long run of the same configuration
(`python -m vortex_b200.runs config2`).

Why the frame: a start without one goes through incr_vort_quant, which
returns randomize_tail's value (src/unit_1.cu:554), and randomize_tail ends
without a return statement (src/unit_1.cu:488-510), so the program may stop
with "Increase ERROR!" before its first step (it did here); the restart
path calls randomize_tail without looking at its value (src/main.c:564).

    python -m oracle.ref_longrun [--steps 3000] [--every 100]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
EXE = os.path.join(HERE, "_ref", "vortex_ref")

CONF = """steps {steps}
saving_step 1000000
dt 0.002
inc_step 65536
pr_file circle1000.txt
viscosity 0.0005
rho 1.0
v_inf_x 1.0
v_inf_y 0.0
v_inf_incr_steps 0
n_of_points 20
x_max 10.0
x_min -2.0
y_max 10.0
y_min -10.0
ve_size {eps!r}
n_col 2
r_col_diff_sign 0.0
r_col_same_sign 0.3
max_ve_g 1e30
rc_x 0.0
rc_y 0.0
matrix_load 0
timings_file output/timings.txt
kadr_file Kadr000000.txt
"""


def run(steps: int, every: int) -> dict:
    if not os.path.exists(EXE):
        return {"unavailable": "oracle/_ref/vortex_ref not built (oracle/build_ref.sh needs the reference sources)"}
    sys.path.insert(0, ROOT)
    from vortex_b200 import profiles
    with tempfile.TemporaryDirectory() as wd:
        profiles.write_profile(os.path.join(wd, "circle1000.txt"), profiles.circle(1000))
        with open(os.path.join(wd, "run.conf"), "w") as fh:
            fh.write(CONF.format(steps=steps, eps=2 * math.pi * 0.5 / 1000))
        with open(os.path.join(wd, "Kadr000000.txt"), "w") as fh:   # the frame src/main.c:190-203 reads
            fh.write("1\n0 0.008000 50 0 0 0 0 0\n")
        t0 = time.perf_counter()
        r = subprocess.run([EXE, "-c", "run.conf", "-l", "3"], cwd=wd, capture_output=True, text=True)
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            return {"unavailable": f"reference program exited {r.returncode}",
                    "output_tail": (r.stdout[-1500:] + r.stderr[-500:])}
        counts = {}
        for line in open(os.path.join(wd, "output", "timings.txt")):
            parts = line.strip().split("\t")
            if len(parts) >= 2 and parts[1].lstrip().startswith("N") and "=" in parts[1]:   # "N = <count>"
                counts[int(parts[0])] = int(parts[1].split("=")[1])
    hist = [{"step": s, "n": counts[s]} for s in sorted(counts) if s % every == 0 or s == max(counts)]
    return {"config": "reference program, cylinder R=0.5, 1000 panels, impulsive start, Re 2000, dt 0.002",
            "steps": steps, "wall_s": wall, "history": hist,
            "n_final": counts[max(counts)] if counts else None,
            "n_max": max(counts.values()) if counts else None}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--every", type=int, default=100)
    a = ap.parse_args()
    print(json.dumps(run(a.steps, a.every)))


if __name__ == "__main__":
    main()
