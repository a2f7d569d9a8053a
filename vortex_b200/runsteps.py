"""Run a number of steps of the cylinder workload (used for timing and
profiling; the profiler range covers only the measured steps).

    python -m vortex_b200.runsteps --n 200000 --steps 3 --warmup 1 --precision fp32

Workload: 1000-panel cylinder, Re = 2000, dt = 0.002 (the benchmark's), from a
seeded warm wake of --n vortices.  With a profiler attached that is started
with its range off (ncu --profile-from-start off), only the --steps measured
steps are captured.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import time

import numpy as np

from . import native as N
from . import profiles


def warm_cloud(n, seed):
    rng = np.random.default_rng(seed)
    x, y = np.empty(0), np.empty(0)
    while len(x) < n:
        m = 2 * (n - len(x)) + 1000
        xx, yy = rng.normal(2.5, 1.0, m), rng.normal(0.0, 0.5, m)
        ok = (xx > 0.5) & (xx < 4.5) & (np.abs(yy) < 1.0) & (xx * xx + yy * yy > 0.51 ** 2)
        x, y = np.concatenate([x, xx[ok]]), np.concatenate([y, yy[ok]])
    return x[:n].copy(), y[:n].copy(), rng.normal(0.0, 1e-3, n)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=200_000)
    ap.add_argument("--panels", type=int, default=1000)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--graph", type=int, default=1)
    a = ap.parse_args()
    P = a.panels
    conf = N.default_conf(dt=0.002, viscosity=5e-4, ve_size=2 * math.pi * 0.5 / P, r_col_same_sign=0.3,
                          drop_eps=1e-8, birth_offset_mode=N.BIRTH_HALF_PANEL, v_inf_incr_steps=0,
                          precision=N.PREC_FP32 if a.precision == "fp32" else N.PREC_FP64)
    sim = N.Sim(conf, profiles.circle(P))
    sim.set_graph(bool(a.graph))
    sim.set_particles(*warm_cloud(a.n, 1234))
    sim.step(a.warmup)
    sim.sync()
    rt = C.CDLL("libcudart.so.12")
    rt.cudaProfilerStart()
    t0 = time.perf_counter()
    sim.step(a.steps)
    sim.sync()
    t1 = time.perf_counter()
    rt.cudaProfilerStop()
    print(json.dumps({"n_end": sim.count(), "steps": a.steps, "ms_per_step": 1e3 * (t1 - t0) / max(a.steps, 1),
                      "precision": a.precision}))
    sim.close()


if __name__ == "__main__":
    main()
