"""Run a number of steps of the benchmark workload (used for timing and
profiling; the profiler range covers only the measured steps).

    python -m vortex_b200.runsteps --n 200000 --steps 3 --warmup 1 --precision fp32
    python -m vortex_b200.runsteps --n 1000000 --diff-cutoff 16 --stage-times 5

Workload: vortex_b200/workloads.py (1000-panel cylinder, Re = 2000,
dt = 0.002, seeded warm wake of --n vortices).  With a profiler attached that
starts with its range off (ncu --profile-from-start off), only the --steps
measured steps are captured.  --stage-times K then runs K more steps stage
by stage with events between and adds the mean stage and pair-kernel times.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time

from . import native as N
from . import workloads as wl


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=200_000)
    ap.add_argument("--panels", type=int, default=wl.PANELS)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--graph", type=int, default=1)
    ap.add_argument("--fmm", type=int, default=1)
    ap.add_argument("--diff-cutoff", type=float, default=None, help="bulk diffusion cut-off, in units of d")
    ap.add_argument("--stage-times", type=int, default=0, metavar="K")
    a = ap.parse_args()
    prec = N.PREC_FP32 if a.precision == "fp32" else N.PREC_FP64
    conf = wl.cylinder_conf(prec, a.panels, fmm=a.fmm)
    if a.diff_cutoff is not None:
        conf.diff_cutoff = a.diff_cutoff
    sim = N.Sim(conf, wl.cylinder_panels(a.panels))
    sim.set_graph(bool(a.graph))
    sim.set_particles(*wl.warm_wake(a.n, 1234))
    sim.step(a.warmup)
    sim.sync()
    rt = C.CDLL("libcudart.so.12")
    sim.pair_counts(clear=True)
    rt.cudaProfilerStart()
    t0 = time.perf_counter()
    sim.step(a.steps)
    sim.sync()
    t1 = time.perf_counter()
    rt.cudaProfilerStop()
    pc = sim.pair_counts()
    out = {"n_end": sim.count(), "steps": a.steps, "ms_per_step": 1e3 * (t1 - t0) / max(a.steps, 1),
           "precision": a.precision, "diff_cutoff": conf.diff_cutoff, "near_field_pairs": pc[0],
           "diffusion_pairs": pc[1]}
    if a.stage_times > 0:
        sim.set_timing(True)
        sim.step(a.stage_times)
        sim.sync()
        t = sim.timing()
        k = float(a.stage_times)
        out["stage_ms"] = {"birth": t[0] / k, "velocity": t[1] / k, "diffusion": t[2] / k, "wall": t[3] / k,
                           "advect_compact_collapse": t[4] / k, "biot_savart_kernel": t[5] / k,
                           "diffusion_kernel": t[6] / k, "step": t[7] / k}
    print(json.dumps(out))
    sim.close()


if __name__ == "__main__":
    main()
