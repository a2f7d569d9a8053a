"""Autotuner of the bulk form's Biot-Savart: direct FP32 sum or quadtree FMM,
and the quadtree's vortices per leaf, chosen by timing the velocity stage of
the body's current state on its own GPU.

    python -m vortex_b200.autotune --n 1000000          # tune the benchmark wake
    python -m vortex_b200.autotune --crossover          # direct vs FMM over N

The expansion order is fixed at 16 terms: with leaves at least eps wide and
the interaction list one cell away, 16 terms keep the far field within the
2e-5 max|V| bound the bulk-form tests state.
"""
from __future__ import annotations

import argparse
import json

from . import native as N
from . import workloads as wl

LEAVES = (8, 16, 32, 64, 128, 256)


def time_velocity(sim: N.Sim, reps: int = 3, device: int = 0) -> float:
    """Median device ms of the velocity stage, timed with CUDA events on the
    sim's own stream."""
    st = sim.stream()
    sim.stage("velocity")      # warm (graph-free stage path, buffers sized)
    ms = []
    for _ in range(reps):
        a, b = N.Event(), N.Event()
        a.record(st)
        sim.stage("velocity")
        b.record(st)
        ms.append(a.elapsed_ms(b))
    ms.sort()
    return ms[len(ms) // 2]


def tune(sim: N.Sim, leaves=LEAVES, direct: bool = True, reps: int = 3, device: int = 0) -> dict:
    """Time every candidate on the sim's current particles and keep the
    fastest (the sim is left set to it).  Returns the table and the choice."""
    table = []
    if direct:
        sim.set_fmm(False)
        table.append({"form": "direct", "leaf": None, "ms": time_velocity(sim, reps, device)})
    for leaf in leaves:
        sim.set_fmm(True, leaf)
        table.append({"form": "fmm", "leaf": leaf, "ms": time_velocity(sim, reps, device)})
    best = min(table, key=lambda r: r["ms"])
    sim.set_fmm(best["form"] == "fmm", best["leaf"] or 8)
    return {"table": table, "best": best}


def crossover(ns=(10_000, 30_000, 100_000, 300_000, 1_000_000), device: int = 0) -> list:
    """Direct versus the best-leaf FMM on the benchmark wake at several N."""
    out = []
    pan = wl.cylinder_panels()
    for n in ns:
        sim = N.Sim(wl.cylinder_conf(N.PREC_FP32), pan, device=device)
        sim.set_particles(*wl.warm_wake(int(n), 1234))
        r = tune(sim, device=device)
        d = next(t["ms"] for t in r["table"] if t["form"] == "direct")
        f = min((t for t in r["table"] if t["form"] == "fmm"), key=lambda t: t["ms"])
        out.append({"n": int(n), "direct_ms": d, "fmm_ms": f["ms"], "fmm_leaf": f["leaf"],
                    "faster": "fmm" if f["ms"] < d else "direct"})
        sim.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--crossover", action="store_true")
    a = ap.parse_args()
    if a.crossover:
        print(json.dumps(crossover()))
        return
    sim = N.Sim(wl.cylinder_conf(N.PREC_FP32), wl.cylinder_panels())
    sim.set_particles(*wl.warm_wake(a.n, 1234))
    print(json.dumps(tune(sim)))
    sim.close()


if __name__ == "__main__":
    main()
