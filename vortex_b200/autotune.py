"""Autotuner of the bulk form's Biot-Savart: direct FP32 sum or quadtree FMM,
the quadtree's vortices per leaf and its expansion order, chosen by timing
the velocity stage of the body's current state on its own GPU.

    python -m vortex_b200.autotune --n 1000000          # tune the benchmark wake
    python -m vortex_b200.autotune --crossover          # direct vs FMM over N

Every FMM setting is first checked against the direct sum at a sample of
the body's own vortices (the probe kernel's direct FP32 sum at their
positions, 4096 of them): settings whose velocity error exceeds the bulk
form's stated bound, 2e-5 of the largest velocity, are rejected before
timing.  Of the rest the fastest is kept.  Times are CUDA events on the
body's own stream (median of `reps` stage launches).
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import native as N
from . import workloads as wl

LEAVES = (8, 16, 32, 64, 128, 256)
ORDERS = (8, 12, 16, 20)
BOUND = 2e-5


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


class _Check:
    """Direct-sum velocities at a seeded sample of the body's vortices."""

    def __init__(self, sim: N.Sim, points: int = 4096, seed: int = 5):
        x, y, _ = sim.particles()
        n = len(x)
        rng = np.random.default_rng(seed)
        self.idx = np.sort(rng.choice(n, size=min(points, n), replace=False)) if n else np.zeros(0, int)
        self.ref = sim.probe(x[self.idx], y[self.idx]) if n else (np.zeros(0), np.zeros(0))
        self.vmax = float(np.hypot(*self.ref).max()) if n else 1.0

    def error(self, sim: N.Sim) -> float:
        """max |V - V_direct| / max |V_direct| over the sample after the
        velocity stage that just ran."""
        if len(self.idx) == 0:
            return 0.0
        vx, vy, _ = sim.velocity()
        return float(np.hypot(vx[self.idx] - self.ref[0], vy[self.idx] - self.ref[1]).max() / self.vmax)


def tune(sim: N.Sim, leaves=LEAVES, orders=ORDERS, direct: bool = True, reps: int = 3, device: int = 0,
         bound: float = BOUND) -> dict:
    """Time every accurate candidate on the sim's current particles and keep
    the fastest (the sim is left set to it).  Returns the table and the
    choice."""
    check = _Check(sim)
    table = []
    if direct:
        sim.set_fmm(False)
        table.append({"form": "direct", "leaf": None, "p": None, "ms": time_velocity(sim, reps, device),
                      "error": check.error(sim)})
    for p in orders:
        for leaf in leaves:
            sim.set_fmm(True, leaf, p)
            sim.stage("velocity")
            err = check.error(sim)
            row = {"form": "fmm", "leaf": leaf, "p": p, "error": err}
            if err <= bound:
                row["ms"] = time_velocity(sim, reps, device)
            else:
                row["rejected"] = f"velocity error {err:.2e} of max |V| above {bound:g}"
            table.append(row)
    ok = [r for r in table if "ms" in r]
    best = min(ok, key=lambda r: r["ms"])
    if best["form"] == "fmm":
        sim.set_fmm(True, best["leaf"], best["p"])
    else:
        sim.set_fmm(False)
    return {"table": table, "best": best, "bound": bound, "check_points": int(len(check.idx))}


def crossover(ns=(10_000, 30_000, 100_000, 300_000, 1_000_000), device: int = 0, orders=ORDERS,
              leaves=(16, 32, 64), reps: int = 2) -> list:
    """Direct versus the best accurate FMM setting on the benchmark wake at
    several N."""
    out = []
    pan = wl.cylinder_panels()
    for n in ns:
        sim = N.Sim(wl.cylinder_conf(N.PREC_FP32), pan, device=device)
        sim.set_particles(*wl.warm_wake(int(n), 1234))
        r = tune(sim, leaves=leaves, orders=orders, device=device, reps=reps)
        d = next(t["ms"] for t in r["table"] if t["form"] == "direct")
        f = min((t for t in r["table"] if t["form"] == "fmm" and "ms" in t), key=lambda t: t["ms"])
        out.append({"n": int(n), "direct_ms": d, "fmm_ms": f["ms"], "fmm_leaf": f["leaf"], "fmm_p": f["p"],
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
