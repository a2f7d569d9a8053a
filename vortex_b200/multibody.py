"""Many bodies on one GPU: the batched run and the served run.

Batched: a seeded population of bodies (workloads.body_spec) advanced
together.  Default form (mode "graph", vx_batch): each kernel of the step
runs once for all bodies and the batched step is one CUDA graph; the step is
timed by events on the batch's stream.  Mode "streams" (vx_step_many): every
body's own step graph launched on its own stream before the next step, timed
from a start event every body stream waits for to an end event after the
main stream waited for every body.

Served: requests drawn from the same population arrive as a Poisson process;
each asks for a number of steps; the vx_server loop admits them by slot and
device-byte budget, keeps them resident, steps all resident bodies every
tick and releases finished ones (continuous batching).

On several GPUs (one process per GPU) the population is partitioned by
body: rank r of w takes bodies / requests r, r + w, r + 2w, ... (share),
runs them on its own GPU with no exchange on the step path, and the ranks'
results are combined on the host afterwards (combine_batch, combine_serve:
throughputs add, latencies take the slowest rank).

    python -m vortex_b200.multibody batch --bodies 256 --steps 20
    python -m vortex_b200.multibody serve --requests 32
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import native as N
from . import workloads as wl


def share(count: int, rank: int = 0, world: int = 1) -> list:
    """Indices of the bodies (or requests) rank `rank` of `world` runs."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    return list(range(rank, count, world))


def combine_batch(parts: list) -> dict:
    """One batched-run record from the ranks' records: bodies, particles
    and throughputs add; the batched step takes the slowest rank."""
    out = dict(parts[0])
    for k in ("bodies", "particles_start", "particles_end", "panels_total", "body_steps_per_s",
              "particle_steps_per_s", "interactions_per_s_effective", "gpu_launches"):
        out[k] = sum(p[k] for p in parts)
    for k in ("ms_per_batched_step", "ms_p50", "ms_p99", "setup_s"):
        out[k] = max(p[k] for p in parts)
    out["batched_steps_per_s"] = min(p["batched_steps_per_s"] for p in parts)
    out["ranks"] = len(parts)
    return out


def combine_serve(parts: list) -> dict:
    """One served-run record from the ranks' records: requests, steps and
    throughputs add; latency percentiles and wall time take the slowest rank."""
    out = dict(parts[0])
    for k in ("requests", "steps_requested", "failed", "body_steps", "body_steps_per_s", "particle_steps_per_s",
              "ticks"):
        out[k] = sum(p[k] for p in parts)
    for k in ("wall_s", "step_ms_p50", "step_ms_p99", "ttc_s_p50", "ttc_s_p99"):
        out[k] = max(p[k] for p in parts)
    out["mean_resident"] = sum(p["mean_resident"] for p in parts)
    out["ranks"] = len(parts)
    return out


def make_population(bodies: int = 256, seed: int = 7, precision: int = N.PREC_FP32, device: int = 0,
                    rank: int = 0, world: int = 1):
    """This rank's share of the seeded population, created on `device`:
    (specs, sims, setup seconds)."""
    specs = [wl.body_spec(seed, i) for i in share(bodies, rank, world)]
    sims = []
    t0 = time.perf_counter()
    for sp in specs:
        conf, pan, x, y, g = wl.make_body(sp, precision)
        s = N.Sim(conf, pan, device=device)
        s.set_particles(x, y, g)
        sims.append(s)
    return specs, sims, time.perf_counter() - t0


def run_batch(bodies: int = 256, steps: int = 20, warmup: int = 3, seed: int = 7,
              precision: int = N.PREC_FP32, device: int = 0, rank: int = 0, world: int = 1,
              mode: str = "graph", population=None) -> dict:
    """The batched run of this rank's share of `bodies` seeded bodies (or of
    an existing population from make_population, which is left open)."""
    own = population is None
    specs, sims, setup_s = population if population else make_population(bodies, seed, precision, device,
                                                                           rank, world)
    bodies = len(specs)
    batch = N.Batch(sims) if mode == "graph" else None
    if batch:
        batch.step(warmup)
        batch.sync()
        stream = batch.stream()
    else:
        N.step_many(sims, warmup)
        for s in sims:
            s.sync()
        stream = 0
    counts0 = np.array([s.count() for s in sims], dtype=np.float64)
    ms = []
    launches0 = batch.info()["kernels"] if batch else sum(s.launches() for s in sims)
    host_ms = []
    for _ in range(steps):
        a, b = N.Event(), N.Event()
        if batch:
            a.record(stream)
            t0 = time.perf_counter()
            batch.step(1)
            host_ms.append(round(1e3 * (time.perf_counter() - t0), 3))
            b.record(stream)
        else:
            a.record(stream)
            for s in sims:
                N.wait_event(s.stream(), a)
            N.step_many(sims, 1)
            for s in sims:
                e = N.Event()
                e.record(s.stream())
                N.wait_event(stream, e)
            b.record(stream)
        ms.append(a.elapsed_ms(b))
    if batch:
        batch.sync()
    counts1 = np.array([s.count() for s in sims], dtype=np.float64)
    launches = (batch.info()["kernels"] if batch else sum(s.launches() for s in sims)) - launches0
    info = batch.info() if batch else None
    nmean = 0.5 * (counts0 + counts1)
    inter = float(np.sum(nmean * nmean))          # direct-sum equivalent pairs per batched step
    total_s = sum(ms) * 1e-3
    out = {"bodies": bodies, "steps": steps, "warmup": warmup, "seed": seed,
           "precision": "fp32" if precision == N.PREC_FP32 else "fp64",
           "mode": ("one launch per kernel of the step for all bodies, the batched step one CUDA graph (vx_batch)"
                    if batch else "every body's own step graph on its own stream (vx_step_many)"),
           "particles_start": int(counts0.sum()), "particles_end": int(counts1.sum()),
           "panels_total": int(sum(sp["panels"] for sp in specs)),
           "batched_steps_per_s": steps / total_s, "body_steps_per_s": bodies * steps / total_s,
           "ms_per_batched_step": float(np.mean(ms)), "ms_p50": float(np.percentile(ms, 50)),
           "ms_p99": float(np.percentile(ms, 99)), "ms_steps": [round(float(m), 3) for m in ms],
           "particle_steps_per_s": float(nmean.sum()) * steps / total_s,
           "interactions_per_s_effective": inter * steps / total_s,
           "gpu_launches": int(launches), "kernels_per_batched_step": launches / steps, "setup_s": setup_s}
    if info:
        out["host_ms_steps"] = host_ms   # host time of each batch.step(1) call (preparation and launch)
        out["graph_instantiations"] = info["graph_instantiations"]
        out["slot_table_rebuilds"] = info["rebuilds"]
        for k in ("host_grow_ms_max", "host_grow_ms_total", "host_refresh_ms_max", "host_refresh_ms_total",
                  "host_phase_ms_max"):
            out[k] = info[k]
        batch.close()
    if own:
        for s in sims:
            s.close()
    return out


def run_serve(requests: int = 32, rate: float = 50.0, budget_gb: float = 160.0, max_active: int = 256,
              seed: int = 11, precision: int = N.PREC_FP32, steps_lo: int = 50, steps_hi: int = 1000,
              device: int = 0, rank: int = 0, world: int = 1, batched: bool = True) -> dict:
    """Poisson arrivals (rate per second) of `requests` bodies of the seeded
    population, each asking for U[steps_lo, steps_hi] steps; this rank serves
    its share of them, at their arrival times."""
    u = wl.uniforms(seed, 2 * requests)
    gaps = -np.log1p(-u[:requests]) / rate
    mine = share(requests, rank, world)
    arrive = np.cumsum(gaps)[mine]
    nsteps = (steps_lo + np.floor(u[requests:] * (steps_hi - steps_lo + 1))).astype(int)[mine]
    specs = [wl.body_spec(seed, i) for i in mine]
    requests = len(mine)
    bodies = [wl.make_body(sp, precision) for sp in specs]
    srv = N.Server(int(budget_gb * 1e9), max_active=max_active, device=device)
    srv.set_batched(batched)
    ids = [None] * requests
    t0 = time.perf_counter()
    nxt = 0
    while True:
        now = time.perf_counter() - t0
        while nxt < requests and arrive[nxt] <= now:
            conf, pan, x, y, g = bodies[nxt]
            ids[nxt] = srv.submit(conf, pan, x, y, g, int(nsteps[nxt]))
            nxt += 1
        resident, queued = srv.tick()
        if resident == 0 and queued == 0:
            if nxt == requests:
                break            # every request submitted has finished or failed
            time.sleep(max(0.0, arrive[nxt] - (time.perf_counter() - t0)))
    wall = time.perf_counter() - t0
    st = srv.stats()
    res = [srv.result(i) for i in ids]
    srv.close()
    return {"requests": requests, "rate_per_s": rate, "budget_gb": budget_gb, "max_active": max_active,
            "stepping": ("resident bodies batched step by step (vx_batch: one launch per kernel of the step)"
                         if batched else "each resident body on its own stream"),
            "seed": seed, "precision": "fp32" if precision == N.PREC_FP32 else "fp64",
            "steps_requested": int(nsteps.sum()), "failed": sum(r["state"] == "failed" for r in res),
            "failures": sorted({r["error"] for r in res if r["state"] == "failed"})[:4],
            "wall_s": wall, "step_ms_p50": st["step_ms_p50"], "step_ms_p99": st["step_ms_p99"],
            "ttc_s_p50": st["ttc_s_p50"], "ttc_s_p99": st["ttc_s_p99"], "mean_resident": st["mean_resident"],
            "body_steps": st["body_steps"], "body_steps_per_s": st["body_steps"] / wall,
            "particle_steps_per_s": st["particle_steps"] / wall, "ticks": st["ticks"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("mode", choices=["batch", "serve"])
    ap.add_argument("--bodies", type=int, default=256)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--requests", type=int, default=32)
    ap.add_argument("--rate", type=float, default=50.0)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--stepping", default="graph", choices=["graph", "streams"],
                    help="batch: one batched graph per step (graph) or every body's graph on its own stream")
    a = ap.parse_args()
    prec = N.PREC_FP32 if a.precision == "fp32" else N.PREC_FP64
    if a.mode == "batch":
        print(json.dumps(run_batch(a.bodies, a.steps, a.warmup, precision=prec, mode=a.stepping)))
    else:
        print(json.dumps(run_serve(a.requests, a.rate, precision=prec)))


if __name__ == "__main__":
    main()
