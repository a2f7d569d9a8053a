"""Benchmark of the vortex-element time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n N0]

Workload (the cylinder configuration the headline metric is quoted on): a
circle of radius 0.5 with 1000 equal panels, U = (1, 0), Re = 2000
(nu = 5e-4), dt = 0.002, core radius = panel length, birth half a panel off
the wall, same-sign collapse within 0.3 eps, |G| < 1e-8 dropped, started from
a seeded warm wake of N0 = 1e6 vortices (vortex_b200/workloads.py).  One step
= birth, Biot-Savart + 3-nearest, vortex and wall diffusion, convection with
absorption, force sums, compaction, collapse.

Our arm times the FP32-bulk form (headline: quadtree FMM Biot-Savart,
neighbour-list diffusion) and the plain FP64 form (direct sums) on the same
GPU; value = whole-job steps/s.  Multi-GPU is weak scaling: each rank
advances its own body, no collective in the step; the slowest rank's device
time is the job time.  The reference arm (--impl reference) times the CPU
oracle (OpenMP C transcription of the reference formulas) on the host cores
on a bounded sample of the same step and extrapolates to a full step.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "steps/sec & particle-interactions/sec FP32-bulk vs FP64 plain, same GPU; p50/p99 latency"
P_PANELS = 1000
FLOP_PER_PAIR_BS = 12      # Biot-Savart pair: sub x2, |r|^2 3, max 1, rcp+mul 2, 2 fma 4
FLOP_PER_PAIR_DIFF = 18    # vortex diffusion pair


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [t.strip() for t in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                mhz.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(mhz)}


def job_time_ms(local_ms: float, dist: bool, device: int = 0) -> float:
    """The job's time: the slowest rank's device time (max over ranks)."""
    if not dist:
        return local_ms
    import torch
    on_gpu = torch.distributed.get_backend() == "nccl"
    t = torch.tensor([local_ms], dtype=torch.float64, device=f"cuda:{device}" if on_gpu else "cpu")
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def workload_config(args, world: int) -> dict:
    """The workload both arms run (identical in both JSON lines)."""
    return {"workload": "cylinder R=0.5, 1000 panels, Re=2000 (nu=5e-4), dt=0.002, core radius = panel length, "
                        f"seeded warm wake N0={args.n} vortices per GPU; one step = birth, Biot-Savart + "
                        "3-nearest, vortex and wall diffusion, convection with absorption, force sums, compaction, "
                        "collapse",
            "panels": P_PANELS, "n_particles_start": args.n,
            "l2": "our arm: flushed between timed steps (256 MiB write); reference arm: host caches",
            "parallelism": f"{world} independent bodies (one per GPU)"}


# Algorithmic DRAM bytes per particle of the memory-bound kernels of a step
# (FP64 SoA state, 4-byte keys and indices, float4 sorted copies); the
# pair kernels are compute-bound and reported in `roofline`.
HBM_BYTES = {
    "k_advect": (64, "read x, y, G, Vx, Vy; write x, y, G"),
    "k_fmm_prep": (16, "read x, y"),
    "k_fmm_leafid": (24, "read x, y; write leaf key and index"),
    "k_cg_prep": (24, "read x, y, d"),
    "k_cg_cellid": (24, "read x, y; write cell key and index"),
    "k_bk_place": (12, "read key; write key and index at the bucket slot"),
    "k_bk_order": (8, "read and write the bucket's indices"),
    "k_fmm_gather": (48, "read order index and key, x, y, G; write float4"),
    "k_cg_gather": (56, "read order index and key, x, y, G, d; write float4"),
    "k_col_prep": (16, "read x, y"),
    "k_col_count": (32, "read x, y; write cell id, in-count and the two merge flags"),
    "k_col_scatter": (64, "read cell id, cell start, x, y, G; write the 32-byte cell-sorted record"),
    "k_col_query<2>": (36, "read the cell-sorted record (x, y, G, index); write COL"),
    "k_col_query<1>": (36, "read the cell-sorted record (x, y, G, index); write COL"),
    "k_cmp_count": (8, "read G"),
    "k_cmp_classify": (8, "read G"),
}


def roofline_hbm(kt: dict, steps: int, n: float, peak_gbs: float) -> list:
    """Per-kernel achieved DRAM bandwidth of the memory-bound passes from the
    per-kernel event times of `steps` instrumented steps at about n vortices."""
    out = []
    for name, (ms, launches) in kt.items():
        if name not in HBM_BYTES or ms <= 0:
            continue
        bpp, what = HBM_BYTES[name]
        b = bpp * n * launches / steps
        t = ms / steps
        gbs = b / (t * 1e-3) / 1e9
        out.append({"kernel": name, "launches_per_step": launches / steps, "ms_per_step": t,
                    "bytes_per_step": b, "bytes_per_particle": bpp, "bytes_counted": what,
                    "achieved_gbs": gbs, "frac": gbs / peak_gbs})
    out.sort(key=lambda r: -r["ms_per_step"])
    return out


def autotune_leaves():
    from vortex_b200 import autotune
    return autotune.LEAVES


def autotune_orders():
    from vortex_b200 import autotune
    return autotune.ORDERS


def measured_peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return json.load(open(path))
    except (OSError, ValueError):
        return {}


def guarded(what, fn, *a, **kw):
    """An optional leg of the line: its record, or the error it raised (the
    headline keys never depend on it)."""
    try:
        return fn(*a, **kw)
    except Exception as e:   # noqa: BLE001 - reported in the line
        import traceback
        traceback.print_exc(file=sys.stderr)
        return {"error": f"{what}: {type(e).__name__}: {e}"[:500]}


def pinned(n, rt):
    p = C.c_void_p()
    if rt.cudaHostAlloc(C.byref(p), C.c_size_t(max(8 * n, 8)), 0) != 0:
        raise RuntimeError("cudaHostAlloc failed")
    return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(n,)), p


def run_ours(args, rank, world, device):
    import torch
    from vortex_b200 import native as Nt
    from vortex_b200 import workloads as wl

    torch.cuda.set_device(device)
    dist = world > 1
    pan = wl.cylinder_panels(P_PANELS)
    x0, y0, g0 = wl.warm_wake(args.n, seed=1234 + rank)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{device}")

    def barrier():
        if dist:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def timed_steps(sim, K, W, tune=False, instrumented=0):
        """W untimed steps, then K steps each bracketed by events on the
        handle's stream with an L2 flush between steps.  With instrumented > 0
        the K steps run as a user's do (the captured step graph) and the
        per-stage and per-kernel event times come from `instrumented` further
        steps launched stage by stage with events between (outside the timed
        region); with 0 the K timed steps themselves carry the events."""
        stream = torch.cuda.ExternalStream(sim.stream(), device=f"cuda:{device}")
        sim.step(W)
        sim.sync()
        tuned = None
        if tune:
            # untimed: the autotuner picks direct or FMM and the leaf size on
            # this state, then two more steps re-capture the step graph
            from vortex_b200 import autotune
            tres = autotune.tune(sim, reps=2, device=device)
            tuned = tres["best"]
            tuned["rejected"] = sum(1 for r in tres["table"] if "rejected" in r)
            tuned["candidates"] = len(tres["table"])
            sim.step(2)
            sim.sync()
        sim.set_timing(instrumented == 0)
        sim.pair_counts(clear=True)
        launches0 = sim.launches()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
        nvec = []
        barrier()
        for k in range(K):
            with torch.cuda.stream(stream):
                flush.zero_()
            nvec.append(sim.state()["n"] + P_PANELS)    # particles after this step's birth
            ev[k][0].record(stream)
            sim.step(1)
            ev[k][1].record(stream)
        barrier()
        ms = [a.elapsed_time(b) for a, b in ev]
        pc = sim.pair_counts()
        launches = sim.launches() - launches0
        kt, pct = K, pc
        if instrumented > 0:
            sim.set_timing(True)
            sim.pair_counts(clear=True)
            for _ in range(instrumented):
                with torch.cuda.stream(stream):
                    flush.zero_()
                sim.step(1)
            sim.sync()
            kt, pct = instrumented, sim.pair_counts()
        t = sim.timing()
        sim.set_timing(False)
        return ms, t, launches, nvec, pc, tuned, kt, pct

    # ---- FP32 bulk (headline) ------------------------------------------
    sim = Nt.Sim(wl.cylinder_conf(Nt.PREC_FP32, P_PANELS), pan, device=device)
    sim.set_particles(x0, y0, g0)
    clocks = ClockSampler(device)
    clocks.start()
    ms, tst, launches, nvec, pc, tuned, KT, pct = timed_steps(sim, args.steps, args.warmup,
                                                             tune=not args.no_autotune, instrumented=5)
    ck = clocks.stop()
    total_ms = job_time_ms(float(sum(ms)), dist, device)
    n_end = sim.count()
    K = args.steps
    # dominant pair kernel of the bulk step, timed by events around it
    kernels = {
        "k_fmm_near (Biot-Savart near field + 3-nearest + far-field evaluation)":
            (tst[5] / KT, pct[0] / KT, FLOP_PER_PAIR_BS),
        "k_diff_cells (vortex diffusion over neighbour lists)":
            (tst[6] / KT, pct[1] / KT, FLOP_PER_PAIR_DIFF),
    }
    kname, (kms, kpairs, kflop) = max(kernels.items(), key=lambda kv: kv[1][0])
    tree = sim.tree_info()
    # per-kernel device times of three further instrumented steps (the
    # memory-bound passes' bandwidth)
    n_kt = sim.count()
    kt = sim.kernel_times(3)
    # ---- end to end through the C ABI with host buffers -------------------
    rt = C.CDLL("libcudart.so.12")
    n_now = sim.count()
    room = n_now + P_PANELS * 12 + 4096      # at most P births per step
    hx, _px = pinned(room, rt)
    hy, _py = pinned(room, rt)
    hg, _pg = pinned(room, rt)
    xs, ys, gs = sim.particles()
    e2e_steps = max(3, min(10, K))
    e2e_t = []
    bi = bo = 0
    # two pinned buffer sets: a step reads its input from one and writes its
    # result into the other, which is the next step's input
    ox, _qx = pinned(room, rt)
    oy, _qy = pinned(room, rt)
    og, _qg = pinned(room, rt)
    m = len(xs)
    hx[:m], hy[:m], hg[:m] = xs, ys, gs
    bufs = [(hx, hy, hg), (ox, oy, og)]
    for k in range(e2e_steps):
        (ix, iy, ig), (wx, wy, wg) = bufs[k % 2], bufs[(k + 1) % 2]
        t0 = time.perf_counter()
        sim.set_particles(ix[:m], iy[:m], ig[:m])
        sim.step(1)
        f = sim.forces()
        m_out = sim.particles_into(wx, wy, wg)
        e2e_t.append(time.perf_counter() - t0)
        bi += 24 * m
        bo += 24 * m_out + f.nbytes
        m = m_out
    sim.close()
    # ---- plain FP64 on the same workload ------------------------------------
    fp64 = None
    if not args.skip_fp64:
        sim64 = Nt.Sim(wl.cylinder_conf(Nt.PREC_FP64, P_PANELS), pan, device=device)
        sim64.set_particles(x0, y0, g0)
        ms64, t64, _, _, _, _, _, _ = timed_steps(sim64, args.fp64_steps, 1)
        sim64.close()
        fp64 = {"steps_per_s": 1e3 * len(ms64) / sum(ms64), "ms_per_step": float(np.mean(ms64)),
                "bs_pair_kernel_ms": t64[5] / len(ms64), "diffusion_pair_kernel_ms": t64[6] / len(ms64),
                "form": "direct O(N^2) sums in FP64"}
    peak32_scalar = Nt.measure_peak(device, fp64=False)
    peak32_packed = Nt.measure_peak(device, mode=2)   # fma.rn.f32x2, two FMAs per instruction
    peak32 = max(peak32_scalar, peak32_packed)
    mufu = Nt.measure_peak(device, mode=3)        # 1e12 (rsqrt + ex2) units per second
    multi = multibody_runs(args, device, rank, world) if args.multibody else None
    cross = None
    if args.crossover and rank == 0:
        from vortex_b200 import autotune
        cross = guarded("crossover", autotune.crossover, device=device)
    plate = guarded("plate leg", plate_leg, args, device) if args.plate_steps > 0 and rank == 0 else None
    if rank != 0:
        return None
    value = world * 1e3 * K / total_ms
    mp = measured_peaks()
    hbm_peak = float(mp.get("hbm_gbs") or 6650.0)
    hbm_src = "MEASURED_PEAKS.json hbm_gbs (copy bandwidth measured on this pool)" if mp.get("hbm_gbs") else \
        "fallback 6.65 TB/s (earlier measurement on this pool)"
    eff = float(np.mean([n * ((n + 31) // 32 * 32) for n in nvec]))
    achieved = kflop * kpairs / (kms * 1e-3) / 1e12
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        tj = json.load(open(tpath)).get(kname.split()[0])
        if tj and tj.get("bytes_per_pair") is not None:
            traffic = tj["bytes_per_pair"] * kpairs
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "steps/s",
        "n_gpus": world,
        "steps": K,
        "warmup": args.warmup,
        "ms_per_step": total_ms / K,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp32",
        "data": "synthetic (seeded warm wake on a jittered lattice; generated circle profile)",
        "config": workload_config(args, world),
        "run": {"n_particles_end": int(n_end),
                "form": "FP32-bulk: FP32 pair sums with FP64 accumulation, FP64 expansions, panel solve, forces "
                        "and positions",
                "launch": "each timed step replays the step's CUDA graph (vx_step, as a user's call does)",
                "biot_savart": (f"autotuned before timing over direct and FMM (leaf {list(autotune_leaves())}, "
                                f"p {list(autotune_orders())}; {tuned['rejected']} of {tuned['candidates']} "
                                f"settings rejected by the 2e-5 max|V| check): {tuned['form']}"
                                + (f", {tuned['leaf']} vortices per leaf, {tuned['p']} terms"
                                   if tuned['form'] == 'fmm' else "")
                                if tuned else "FMM, 32 vortices per leaf, 16 terms (default)")},
        "particle_interactions_per_s": {"effective": world * eff * 1e3 * K / total_ms,
                                        "executed": world * (pc[0] + pc[1]) / (total_ms * 1e-3),
                                        "effective_definition": "N_targets x N_sources per step (direct-sum equivalent)",
                                        "executed_definition": "near-field + diffusion pair evaluations"},
        "latency_ms": {"p50": float(np.percentile(ms, 50)), "p99": float(np.percentile(ms, 99)),
                       "steps": [round(float(t), 3) for t in ms]},
        "stage_ms": {"birth": tst[0] / KT, "velocity": tst[1] / KT, "diffusion": tst[2] / KT,
                     "wall": tst[3] / KT, "advect_compact_collapse": tst[4] / KT,
                     "measured_on": f"{KT} further steps launched stage by stage with events between"},
        "structures": tree,
        "fp64_plain": fp64,
        "speedup_fp32_over_fp64": (value / world) / fp64["steps_per_s"] if fp64 else None,
        "roofline": {"kernel": kname, "bound": "fp32-simt", "achieved": achieved, "peak": peak32,
                     "unit": "TFLOP/s", "frac": achieved / peak32, "traffic": traffic,
                     "peak_source": "measured FP32 FMA throughput of this GPU (vx_measure_peak), the larger of "
                                    "scalar FMA and packed f32x2 FMA",
                     "peak_fp32_scalar": peak32_scalar, "peak_fp32_packed": peak32_packed,
                     "flop_per_pair": kflop, "pairs_per_launch": kpairs, "launch_ms": kms,
                     "mufu_ceiling": ({"bound": "special-function pipe (one rsqrt + one ex2 per pair)",
                                       "achieved_tpairs_per_s": kpairs / (kms * 1e-3) / 1e12,
                                       "peak_tpairs_per_s": mufu,
                                       "frac": kpairs / (kms * 1e-3) / 1e12 / mufu,
                                       "peak_source": "measured rsqrt+ex2 throughput of this GPU "
                                                      "(vx_measure_peak mode 3)"}
                                      if kname.startswith("k_diff_cells") else None)},
        "roofline_hbm": {"peak_gbs": hbm_peak, "peak_source": hbm_src,
                         "n_particles": n_kt,
                         "timing": "3 instrumented steps, an event pair around every kernel (about 1 us of event "
                                   "overhead in each time)",
                         "kernels": roofline_hbm(kt, 3, n_kt, hbm_peak)},
        "e2e": {"value": e2e_steps / sum(e2e_t), "unit": "steps/s",
                "h2d_bytes_per_step": bi // e2e_steps, "d2h_bytes_per_step": bo // e2e_steps},
        "gpu_launches": int(launches),
        "clocks": ck,
    }
    line["cpu_baseline"] = guarded("cpu baseline", cpu_baseline, args, x0, y0, g0, pan)
    if args.ref_cuda_steps > 0 and world == 1:
        line["reference_cuda_build"] = guarded("reference CUDA build", ref_cuda_build, args, x0, y0, g0)
    if multi:
        line["batched"], line["served"] = multi
    if plate:
        line["plate_config"] = plate
    if cross:
        line["crossover"] = (cross if isinstance(cross, dict) else
                             {"what": "velocity stage (FP32) on the benchmark wake: direct sum against the best "
                                      "accurate FMM setting, ms", "rows": cross})
    return line


def plate_leg(args, device):
    """The plate configuration at its scale: the 2576-panel rounded plate at
    20 degrees of incidence, Re 1e4, dt 0.001, FP32 bulk, from a seeded warm
    wake of args.plate_n vortices: steps/s over args.plate_steps event-timed
    steps (graph replay) and the 64 x 64 probe grid against the plain FP64
    direct sum over the same vortices.  (The 5000-step run with its Cd/Cl
    statistics is `python -m vortex_b200.runs config3`.)"""
    from vortex_b200 import native as Nt
    from vortex_b200 import profiles
    from vortex_b200 import runs
    from vortex_b200 import workloads as wl
    pan = profiles.rotate(profiles.rounded_plate(2576), -20.0)
    sim = Nt.Sim(runs.plate_conf(Nt.PREC_FP32, pan), pan, device=device)
    sim.set_particles(*wl.warm_wake(args.plate_n, seed=4321))
    sim.step(2)
    sim.sync()
    st = sim.stream()
    ms = []
    for _ in range(args.plate_steps):
        a, b = Nt.Event(), Nt.Event()
        a.record(st)
        sim.step(1)
        b.record(st)
        ms.append(a.elapsed_ms(b))
    rec = {"workload": "rounded plate chord 1, thickness 0.02, 2576 panels, 20 deg incidence, Re 1e4, dt 0.001, "
                       f"FP32 bulk, seeded warm wake of {args.plate_n} vortices",
           "steps": args.plate_steps, "steps_per_s": 1e3 * len(ms) / sum(ms), "ms_p50": float(np.percentile(ms, 50)),
           "n_particles_end": sim.count(), "probe_grid_vs_fp64_direct": runs.probe_error(sim, pan, device)}
    sim.close()
    return rec


def multibody_runs(args, device, rank, world):
    """The seeded population batched and served, partitioned by body over the
    ranks (each rank its share on its own GPU, no exchange while stepping),
    the ranks' records gathered and combined on the host.  Every rank takes
    part in the gathers (also when its own part failed); rank 0 gets the
    combined records."""
    from vortex_b200 import multibody as MB
    from vortex_b200 import native as Nt

    def batched_part():
        pop = MB.make_population(args.batch_bodies, device=device, rank=rank, world=world)
        try:
            batched = MB.run_batch(steps=args.batch_steps, warmup=3, device=device, rank=rank, world=world,
                                   mode="graph", population=pop)
            # the same bodies (a few steps later) as concurrent per-body step
            # graphs, for comparison
            streams = MB.run_batch(steps=5, warmup=1, device=device, rank=rank, world=world, mode="streams",
                                   population=pop)
        finally:
            for s in pop[1]:
                s.close()
        batched["per_body_streams"] = {k: streams[k] for k in ("mode", "ms_per_batched_step", "body_steps_per_s",
                                                               "particle_steps_per_s", "kernels_per_batched_step")}
        sub32 = MB.run_batch(bodies=16, steps=2, warmup=1, device=device, rank=rank, world=world)
        sub64 = MB.run_batch(bodies=16, steps=2, warmup=1, precision=Nt.PREC_FP64, device=device, rank=rank,
                             world=world)
        batched["fp32_vs_fp64_first16_bodies"] = sub32["body_steps_per_s"] / sub64["body_steps_per_s"]
        return batched

    batched = guarded("batched run", batched_part)
    served = guarded("served run", MB.run_serve, requests=args.serve_requests, device=device, rank=rank,
                     world=world)
    if world == 1:
        return batched, served
    import torch.distributed as D
    parts = [None] * world
    D.all_gather_object(parts, (batched, served))
    bad_b = [p[0] for p in parts if "error" in p[0]]
    bad_s = [p[1] for p in parts if "error" in p[1]]
    if bad_b:
        b = bad_b[0]
    else:
        b = MB.combine_batch([p[0] for p in parts])
        b["fp32_vs_fp64_first16_bodies"] = float(np.mean([p[0]["fp32_vs_fp64_first16_bodies"] for p in parts]))
    return b, (bad_s[0] if bad_s else MB.combine_serve([p[1] for p in parts]))


def cpu_sample(x, y, g, pan, n_targets, n_panels):
    """Time the oracle's plain FP64 step pieces on a sample and extrapolate
    to a full step of len(x) particles (pair sums dominate on the CPU)."""
    from oracle import oracle as O
    n = len(x)
    p = O.make_params(dt=0.002, nu=5e-4, eps=2 * math.pi * 0.5 / P_PANELS, r_col_same_sign=0.3,
                      prof_x_min=-0.5, prof_x_max=0.5, prof_y_min=-0.5, prof_y_max=0.5, drop_eps=1e-8,
                      birth_mode=O.BIRTH_HALF_PANEL)
    cap = (n + 31) // 32 * 32
    xs, ys, gs = np.zeros(cap), np.zeros(cap), np.zeros(cap)
    xs[:n], ys[:n], gs[:n] = x, y, g
    O.fill_tail(xs, ys, gs, n, cap)
    T = n_targets
    i0 = n // 2 - T // 2
    vx, vy, d = np.zeros(T), np.zeros(T), np.zeros(T)
    lib = O.lib()
    ptr = [O._p(a) for a in (xs, ys, gs)]
    t0 = time.perf_counter()
    lib.vxo_velocity_targets(C.byref(p), *ptr, C.c_int64(n), C.c_int64(i0), C.c_int64(i0 + T),
                             O._p(vx), O._p(vy), O._p(d))
    t1 = time.perf_counter()
    lib.vxo_diffusion_targets(C.byref(p), *ptr, C.c_int64(n), C.c_int64(i0), C.c_int64(i0 + T),
                              O._p(d), O._p(vx), O._p(vy))
    t2 = time.perf_counter()
    sub = pan[:n_panels].copy()
    sub["nr"] = np.minimum(sub["nr"], n_panels - 1)
    O.birth_rhs(p, sub, xs[:n], ys[:n], gs[:n])
    t3 = time.perf_counter()
    step_s = (t2 - t0) * n / T + (t3 - t2) * P_PANELS / n_panels
    return step_s, t3 - t0


def cpu_baseline(args, x, y, g, pan):
    from oracle import oracle as O
    step_s, spent = cpu_sample(x, y, g, pan, args.cpu_targets, 32)
    return {"value": 1.0 / step_s, "unit": "steps/s", "cores": O.lib().vxo_num_threads(), "kind": "port",
            "sample": f"oracle FP64 (OpenMP): Biot-Savart+3-nearest and vortex diffusion for "
                      f"{args.cpu_targets} of {len(x)} targets over all sources, birth RHS for 32 of "
                      f"{P_PANELS} panels over all sources; extrapolated to one full step "
                      f"({spent:.1f} s measured)"}


REF_CONF = """steps {steps}
saving_step 100000
dt 0.002
inc_step {inc}
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


def ref_cuda_build(args, x, y, g):
    """The reference's own CUDA program (its src/main.c + src/unit_1.cu +
    src/kernel.cu, -DNO_TREE, sm_100a, built by oracle/build_ref.sh) on the
    same workload, restarted from a frame holding the same warm wake; its
    per-step device time is the Creation + Speed + Step event times it logs
    (cumulative seconds per step in its timings file)."""
    import tempfile
    from vortex_b200 import profiles
    exe = os.path.join(ROOT, "oracle", "_ref", "vortex_ref")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/vortex_ref not built (oracle/build_ref.sh needs the reference sources)"}
    K = args.ref_cuda_steps
    with tempfile.TemporaryDirectory() as wd:
        profiles.write_profile(os.path.join(wd, "circle1000.txt"), profiles.circle(P_PANELS))
        with open(os.path.join(wd, "run.conf"), "w") as fh:
            fh.write(REF_CONF.format(steps=K, inc=1 << 20, eps=2 * math.pi * 0.5 / P_PANELS))
        with open(os.path.join(wd, "Kadr000000.txt"), "w") as fh:
            fh.write(f"{len(x)}\n")
            fh.writelines(f"{i} 0.008000 {x[i]:.17g} {y[i]:.17g} 0 0 0 {g[i]:.17g}\n" for i in range(len(x)))
        t0 = time.perf_counter()
        r = subprocess.run([exe, "-c", "run.conf", "-l", "1"], cwd=wd, capture_output=True, text=True,
                           timeout=args.ref_cuda_timeout)
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            return {"unavailable": f"reference program exited {r.returncode}"}
        rows = []
        for line in open(os.path.join(wd, "output", "timings.txt")):
            parts = line.strip().split("\t")
            if len(parts) >= 5:
                rows.append((int(parts[0]), int(parts[1].split("=")[1]),
                             sum(float(q.split("=")[1]) for q in parts[2:5])))
    # the reference's stop_timer returns seconds (src/unit_1.cu:604-613)
    per_step = [1e3 * (b[2] - a[2]) for a, b in zip(rows[:-1], rows[1:]) if b[0] > a[0]]
    if not per_step:
        return {"unavailable": "reference timings file had no per-step lines"}
    ms = float(np.median(per_step[1:] if len(per_step) > 1 else per_step))
    return {"steps_per_s": 1e3 / ms, "ms_per_step": ms, "steps": len(per_step), "n_start": len(x),
            "n_end": rows[-1][1], "wall_s": wall,
            "source": "reference src/main.c + src/unit_1.cu + src/kernel.cu (-DNO_TREE, sm_100a) via "
                      "oracle/build_ref.sh; median of its per-step Creation+Speed+Step CUDA-event times"}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    from oracle import oracle as O
    from vortex_b200 import workloads as wl
    pan = wl.cylinder_panels(P_PANELS)
    x, y, g = wl.warm_wake(args.n, seed=1234)
    for _ in range(args.warmup):
        cpu_sample(x, y, g, pan, args.ref_targets, 16)
    t0 = time.perf_counter()
    est = [cpu_sample(x, y, g, pan, args.ref_targets, 16)[0] for _ in range(args.steps)]
    measured_s = time.perf_counter() - t0
    step_s = float(np.mean(est))
    # each timed "step" is a bounded sample of one step: the sampled targets'
    # pair sums and 16 panels' birth sums, extrapolated to the full step
    frac = measured_s / args.steps / step_s
    v = 1.0 / step_s
    return {"metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp64",
            "data": "synthetic (seeded warm wake on a jittered lattice; generated circle profile)",
            "config": workload_config(args, world),
            "impl": "reference",
            "extrapolated": True,
            "measured_s": measured_s,
            "sample_fraction_of_step": frac,
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": O.lib().vxo_num_threads(), "kind": "port",
                             "sample": f"each step: oracle FP64 (OpenMP) Biot-Savart+3-nearest and diffusion "
                                       f"for {args.ref_targets} targets over all {args.n} sources, birth RHS "
                                       "for 16 panels; extrapolated to a full step"},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", "--particles", dest="n", type=int, default=1_000_000)
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--cpu-targets", type=int, default=2048)
    ap.add_argument("--ref-targets", type=int, default=1024)
    ap.add_argument("--ref-cuda-steps", type=int, default=3,
                    help="also time the reference's own CUDA build for this many steps (0: off)")
    ap.add_argument("--ref-cuda-timeout", type=float, default=900.0)
    ap.add_argument("--no-autotune", action="store_true", help="skip the untimed autotuning before timing")
    ap.add_argument("--plate-steps", type=int, default=10, help="steps of the plate leg (0: skip)")
    ap.add_argument("--plate-n", type=int, default=3_000_000)
    ap.add_argument("--no-crossover", dest="crossover", action="store_false",
                    help="skip the direct-vs-FMM crossover table (untimed)")
    ap.add_argument("--no-multibody", dest="multibody", action="store_false",
                    help="skip the seeded multi-body population batched and served")
    ap.add_argument("--batch-bodies", type=int, default=256)
    ap.add_argument("--batch-steps", type=int, default=20)
    ap.add_argument("--serve-requests", type=int, default=32)
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if line:
            print(json.dumps(line), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        line = run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()
    if line:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
