"""Long runs of two configurations on one GPU (FP32-bulk form; config2 also
in the plain FP64 form):

    python -m vortex_b200.runs config2 [--steps 3000] [--precision fp64] [--rules reference]
    python -m vortex_b200.runs config3 [--steps 5000] [--n0 3000000]

config2: the 1000-panel cylinder of radius 0.5 (the benchmark's body),
impulsively started at Re 2000 (nu 5e-4), dt 0.002, core radius = panel
length, birth half a panel off the wall, same-sign collapse within 0.3 eps,
|G| < 1e-8 dropped; the vortex count and the step time over the run, and
Cd / Cl (D = 1) over its second half.

config3: the 2576-panel rounded plate of chord 1 and thickness 0.02 at 20
degrees of incidence (nose up: the reference's turn.py rotation by -20),
Re 1e4 (nu 1e-4), dt 0.001, core radius = mean panel length, started from a
seeded warm wake of n0 vortices (workloads.warm_wake); steps/s over the run,
the velocity at the 4096 points of a 64 x 64 grid over [-1, 3] x [-1, 1]
from the bulk form's probe against the plain FP64 direct sum over the same
vortices (at the start and at the end), and the mean and RMS of Cd and Cl
(chord 1) over the last 2000 steps.

Both print one JSON record; times are CUDA events on the body's stream.
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import native as N
from . import profiles
from . import workloads as wl


def _timed_steps(sim, steps, every, record):
    """Step `steps` times; per step the forces, every `every` steps the
    count and the mean step time since the last record."""
    st = sim.stream()
    forces, counts = [], []
    a = N.Event()
    a.record(st)
    done = 0
    total_ms = 0.0
    for k in range(steps):
        sim.step(1)
        f = sim.forces()
        forces.append((f[1], f[2]))
        if (k + 1) % every == 0 or k + 1 == steps:
            b = N.Event()
            b.record(st)
            ms = a.elapsed_ms(b)
            total_ms += ms
            counts.append({"step": k + 1, "n": sim.count(), "ms_per_step": ms / (k + 1 - done)})
            done = k + 1
            a = b
    record["total_ms"] = total_ms
    record["history"] = counts
    return np.array(forces)


def _stats(f, window, scale):
    cd, cl = scale * f[window, 0], scale * f[window, 1]
    return {"cd_mean": float(cd.mean()), "cd_rms": float(cd.std()), "cl_mean": float(cl.mean()),
            "cl_rms": float(cl.std())}


def config2(steps: int = 3000, every: int = 100, device: int = 0, precision: int = N.PREC_FP32,
            reference_rules: bool = False) -> dict:
    """reference_rules: new vortices where the reference's program puts them
    (panel midpoint + 1e-6 n, include/kernel.cuh:109-116) and |G| < 1e-12
    dropped (its DELT, include/definitions.h:36), instead of the
    configuration's half a panel off the wall and 1e-8."""
    pan = wl.cylinder_panels(1000)
    kw = dict(birth_offset_mode=N.BIRTH_REF, drop_eps=1e-12) if reference_rules else {}
    sim = N.Sim(wl.cylinder_conf(precision, 1000, **kw), pan, device=device)
    form = "FP32-bulk" if precision == N.PREC_FP32 else "plain FP64"
    rules = ("the reference program's birth offset and drop threshold" if reference_rules
             else "birth half a panel off the wall, |G| < 1e-8 dropped")
    rec = {"config": f"cylinder R=0.5, 1000 panels, impulsive start, Re 2000, dt 0.002, {form}, {rules}",
           "steps": steps}
    t0 = time.perf_counter()
    f = _timed_steps(sim, steps, every, rec)
    rec["wall_s"] = time.perf_counter() - t0
    rec["steps_per_s"] = steps / (rec["total_ms"] * 1e-3)
    rec["n_final"] = sim.count()
    rec["n_max"] = max(h["n"] for h in rec["history"])
    rec["forces_second_half"] = _stats(f, slice(steps // 2, steps), 2.0)
    sim.close()
    return rec


def plate_conf(precision: int, pan, **kw):
    base = dict(steps=5000, dt=0.001, viscosity=1e-4, rho=1.0, v_inf_x=1.0, v_inf_y=0.0, x_min=-2.0,
                x_max=10.0, y_min=-10.0, y_max=10.0, ve_size=float(np.mean(pan["length"])), n_of_points=20,
                n_col=2, r_col_diff_sign=0.0, r_col_same_sign=0.3, max_ve_g=1e30, v_inf_incr_steps=0,
                drop_eps=1e-8, birth_offset_mode=N.BIRTH_HALF_PANEL, precision=precision, inc_step=65536,
                gj_pivot=2)
    base.update(kw)
    return N.default_conf(**base)


def probe_grid():
    gx, gy = np.meshgrid(np.linspace(-1.0, 3.0, 64), np.linspace(-1.0, 1.0, 64), indexing="xy")
    return gx.ravel(), gy.ravel()


def probe_error(sim32, pan, device=0) -> dict:
    """Bulk-form probe velocities against the plain FP64 direct sum over the
    same vortices (the FP64 twin holds a copy of the bulk body's vortices)."""
    px, py = probe_grid()
    u32, v32 = sim32.probe(px, py)
    x, y, g = sim32.particles()
    s64 = N.Sim(plate_conf(N.PREC_FP64, pan), pan, device=device)
    s64.set_particles(x, y, g)
    vinf = sim32.state()["vinf"]
    s64.set_vinf(*vinf)
    u64, v64 = s64.probe(px, py)
    s64.close()
    err = np.hypot(u32 - u64, v32 - v64)
    vmax = float(np.hypot(u64, v64).max())
    return {"points": len(px), "n_vortices": len(x), "max_abs": float(err.max()), "max_rel_to_max_v": float(err.max() / vmax),
            "rms_rel_to_max_v": float(np.sqrt(np.mean(err ** 2)) / vmax),
            "max_rel_pointwise": float((err / np.maximum(np.hypot(u64, v64), 1e-30)).max())}


def config3(steps: int = 5000, n0: int = 3_000_000, every: int = 250, device: int = 0) -> dict:
    pan = profiles.rotate(profiles.rounded_plate(2576), -20.0)
    sim = N.Sim(plate_conf(N.PREC_FP32, pan), pan, device=device)
    x, y, g = wl.warm_wake(n0, seed=4321)
    sim.set_particles(x, y, g)
    rec = {"config": "plate chord 1, thickness 0.02, 2576 panels, 20 deg incidence, Re 1e4, dt 0.001, FP32-bulk, "
                     f"seeded warm wake of {n0} vortices", "steps": steps, "n0": n0}
    rec["probe_start"] = probe_error(sim, pan, device)
    t0 = time.perf_counter()
    f = _timed_steps(sim, steps, every, rec)
    rec["wall_s"] = time.perf_counter() - t0
    rec["steps_per_s"] = steps / (rec["total_ms"] * 1e-3)
    rec["n_final"] = sim.count()
    rec["probe_end"] = probe_error(sim, pan, device)
    w = slice(max(0, steps - 2000), steps)
    rec["forces_last_2000"] = _stats(f, w, 2.0)
    sim.close()
    return rec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("which", choices=["config2", "config3"])
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--n0", type=int, default=3_000_000)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"],
                    help="config2: the FP32-bulk form (default) or the plain FP64 form")
    ap.add_argument("--rules", default="config", choices=["config", "reference"],
                    help="config2: the configuration's birth offset and drop threshold (default) or the "
                         "reference program's")
    a = ap.parse_args()
    if a.which == "config2":
        prec = N.PREC_FP32 if a.precision == "fp32" else N.PREC_FP64
        print(json.dumps(config2(a.steps or 3000, precision=prec, reference_rules=a.rules == "reference")))
    else:
        print(json.dumps(config3(a.steps or 5000, a.n0)))


if __name__ == "__main__":
    main()
