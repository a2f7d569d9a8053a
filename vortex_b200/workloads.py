"""Seeded synthetic workloads shared by the benchmark and the profiling runner.

The headline workload is the 1000-panel cylinder of radius 0.5 at Re = 2000
(nu = 5e-4), dt = 0.002, core radius = panel length, birth half a panel off
the wall, same-sign collapse within 0.3 eps, |G| < 1e-8 dropped.  The
reference holds about 1e6 vortices in this run after ~3000 steps; the
stand-in for that state is a warm wake of n vortices on a jittered lattice
in the 4 x 2 box behind the cylinder ([0.55, 4.55] x [-1, 1]), spacing
a = sqrt(8/n), jitter +-a/4 (nearest neighbours start farther apart than the
collapse radius), carrying a smooth vorticity field sampled at the vortices
(G = omega * a^2): a staggered street of five Gaussian vortices of
circulation -+2 and radius 0.2 (negative above the axis, positive below,
1.0 to 4.2 in x, 0.8 apart) over a shear background -0.5 tanh(y / 0.2).
Neighbouring vortices carry like-signed, similar strengths, as in a wake
that has run for some time, so the diffusion velocity stays moderate and
the count stays near n over the timed steps.
"""
from __future__ import annotations

import math

import numpy as np

from . import native as N
from . import profiles

PANELS = 1000


def cylinder_conf(precision: int, panels: int = PANELS, **kw) -> "N.Conf":
    base = dict(steps=1000, saving_step=100, dt=0.002, viscosity=5e-4, rho=1.0, v_inf_x=1.0, v_inf_y=0.0,
                x_min=-2.0, x_max=10.0, y_min=-10.0, y_max=10.0, ve_size=2 * math.pi * 0.5 / panels,
                n_of_points=20, n_col=2, r_col_diff_sign=0.0, r_col_same_sign=0.3, max_ve_g=1e30,
                v_inf_incr_steps=0, drop_eps=1e-8, birth_offset_mode=N.BIRTH_HALF_PANEL,
                precision=precision, inc_step=8192)
    base.update(kw)
    return N.default_conf(**base)


def cylinder_panels(panels: int = PANELS) -> np.ndarray:
    return profiles.circle(panels)


def warm_wake(n: int, seed: int = 1234):
    rng = np.random.default_rng(seed)
    a = math.sqrt(8.0 / n)
    nx, ny = int(math.ceil(4.0 / a)), int(math.ceil(2.0 / a))
    while nx * ny < n:
        nx += 1
    ix, iy = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")
    x = 0.55 + (ix.ravel() + 0.5) * (4.0 / nx)
    y = -1.0 + (iy.ravel() + 0.5) * (2.0 / ny)
    pick = rng.permutation(nx * ny)[:n]
    x = x[pick] + rng.uniform(-0.25, 0.25, n) * (4.0 / nx)
    y = y[pick] + rng.uniform(-0.25, 0.25, n) * (2.0 / ny)
    omega = -0.5 * np.tanh(y / 0.2)
    for k in range(5):
        xc, yc = 1.0 + 0.8 * k, (0.3 if k % 2 == 0 else -0.3)
        sign = -1.0 if k % 2 == 0 else 1.0
        omega += sign * 2.0 / (math.pi * 0.04) * np.exp(-((x - xc) ** 2 + (y - yc) ** 2) / 0.04)
    g = omega * (8.0 / n)
    return x, y, g


# ---------------------------------------------------------------------------
# Seeded multi-body workloads (batched and served runs).
#
# Random numbers come from SplitMix64 (S. Vigna's published generator: state
# advanced by the golden-ratio increment 0x9E3779B97F4A7C15, output mixed by
# two xor-shift-multiply rounds), restated here.  Because the state of draw k
# is seed + (k + 1) * increment, a whole stream is evaluated at once with
# numpy's wrapping uint64 arithmetic.
_GAMMA = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, count: int, offset: int = 0) -> np.ndarray:
    """Draws offset .. offset+count-1 of the SplitMix64 stream of `seed`."""
    k = np.arange(offset + 1, offset + count + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + k * _GAMMA
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def uniforms(seed: int, count: int, offset: int = 0) -> np.ndarray:
    """U[0, 1) doubles from the top 53 bits of each draw."""
    return (splitmix64(seed, count, offset) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def normals(seed: int, count: int, offset: int = 0) -> np.ndarray:
    """N(0, 1) by the Box-Muller transform of consecutive uniform pairs."""
    m = (count + 1) // 2
    u = uniforms(seed, 2 * m, offset)
    r = np.sqrt(-2.0 * np.log1p(-u[0::2]))
    t = 2.0 * math.pi * u[1::2]
    return np.concatenate([r * np.cos(t), r * np.sin(t)])[:count]


def _log_uniform(u: float, lo: float, hi: float) -> float:
    return math.exp(math.log(lo) + u * (math.log(hi) - math.log(lo)))


def body_spec(seed: int, index: int) -> dict:
    """Parameters of body `index` of the seeded population: an ellipse
    (a = 0.5, b ~ U[0.05, 0.5]) or a plate (chord 1, thickness 0.02, rounded
    ends, angle ~ U[0, 45] degrees), panels log-uniform in [200, 3320],
    Re log-uniform in [500, 2e4] (nu = 1/Re at U = 1 and unit length),
    dt = 0.005 * 200 / panels, a warm cloud of log-uniform [1e3, 5e5]
    vortices."""
    u = uniforms(seed ^ 0x5EED, 8, offset=8 * index)
    kind = "ellipse" if u[0] < 0.5 else "plate"
    P = int(round(_log_uniform(u[1], 200, 3320)))
    return {"index": index, "kind": kind, "panels": P,
            "b": 0.05 + 0.45 * u[2], "angle": 45.0 * u[3],
            "re": _log_uniform(u[4], 500.0, 2e4), "n0": int(round(_log_uniform(u[5], 1e3, 5e5))),
            "dt": 0.005 * 200.0 / P, "cloud_seed": int(splitmix64(seed, 1, offset=index)[0])}


def make_body(spec: dict, precision: int):
    """(conf, panels, x, y, G) of a body_spec: Gaussian cloud in the 4 x 2 wake
    box [0.55, 4.55] x [-1, 1] (centre (2.55, 0), sigmas 1 and 0.5, folded
    back into the box), G ~ N(0, 1e-3); eps = mean panel length, birth half
    a panel off the wall, same-sign collapse within 0.3 eps, |G| < 1e-8
    dropped; the panel system is inverted with the reference's pivot rule,
    or with partial pivoting where that rule meets a tiny pivot (thin
    bodies).  The store grows by at least 16 steps' births at a time (a
    growth re-records the body's part of a batched step)."""
    P = spec["panels"]
    if spec["kind"] == "ellipse":
        pan = profiles.ellipse(P, 0.5, spec["b"])
    else:
        pan = profiles.rotate(profiles.rounded_plate(P, 1.0, 0.02), -spec["angle"])
    eps = float(np.mean(pan["length"]))
    n = spec["n0"]
    z = normals(spec["cloud_seed"], 3 * n)

    def fold(v, lo, hi):
        w = hi - lo
        t = np.mod(v - lo, 2 * w)
        return lo + np.where(t > w, 2 * w - t, t)

    x = fold(2.55 + 1.0 * z[:n], 0.55, 4.55)
    y = fold(0.5 * z[n:2 * n], -1.0, 1.0)
    g = 1e-3 * z[2 * n:]
    conf = N.default_conf(steps=1000, dt=spec["dt"], viscosity=1.0 / spec["re"], rho=1.0, v_inf_x=1.0,
                          v_inf_y=0.0, x_min=-2.0, x_max=10.0, y_min=-10.0, y_max=10.0, ve_size=eps,
                          n_of_points=20, n_col=2, r_col_diff_sign=0.0, r_col_same_sign=0.3, max_ve_g=1e30,
                          v_inf_incr_steps=0, drop_eps=1e-8, birth_offset_mode=N.BIRTH_HALF_PANEL,
                          precision=precision, inc_step=max(8192, -(-16 * P // 8192) * 8192), gj_pivot=2)
    return conf, pan, x, y, g
