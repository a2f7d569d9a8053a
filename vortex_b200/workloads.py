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
