"""Shared scene builders for the parity tests (seeded, deterministic)."""
from __future__ import annotations

import math

import numpy as np

from oracle import oracle as O
from vortex_b200 import profiles


def conf_kwargs(P=200, **kw):
    """Config-1 style run parameters: circle R=0.5, eps = panel length."""
    eps = 2 * math.pi * 0.5 / P
    base = dict(dt=0.005, viscosity=1e-3, rho=1.0, v_inf_x=1.0, v_inf_y=0.0, x_min=-2.0, x_max=10.0,
                y_min=-10.0, y_max=10.0, ve_size=eps, n_of_points=20, n_col=2, rc_x=0.0, rc_y=0.0,
                r_col_diff_sign=0.0, r_col_same_sign=0.3, max_ve_g=1e30, v_inf_incr_steps=0,
                drop_eps=1e-12, birth_offset_mode=0, precision=0)
    base.update(kw)
    return base


def oracle_params(pan, ck):
    bb = profiles.profile_bbox(pan, (ck["x_min"], ck["x_max"], ck["y_min"], ck["y_max"]))
    return O.make_params(dt=ck["dt"], nu=ck["viscosity"], rho=ck["rho"], vinf_x=ck["v_inf_x"],
                         vinf_y=ck["v_inf_y"], eps=ck["ve_size"], r_col_diff_sign=ck["r_col_diff_sign"],
                         r_col_same_sign=ck["r_col_same_sign"], max_ve_g=ck["max_ve_g"],
                         x_min=ck["x_min"], x_max=ck["x_max"], y_min=ck["y_min"], y_max=ck["y_max"],
                         prof_x_min=bb[0], prof_x_max=bb[1], prof_y_min=bb[2], prof_y_max=bb[3],
                         rc_x=ck["rc_x"], rc_y=ck["rc_y"], drop_eps=ck["drop_eps"],
                         n_of_points=ck["n_of_points"], n_col=ck["n_col"],
                         birth_mode=ck["birth_offset_mode"], prec=O.PREC_FP64)


def wake_cloud(n, seed=0, R=0.5, g_scale=2e-3):
    """Particles around and behind a cylinder of radius R, none inside it."""
    rng = np.random.default_rng(seed)
    n1 = n // 2
    th = rng.uniform(0, 2 * math.pi, n1)
    r = R + rng.exponential(0.05, n1) + 1e-4
    x1, y1 = r * np.cos(th), r * np.sin(th)
    x2 = rng.uniform(R, 3.0, n - n1)
    y2 = rng.normal(0.0, 0.35, n - n1)
    inside = x2 ** 2 + y2 ** 2 < (R + 1e-3) ** 2
    x2[inside] += 2 * R
    x = np.concatenate([x1, x2])
    y = np.concatenate([y1, y2])
    g = rng.normal(0.0, g_scale, n)
    return x, y, g


def with_tail(x, y, g, extra=64, seed=1):
    """Append a dead tail (G=0) like the reference's padded slots: some near
    the body (absorbed vortices keep their position), some far away."""
    rng = np.random.default_rng(seed)
    tx = np.concatenate([rng.uniform(-0.4, 0.4, extra // 2), np.full(extra - extra // 2, 1e10)])
    ty = np.concatenate([rng.uniform(-0.4, 0.4, extra // 2), np.full(extra - extra // 2, 1e10)])
    return (np.concatenate([x, tx]), np.concatenate([y, ty]), np.concatenate([g, np.zeros(extra)]))


def rel_err(a, b, scale=None):
    a, b = np.asarray(a), np.asarray(b)
    s = scale if scale is not None else max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / s) if a.size else 0.0
