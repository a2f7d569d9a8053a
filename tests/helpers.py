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


def inside_polygon(px, py, pan):
    """Even-odd test of points against the closed polygon of the panels'
    left endpoints."""
    x0, y0 = pan["left"][:, 0], pan["left"][:, 1]
    x1, y1 = pan["right"][:, 0], pan["right"][:, 1]
    inside = np.zeros(len(px), dtype=bool)
    for a in range(0, len(px), 4096):
        X = px[a:a + 4096, None]
        Y = py[a:a + 4096, None]
        crosses = (y0[None, :] > Y) != (y1[None, :] > Y)
        with np.errstate(divide="ignore", invalid="ignore"):
            xc = x0[None, :] + (Y - y0[None, :]) * (x1 - x0)[None, :] / (y1 - y0)[None, :]
        inside[a:a + 4096] = np.logical_xor.reduce(crosses & (X < xc), axis=1)
    return inside


def scale_body(name):
    """The configurations' own bodies: the 1000-panel cylinder (the
    benchmark's; Re 2000, dt 0.002) and the 2576-panel rounded plate of
    chord 1 turned to 20 degrees of incidence (Re 1e4, dt 0.001); core
    radius = mean panel length, same-sign collapse within 0.3 eps."""
    if name == "circle1000":
        pan = profiles.circle(1000)
        ck = conf_kwargs(1000, dt=0.002, viscosity=5e-4)
    elif name == "plate2576":
        pan = profiles.rotate(profiles.rounded_plate(2576), 20.0)
        ck = conf_kwargs(2576, dt=0.001, viscosity=1e-4, ve_size=float(pan["length"].mean()))
    else:
        raise ValueError(name)
    return pan, ck


def body_cloud(pan, n, seed=0, g_scale=2e-3):
    """A wake-like cloud around and behind any body, none inside it: half
    near the wall (off the panels' control points along their normals, an
    exponential distance), half in a box behind the body."""
    rng = np.random.default_rng(seed)
    n1 = n // 2
    k = rng.integers(0, len(pan), n1)
    off = rng.exponential(0.03, n1) + 1e-4
    t = rng.uniform(-0.5, 0.5, n1) * pan["length"][k]
    x1 = pan["contr"][k, 0] + off * pan["norm"][k, 0] + t * pan["tang"][k, 0]
    y1 = pan["contr"][k, 1] + off * pan["norm"][k, 1] + t * pan["tang"][k, 1]
    xmin, xmax = pan["left"][:, 0].min(), pan["left"][:, 0].max()
    ymin, ymax = pan["left"][:, 1].min(), pan["left"][:, 1].max()
    x2 = rng.uniform(xmin, xmax + 2.5, n - n1)
    y2 = rng.normal(0.5 * (ymin + ymax), 0.3 + 0.5 * (ymax - ymin), n - n1)
    x, y = np.concatenate([x1, x2]), np.concatenate([y1, y2])
    bad = inside_polygon(x, y, pan)
    x[bad] += (xmax - xmin) + 0.5      # moved downstream, clear of the body
    g = rng.normal(0.0, g_scale, n)
    return x, y, g
