"""The oracle against golden vectors recorded from the reference's own CUDA
build (tests/golden/ref_*.npz, made by tests/golden/make_ref_goldens.py on a
B200 with oracle/_ref/libvortex_ref.so).

Cases: the 200-panel circle of configuration 1 (steps 1, 4, 30), a mixed
run (steps 2, 20) and the reference's own 1000-panel circle profile
(krug_1000, steps 2 and 6).  Each recorded step is replayed stage by stage
from the reference's own state:
  * birth: positions exact; strengths within 1e-6 of the largest, or, where
    the reference's FP32 right-hand side is further from the FP64 one (at
    1000 panels its sums over the wake differ from FP64 by up to 2e-3 of the
    largest strength), at least three times closer to the reference than the
    FP64 evaluation (the oracle repeats the reference's FP32 terms; only the
    order of accumulation differs);
  * velocity in the oracle's reference-precision mode: 3-nearest distance d
    bit-exact, velocity within 5e-5 absolute (FP32 sums, exp/atan differences);
    in FP64 mode within 2e-3 (the reference's FP32 rounding, amplified by the
    diffusion quotient I2/I1 near cancellations), and d within the FP32
    rounding of the coordinates it is computed from, 4 eps32 (|x| + |y|) plus
    1e-7 of d;
  * convection, sums, compaction and both collapse passes from the
    reference's own velocities: the same count, identical strengths,
    positions within 2 ulp (the reference's compiler fuses some products),
    absorbed circulation and forces within 1e-12 relative;
  * probe velocity within 5e-6 (FP32) of the reference.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from vortex_b200 import profiles

GOLD = os.path.join(os.path.dirname(__file__), "golden")
CASES = ([("cfg1", k) for k in (1, 4, 30)] + [("mixed", k) for k in (2, 20)]
         + [("krug1000", k) for k in (2, 6)])


def load(name):
    z = np.load(os.path.join(GOLD, f"ref_{name}.npz"))
    c = dict(zip(list(z["conf_keys"]), z["conf_vals"]))
    pan = z["panels"].view(profiles.PANEL_DTYPE)
    return z, c, pan


def params(c, prec):
    return O.make_params(dt=c["dt"], nu=c["viscosity"], rho=c["rho"], vinf_x=c["v_inf_x"],
                         vinf_y=c["v_inf_y"], eps=c["ve_size"], r_col_diff_sign=c["r_col_diff_sign"],
                         r_col_same_sign=c["r_col_same_sign"], max_ve_g=c["max_ve_g"],
                         x_min=c["x_min"], x_max=c["x_max"], y_min=c["y_min"], y_max=c["y_max"],
                         prof_x_min=c["profile_x_min"], prof_x_max=c["profile_x_max"],
                         prof_y_min=c["profile_y_min"], prof_y_max=c["profile_y_max"],
                         rc_x=c["rc_x"], rc_y=c["rc_y"], drop_eps=1e-12, n_of_points=int(c["n_of_points"]),
                         n_col=int(c["n_col"]), birth_mode=O.BIRTH_REF, prec=prec)


@pytest.mark.parametrize("name,k", CASES)
def test_birth_matches_reference(name, k):
    z, c, pan = load(name)
    p = params(c, O.PREC_REF)
    pre, n0, dg = z[f"s{k}_pre_pos"], int(z[f"s{k}_pre_n"]), float(z[f"s{k}_pre_dg"])
    born = z[f"s{k}_born_pos"]
    P = len(pan)
    _, M = O.panel_matrix(pan)
    R = O.birth_rhs(p, pan, pre[:n0, 0], pre[:n0, 1], pre[:n0, 2])
    bx, by, bg = O.birth_place(p, pan, O.birth_gamma(M, R, dg))
    assert np.array_equal(bx, born[n0:n0 + P, 0]) and np.array_equal(by, born[n0:n0 + P, 1])
    ref = born[n0:n0 + P, 2]
    R64 = O.birth_rhs(params(c, O.PREC_FP64), pan, pre[:n0, 0], pre[:n0, 1], pre[:n0, 2])
    bg64 = O.birth_place(params(c, O.PREC_FP64), pan, O.birth_gamma(M, R64, dg))[2]
    bound = max(1e-6 * np.abs(ref).max(), np.abs(bg64 - ref).max() / 3)
    assert np.abs(bg - ref).max() <= bound, (np.abs(bg - ref).max(), bound)
    assert np.array_equal(born[:n0], pre[:n0])


@pytest.mark.parametrize("name,k", CASES)
@pytest.mark.parametrize("prec", [O.PREC_REF, O.PREC_FP64])
def test_velocity_matches_reference(name, k, prec):
    z, c, pan = load(name)
    p = params(c, prec)
    born, vel, d = z[f"s{k}_born_pos"], z[f"s{k}_vel"], z[f"s{k}_d"]
    n = int(z[f"s{k}_pre_n"]) + len(pan)
    s = len(born)
    x, y, g = born[:, 0].copy(), born[:, 1].copy(), born[:, 2].copy()
    vx, vy, dd = O.velocity(p, x, y, g, n, s)
    vx, vy = O.diffusion(p, x, y, g, n, dd, vx, vy)
    vx, vy = O.wall_diffusion(p, pan, x, y, n, dd, vx, vy)
    err = max(np.abs(vx - vel[:n, 0]).max(), np.abs(vy - vel[:n, 1]).max())
    if prec == O.PREC_REF:
        assert np.array_equal(dd, d[:n]), "FP32 3-nearest distance must match the reference bit for bit"
        assert err < 5e-5
    else:
        eps32 = 2.0 ** -24
        assert np.all(np.abs(dd - d[:n]) <= 4 * eps32 * (np.abs(x[:n]) + np.abs(y[:n])) + 1e-7 * d[:n])
        assert err < 2e-3


@pytest.mark.parametrize("name,k", CASES)
def test_step_matches_reference(name, k):
    z, c, pan = load(name)
    p = params(c, O.PREC_FP64)
    born, vel, post = z[f"s{k}_born_pos"], z[f"s{k}_vel"], z[f"s{k}_post_pos"]
    P = len(pan)
    n = int(z[f"s{k}_pre_n"]) + P
    s = len(born)
    x, y, g, t = O.advect(p, pan, born[:, 0], born[:, 1], born[:, 2], vel[:, 0], vel[:, 1], n, P)
    dg, fx, fy, m = O.sums(p, t)
    x, y, g, nn = O.compact(x, y, g, n)
    x, y, g, nn = O.collapse(p, 1, x, y, g, nn)
    x, y, g, nn = O.collapse(p, 2, x, y, g, nn)
    assert nn == int(z[f"s{k}_post_n"])
    assert np.array_equal(g[:s], post[:, 2])
    ulp = np.spacing(np.maximum(np.abs(post[:, :2]), 1e-300))
    assert np.all(np.abs(np.stack([x[:s], y[:s]], 1) - post[:, :2]) <= 2 * ulp)
    ref = z[f"s{k}_post_scalars"]
    for a, b in zip((dg, fx, fy, m), ref):
        assert abs(a - b) <= 1e-12 * max(1.0, abs(b))


@pytest.mark.parametrize("name,k", CASES)
def test_probe_matches_reference(name, k):
    z, c, pan = load(name)
    p = params(c, O.PREC_REF)
    post, nn = z[f"s{k}_post_pos"], int(z[f"s{k}_post_n"])
    px, py = np.full(500, -0.15), 0.01 + 0.002 * np.arange(500)
    vx, vy = O.probe(p, post[:, 0].copy(), post[:, 1].copy(), post[:, 2].copy(), nn, px, py)
    ref = z[f"s{k}_probe"]
    assert max(np.abs(vx - ref[:, 0]).max(), np.abs(vy - ref[:, 1]).max()) < 5e-6
