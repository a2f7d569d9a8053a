"""CPU checks of the oracle against the reference's own outputs, and of the
closed forms the CUDA kernels implement (compaction permutation, parallel
collapse resolution) against the oracle's serial restatements."""
import math
import os

import numpy as np
import pytest

from oracle import oracle as O
from oracle import refdrv
from tests.helpers import conf_kwargs, oracle_params, wake_cloud
from vortex_b200 import profiles

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("P", [40, 200])
def test_oracle_matrix_bit_exact_with_reference_golden(P):
    ref = np.load(os.path.join(GOLD, "ref_matrix.npz"))[f"circle{P}"]
    _, M = O.panel_matrix(profiles.circle(P))
    assert np.array_equal(M, ref)


@pytest.mark.skipif(not refdrv.available(), reason="oracle/_ref not built")
def test_oracle_matrix_bit_exact_with_reference_build():
    pan = profiles.ellipse(96, 0.5, 0.2)
    M = refdrv.matr_creation(pan)
    _, Mo = O.panel_matrix(pan)
    assert np.array_equal(M[:97, :97], Mo)


def test_panel_system_properties():
    pan = profiles.circle(64)
    L, M = O.panel_matrix(pan)
    assert np.abs(L @ M - np.eye(65)).max() < 1e-10
    assert np.allclose(L[64, :64], pan["length"]) and np.all(L[:64, 64] == 1.0)
    assert np.all(np.diag(L)[:64] == -0.5)


def test_singular_panel_system_is_reported():
    pan = profiles.circle(16)
    pan["length"][:] = 0.0        # a zero Kelvin row: the last pivot falls below 1e-12
    with pytest.raises(RuntimeError):
        O.panel_matrix(pan)


GOLDEN_PROFILE = os.path.join(os.path.dirname(__file__), "golden", "krug_1000_profile.npz")


def test_circle_generator_matches_shipped_profile():
    """The generated 1000-panel circle against the reference's shipped
    profiles/Profile_file_krug_1000.txt (recorded as a fixture by
    tests/golden/make_profile_golden.py)."""
    ref = np.load(GOLDEN_PROFILE)
    mine = profiles.circle(1000)
    for f in ("left", "right", "contr", "birth", "norm", "tang"):
        assert np.abs(ref[f] - mine[f]).max() < 1e-6    # the file prints 6 digits
    assert np.abs(ref["length"] - mine["length"]).max() < 1e-8
    assert np.array_equal(ref["nl"], mine["nl"]) and np.array_equal(ref["nr"], mine["nr"])


def test_rotation_round_trip(tmp_path):
    pan = profiles.rounded_plate(2576)
    rot = profiles.rotate(pan, 20.0)
    back = profiles.rotate(rot, -20.0)
    for f in ("left", "right", "norm", "tang"):
        assert np.abs(back[f] - pan[f]).max() < 1e-15
    p = tmp_path / "plate.txt"
    profiles.write_profile(p, rot)
    rd = profiles.read_profile(p)
    for f in ("left", "right", "contr", "birth", "norm", "tang", "length"):
        assert np.array_equal(rd[f], rot[f])


def compact_closed_form(x, y, g, n0, eps):
    """Parallel closed form used by the CUDA compaction (vx_compact.cu)."""
    live = np.abs(g[:n0]) >= eps
    scan = np.concatenate([[0], np.cumsum(live)])
    m = int(scan[n0])
    H = m - scan[m]
    holes = np.flatnonzero(~live[:m])
    nx, ny, ng = x.copy(), y.copy(), g.copy()
    for q in np.flatnonzero(live[m:]) + m:
        h = holes[H - 1 - (scan[q] - scan[m])]
        nx[h], ny[h], ng[h] = x[q], y[q], g[q]
    for e in range(m, n0):
        if e == n0 - 1 or live[e + 1]:
            grp = m - scan[e + 1]
            src = holes[grp] if grp < H else m
        else:
            src = e + 1
        nx[e], ny[e], ng[e] = x[src], y[src], 0.0
    return nx, ny, ng, m


def test_compaction_closed_form_matches_serial_swap_remove():
    rng = np.random.default_rng(1)
    for _ in range(1500):
        n0 = int(rng.integers(1, 50))
        x, y = rng.normal(size=n0 + 4), rng.normal(size=n0 + 4)
        g = np.where(rng.random(n0 + 4) < rng.random(), 0.0, rng.normal(size=n0 + 4))
        a = O.compact(x, y, g, n0)
        b = compact_closed_form(x, y, g, n0, 1e-12)
        assert a[3] == b[3]
        for u, v in zip(a[:3], b[:3]):
            assert np.array_equal(u, v)


def collapse_parallel(pas, x, y, g, col):
    """Round-based resolution used by the CUDA collapse (vx_collapse.cu)."""
    n = len(col)
    cand = np.flatnonzero(col >= 0)
    state = dict.fromkeys(cand.tolist(), 0)
    in_cnt = np.bincount(col[cand], minlength=n)
    has_app = np.zeros(n, bool)
    while any(v == 0 for v in state.values()):
        dec = {i: (2 if has_app[i] else 1) for i, v in state.items() if v == 0 and (has_app[i] or in_cnt[i] == 0)}
        for i, v in dec.items():
            state[i] = v
            in_cnt[col[i]] -= 1
            if v == 1:
                has_app[col[i]] = True
    first = np.full(n, n)
    for i, v in state.items():
        if v == 1:
            first[col[i]] = min(first[col[i]], i)
    nx, ny, ng = x.copy(), y.copy(), g.copy()
    for i, v in state.items():
        if v != 1:
            continue
        j = col[i]
        xj, yj, gj = (x[j], y[j], g[j]) if first[j] == i else (1e10, 1e10, 0.0)
        if pas == 1:
            ai, aj = abs(g[i]), abs(gj)
            mn = ai + aj
            nx[i], ny[i], ng[i] = (x[i] * ai + xj * aj) / abs(mn), (y[i] * ai + yj * aj) / abs(mn), g[i] + gj
        else:
            s = g[i] + gj
            nx[i], ny[i], ng[i] = (x[i] * g[i] + xj * gj) / s, (y[i] * g[i] + yj * gj) / s, s
    for i, v in state.items():
        if v == 1:
            nx[col[i]] = ny[col[i]] = 1e10
            ng[col[i]] = 0.0
    return nx, ny, ng


@pytest.mark.parametrize("pas", [1, 2])
def test_parallel_collapse_resolution_matches_serial_merge(pas):
    rng = np.random.default_rng(2 + pas)
    for _ in range(1500):
        n = int(rng.integers(2, 30))
        x, y, g = rng.normal(size=n), rng.normal(size=n), rng.normal(size=n)
        col = np.full(n, -1, np.int32)
        for i in range(n - 1):
            if rng.random() < 0.6:
                col[i] = rng.integers(i + 1, min(n, i + 4))
        a = O.collapse_merge(pas, x, y, g, n, col)
        b = collapse_parallel(pas, x, y, g, col)
        for u, v in zip(a, b):
            assert np.array_equal(u, v)


def test_oracle_step_conserves_circulation_with_kelvin():
    """Birth makes the total circulation of the new vortices equal the
    absorbed circulation (Kelvin row), so sum(G) after birth = sum before + dg."""
    P = 64
    pan = profiles.circle(P)
    ck = conf_kwargs(P)
    p = oracle_params(pan, ck)
    _, M = O.panel_matrix(pan)
    x, y, g = wake_cloud(500, seed=2)
    R = O.birth_rhs(p, pan, x, y, g)
    gam = O.birth_gamma(M, R, 1.25e-3)
    _, _, bg = O.birth_place(p, pan, gam)
    assert abs(bg.sum() - 1.25e-3) < 1e-14


def test_reference_precision_mode_close_to_fp64():
    pan = profiles.circle(100)
    ck = conf_kwargs(100)
    p64 = oracle_params(pan, ck)
    p32 = oracle_params(pan, ck)
    p32.prec = O.PREC_REF
    x, y, g = wake_cloud(800, seed=9)
    a = O.velocity(p64, x, y, g, 800, s=800)
    b = O.velocity(p32, x, y, g, 800, s=800)
    assert np.abs(a[0] - b[0]).max() < 1e-4 and np.abs(a[2] - b[2]).max() < 1e-6
