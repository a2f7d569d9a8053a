"""Degenerate inputs of the pair stages (velocity with the 3-nearest search,
vortex diffusion) on all three forms: plain FP64, bulk FP32 with direct
sums, bulk FP32 with the quadtree FMM.

Scenes: one vortex, two, five (fewer sources than the 3-nearest search needs,
so the padding slots beyond n take part, as in the reference); 3000 vortices
on one horizontal line (zero height: a one-row cell grid, FMM box from the
width alone); 1500 pairs of coincident vortices (r = 0 pairs are skipped by
the 0.001 eps rule, the nearest distance is 0); 64 vortices on one point
(zero extent: one cell, an FMM tree without expansions, d = 0 everywhere);
a wake with one vortex in the far corner of the flow window (its 3-nearest
distance is about 10, so its diffusion window covers the whole grid).

Strengths are of one sign, so I1 of the diffusion quotient never cancels and
the bulk bounds hold for every vortex:
  * plain FP64 against the oracle: 3-nearest distance bit-exact, velocities
    within 1e-12 (sums in another order);
  * bulk against plain FP64: velocity within 2e-5 max |V|; 3-nearest
    distance within 2e-6 absolute (FP32 rounding of coordinates of order
    10); diffusion increment within 1e-4 of the largest FP64 increment, and
    exactly zero where the FP64 increment is (no source beyond r > 0.001 eps).
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import conf_kwargs, oracle_params, wake_cloud, with_tail
from vortex_b200 import native as N
from vortex_b200 import profiles

pytestmark = pytest.mark.gpu

P = 200
SCENES = ["one", "two", "five", "line", "coincident_pairs", "one_point", "outlier"]


def scene(name):
    rng = np.random.default_rng(SCENES.index(name) + 90)
    if name in ("one", "two", "five"):
        n = {"one": 1, "two": 2, "five": 5}[name]
        x, y, _ = wake_cloud(n, seed=n)
        g = rng.uniform(0.5, 1.5, n) * 1e-2
    elif name == "line":
        n = 3000
        x = rng.uniform(0.6, 4.0, n)
        y = np.full(n, 0.25)
        g = rng.uniform(0.5, 1.5, n) * 1e-3
    elif name == "coincident_pairs":
        x0, y0, _ = wake_cloud(1500, seed=77)
        x, y = np.repeat(x0, 2), np.repeat(y0, 2)
        g = rng.uniform(0.5, 1.5, len(x)) * 1e-3
    elif name == "one_point":
        x, y = np.full(64, 1.5), np.full(64, 0.1)
        g = rng.uniform(0.5, 1.5, 64) * 1e-3
    elif name == "outlier":
        x, y, _ = wake_cloud(20000, seed=78)
        x[17], y[17] = 9.5, -9.5
        g = rng.uniform(0.5, 1.5, len(x)) * 1e-3
    else:
        raise KeyError(name)
    return with_tail(x, y, g, extra=64) + (len(x),)


def forms():
    ck = conf_kwargs(P)
    pan = profiles.circle(P)
    sims = {
        "fp64": N.Sim(N.default_conf(**dict(ck, precision=N.PREC_FP64)), pan),
        "fp32": N.Sim(N.default_conf(**dict(ck, precision=N.PREC_FP32, fmm=0)), pan),
        "fmm": N.Sim(N.default_conf(**dict(ck, precision=N.PREC_FP32, fmm=1)), pan),
    }
    return sims, oracle_params(pan, ck)


@pytest.mark.parametrize("name", SCENES)
def test_velocity_and_nearest_on_degenerate_scenes(name):
    xs, ys, gs, n = scene(name)
    sims, p = forms()
    out = {}
    for k, s in sims.items():
        s.set_slots(xs, ys, gs, n)
        s.stage("velocity")
        out[k] = s.velocity()
    ovx, ovy, od = O.velocity(p, xs, ys, gs, n)
    vx, vy, d = out["fp64"]
    assert np.array_equal(d, od), "3-nearest distance must be bit-exact"
    assert np.abs(vx - ovx).max() < 1e-12 and np.abs(vy - ovy).max() < 1e-12
    vmax = max(np.abs(ovx).max(), np.abs(ovy).max())
    for k in ("fp32", "fmm"):
        ax, ay, ad = out[k]
        assert np.abs(ax - ovx).max() <= 2e-5 * vmax, (k, np.abs(ax - ovx).max())
        assert np.abs(ay - ovy).max() <= 2e-5 * vmax, (k, np.abs(ay - ovy).max())
        assert np.abs(ad - od).max() <= 2e-6, (k, np.abs(ad - od).max())
    if name == "one_point":
        assert np.all(od == 0.0)
        assert np.all(ovx == 1.0) and np.all(ovy == 0.0)
    if name == "coincident_pairs":
        assert np.all(od > 0.0)        # the twin at r = 0 is one of three
    for s in sims.values():
        s.close()


@pytest.mark.parametrize("name", SCENES)
def test_diffusion_on_degenerate_scenes(name):
    xs, ys, gs, n = scene(name)
    sims, p = forms()
    vx0, vy0, d = O.velocity(p, xs, ys, gs, n)
    evx, evy = O.diffusion(p, xs[:n], ys[:n], gs[:n], n, d, vx0, vy0)
    edv = np.hypot(evx - vx0, evy - vy0)
    scale = edv.max()
    for k, s in sims.items():
        s.set_slots(xs, ys, gs, n)
        s.set_velocity(vx0, vy0, d)
        s.stage("diffusion")
        vx, vy, _ = s.velocity()
        if k == "fp64":
            assert np.abs(vx - evx).max() < 1e-12 and np.abs(vy - evy).max() < 1e-12
            continue
        err = np.hypot((vx - vx0) - (evx - vx0), (vy - vy0) - (evy - vy0))
        assert err.max() <= 1e-4 * scale, (k, err.max(), scale)
        assert np.all(vx[edv == 0] == vx0[edv == 0]) and np.all(vy[edv == 0] == vy0[edv == 0]), k
    if name in ("one", "one_point"):
        assert scale == 0.0            # nothing within reach but the vortex itself
    else:
        assert scale > 0.0
    for s in sims.values():
        s.close()
