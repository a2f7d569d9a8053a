"""Batched steps (vx_batch): every kernel of the step runs once for all the
bodies of the batch, and the batched step is one CUDA graph.

Each body of a batch must come out bit-identical to a twin stepped alone
with vx_step: same count, every slot (the dead tail included) equal, the
same velocities and 3-nearest distances of the last step, the same force
sums.  The bodies differ in shape, panel count, cloud size and form (three
FP32-bulk bodies of the seeded population's kinds and one plain FP64 body),
and some outgrow their stores inside the batch, so the batch re-records
them, rewrites its tables and grows them stream-ordered while steps are in
flight.  The batched step takes one launch per kernel of the step, not one
per body.
"""
import numpy as np
import pytest

from vortex_b200 import native as N
from vortex_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _bodies():
    """(conf, panels, x, y, g) of four unlike bodies."""
    out = []
    specs = [dict(index=0, kind="ellipse", panels=260, b=0.2, angle=0.0, re=800.0, n0=3000, dt=0.005 * 200 / 260,
                  cloud_seed=11),
             # a store of 32 768 slots (the cloud's need and the smallest
             # growth margin, 8192) that 900 births a step outgrow within the
             # test's 14 steps
             dict(index=1, kind="plate", panels=900, b=0.1, angle=25.0, re=5000.0, n0=23500, dt=0.005 * 200 / 900,
                  cloud_seed=12),
             dict(index=2, kind="ellipse", panels=1500, b=0.45, angle=0.0, re=12000.0, n0=150000,
                  dt=0.005 * 200 / 1500, cloud_seed=13)]
    for sp in specs:
        conf, pan, x, y, g = wl.make_body(sp, N.PREC_FP32)
        conf.inc_step = 8192          # the smallest growth margin: body 1 outgrows its store
        out.append((conf, pan, x, y, g))
    sp = dict(index=3, kind="ellipse", panels=200, b=0.3, angle=0.0, re=1000.0, n0=1500, dt=0.005, cloud_seed=14)
    out.append(wl.make_body(sp, N.PREC_FP64))
    return out


def _make(spec):
    conf, pan, x, y, g = spec
    s = N.Sim(conf, pan)
    s.set_particles(x, y, g)
    return s


def _state(s):
    st = s.state()
    cap = int(st["n"]) + 64
    x, y, g = s.get_slots(cap)
    vx, vy, d = s.velocity()
    return int(st["n"]), x, y, g, vx, vy, d, s.forces()


def test_batch_matches_bodies_stepped_alone():
    specs = _bodies()
    alone = [_make(sp) for sp in specs]
    mine = [_make(sp) for sp in specs]
    steps = 14
    l0 = [a.launches() for a in alone]
    for s in alone:
        s.step(steps)
        s.sync()
    per_body = max(a.launches() - l for a, l in zip(alone, l0)) / steps
    caps0 = [s.device_bytes() for s in mine]
    with N.Batch(mine) as b:
        b.step(5)
        b.step(steps - 5)
        b.sync()
        info = b.info()
        # a body in a batch is stepped only through the batch
        with pytest.raises(N.VxError, match="batch"):
            mine[0].step(1)
        for k, (a, m) in enumerate(zip(alone, mine)):
            sa, sm = _state(a), _state(m)
            assert sa[0] == sm[0], f"body {k}: count {sa[0]} alone, {sm[0]} batched"
            for q, name in enumerate(("x", "y", "g", "vx", "vy", "d", "forces"), start=1):
                assert np.array_equal(sa[q], sm[q]), f"body {k}: {name} differs"
    # somebody outgrew its store inside the batch
    assert any(s.device_bytes() > c for s, c in zip(mine, caps0))
    # one launch per kernel of the step for all bodies, not one per body: the
    # plain FP64 body's direct sums and the bulk bodies' quadtree and grid
    # passes are different kernels, so the batch's step is their union, at
    # most two bodies' worth (four bodies alone would be four)
    assert info["steps"] == steps
    assert info["kernels_per_step"] <= 2 * per_body, (info, per_body)
    assert info["kernels"] <= steps * 2 * per_body
    # back on their own streams the bodies step alone again, still in step
    for a, m in zip(alone, mine):
        a.step(2)
        m.step(2)
        sa, sm = _state(a), _state(m)
        assert sa[0] == sm[0] and np.array_equal(sa[1], sm[1]) and np.array_equal(sa[3], sm[3])
    for s in alone + mine:
        s.close()


def test_batch_of_the_seeded_population_steps_and_reports_launches():
    """Eight bodies of the seeded population (ellipses and plates, 200-3320
    panels, clouds of 1e3-5e5): a few batched steps run, the counts stay
    consistent with the bodies' own step-by-step bookkeeping, and the
    batch's launches per step stay at the length of one body's step."""
    sims = []
    for i in range(8):
        conf, pan, x, y, g = wl.make_body(wl.body_spec(7, i), N.PREC_FP32)
        s = N.Sim(conf, pan)
        s.set_particles(x, y, g)
        sims.append(s)
    n0 = [s.count() for s in sims]
    with N.Batch(sims) as b:
        b.step(4)
        b.sync()
        info = b.info()
    P = [len(wl.make_body(wl.body_spec(7, i), N.PREC_FP32)[1]) for i in range(8)]
    for s, n, p in zip(sims, n0, P):
        m = s.count()
        assert 0 < m <= n + 4 * p
        assert s.state()["step"] == 4
    assert info["kernels_per_step"] < 300
    for s in sims:
        s.close()


def test_members_join_and_leave_between_steps():
    """Continuous membership: A runs alone in the batch for 3 steps, B joins
    for 4, then A leaves and C joins for 5 more.  Each body ends exactly as
    its twin stepped alone for its own number of steps (7, 9, 5), and the
    results gathered after the last batched step are the members' own
    counts and force sums."""
    specs = _bodies()[:3]
    alone = [_make(sp) for sp in specs]
    mine = [_make(sp) for sp in specs]
    for s, k in zip(alone, (7, 9, 5)):
        s.step(k)
        s.sync()
    A, B, C = mine
    b = N.Batch([A])
    b.step(3)
    b.add(B)
    b.step(4)
    b.remove(A)
    b.add(C)
    b.step(5)
    res = b.last_results()
    assert set(res) == {B.h.value, C.h.value}
    for m in (B, C):
        n, dg, fx, fy, mm = res[m.h.value]
        f = m.forces()
        assert n == m.count() and dg == f[0] and fx == f[1] and fy == f[2] and mm == f[3]
    b.close()
    for k, (a, m) in enumerate(zip(alone, mine)):
        sa, sm = _state(a), _state(m)
        assert sa[0] == sm[0], f"body {k}: count {sa[0]} alone, {sm[0]} batched"
        for q, name in enumerate(("x", "y", "g", "vx", "vy", "d", "forces"), start=1):
            assert np.array_equal(sa[q], sm[q]), f"body {k}: {name} differs"
    for s in alone + mine:
        s.close()
