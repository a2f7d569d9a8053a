"""Many bodies on one GPU: vx_step_many and the vx_server request loop.

* step_many advances every body exactly as its own vx_step does (same bits);
* a request's result (force history, final count) is the same alone and in
  a mix of other requests arriving before and after it (bit-identical: each
  body runs in its own handle with deterministic kernels);
* admission respects the slot count and the device-byte budget, holds later
  requests until memory frees up, and rejects a request that alone exceeds
  the budget; the estimate covers what a body actually holds.
"""
import numpy as np
import pytest

from vortex_b200 import native as N
from vortex_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def small_body(i, n0=3000, panels=200):
    sp = wl.body_spec(5, i)
    sp.update(n0=n0 + 500 * i, panels=panels + 40 * i, dt=0.005 * 200.0 / (panels + 40 * i))
    return wl.make_body(sp, N.PREC_FP32)


def test_step_many_matches_individual_steps():
    bodies = [small_body(i) for i in range(3)]
    a = [N.Sim(c, p) for c, p, *_ in bodies]
    b = [N.Sim(c, p) for c, p, *_ in bodies]
    for (c, p, x, y, g), s, t in zip(bodies, a, b):
        s.set_particles(x, y, g)
        t.set_particles(x, y, g)
    N.step_many(a, 6)
    for t in b:
        t.step(6)
    for s, t in zip(a, b):
        xs, ys, gs = s.particles()
        xt, yt, gt = t.particles()
        assert np.array_equal(xs, xt) and np.array_equal(ys, yt) and np.array_equal(gs, gt)
        assert np.array_equal(s.forces(), t.forces())
    for s in a + b:
        s.close()


def run_requests(subs, budget=int(8e9), max_active=8, batched=True):
    """subs: (tick at which to submit, body, steps); returns results by index."""
    srv = N.Server(budget, max_active=max_active)
    srv.set_batched(batched)
    ids = {}
    tick = 0
    while True:
        for k, (at, body, steps) in enumerate(subs):
            if at == tick:
                c, p, x, y, g = body
                ids[k] = srv.submit(c, p, x, y, g, steps)
        res, q = srv.tick()
        tick += 1
        if len(ids) == len(subs) and res == 0 and q == 0:
            break
    out = {k: srv.result(i) for k, i in ids.items()}
    stats = srv.stats()
    srv.close()
    return out, stats


@pytest.mark.parametrize("batched", [True, False])
def test_result_same_alone_and_in_mix(batched):
    """A request's result is the same alone and in a mix that arrives before
    and after it, stepped in one batch with the others (batched) or on its
    own stream beside them; the two ways give the same bits too."""
    A = small_body(0)
    alone, _ = run_requests([(0, A, 12)], batched=batched)
    mix, st = run_requests([(0, small_body(1), 20), (2, A, 12), (3, small_body(2), 5), (7, small_body(3), 9)],
                           batched=batched)
    a, m = alone[0], mix[1]
    assert a["state"] == m["state"] == "done" and a["steps"] == m["steps"] == 12
    assert np.array_equal(a["forces"], m["forces"])
    assert a["n_final"] == m["n_final"]
    assert st["finished"] == 4 and st["step_ms_p99"] >= st["step_ms_p50"] > 0
    assert st["mean_resident"] > 1.0        # the bodies did overlap
    other, _ = run_requests([(0, A, 12)], batched=not batched)
    assert np.array_equal(a["forces"], other[0]["forces"]) and a["n_final"] == other[0]["n_final"]


def test_small_body_is_not_held_back_by_a_large_one():
    """Per-body streams: each body is relaunched as soon as its own step is
    collected: a small
    body finishes its steps while a large one submitted with it, asking for
    as many steps, is still running."""
    big = small_body(0, n0=600000, panels=400)
    small = small_body(1, n0=1000, panels=100)
    srv = N.Server(int(16e9), max_active=4)
    srv.set_batched(False)          # per-body streams (a batch steps its members together)
    ib = srv.submit(*big, 12)
    isml = srv.submit(*small, 12)
    seen = False
    for _ in range(500):
        res, q = srv.tick()
        if srv.result(isml)["state"] == "done" and srv.result(ib)["state"] == "resident":
            seen = True
        if res == 0 and q == 0:
            break
    assert srv.result(ib)["state"] == srv.result(isml)["state"] == "done"
    assert seen
    srv.close()


def test_failed_creation_is_reported_and_the_rest_run():
    """A body whose panel system the reference's pivot rule cannot invert
    (thin rounded plate, gj_pivot 0) fails at creation on the worker thread:
    its request reports "failed", frees its slot and budget, and the request
    submitted with it runs to the end."""
    from tests.helpers import conf_kwargs
    from vortex_b200 import profiles as PR
    pan = PR.rotate(PR.rounded_plate(655), -30.0)
    ck = conf_kwargs(len(pan), ve_size=float(pan["length"].mean()))
    bad = N.default_conf(**dict(ck, gj_pivot=0))
    x, y, g = np.linspace(1.0, 2.0, 10), np.zeros(10), np.full(10, 1e-3)
    srv = N.Server(int(8e9), max_active=4)
    ib = srv.submit(bad, pan, x, y, g, 3)
    ig = srv.submit(*small_body(0), 4)
    for _ in range(200):
        res, q = srv.tick()
        if res == 0 and q == 0:
            break
    assert srv.result(ib)["state"] == "failed"
    assert srv.result(ig)["state"] == "done" and srv.result(ig)["steps"] == 4
    assert srv.stats()["bytes_reserved"] == 0
    srv.close()


def test_admission_by_slots_and_budget():
    body = small_body(0)
    c, p = body[0], body[1]
    est = N.estimate_bytes(c, len(p), len(body[2]) + len(p) * 6)
    # budget for one body at a time: the second waits until the first is done
    srv = N.Server(int(est * 1.5), max_active=4)
    i1 = srv.submit(*body, 6)
    i2 = srv.submit(*body, 6)
    srv.tick()
    assert srv.result(i1)["state"] == "resident" and srv.result(i2)["state"] == "queued"
    ticks = 1
    while srv.result(i2)["state"] != "done":
        srv.tick()
        ticks += 1
        assert ticks < 50
    assert srv.result(i1)["state"] == "done"
    assert ticks >= 12                       # strictly one after the other
    srv.close()
    # a request larger than the whole budget is refused at once
    srv = N.Server(int(est * 0.5), max_active=4)
    with pytest.raises(N.VxError, match="budget"):
        srv.submit(*body, 6)
    srv.close()
    # slots: max_active = 1 serialises as well
    res, st = run_requests([(0, body, 4), (0, small_body(1), 4)], max_active=1)
    assert all(r["state"] == "done" for r in res.values()) and st["mean_resident"] <= 1.0


def test_estimate_covers_resident_bytes():
    c, p, x, y, g = small_body(2)
    s = N.Sim(c, p)
    s.set_particles(x, y, g)
    s.step(10)
    held = s.device_bytes()
    est = N.estimate_bytes(c, len(p), len(x) + 10 * len(p))
    assert held <= est
    s.close()
