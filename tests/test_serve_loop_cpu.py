"""Host logic of the served run (vortex_b200.multibody.run_serve) on CPU,
against a stand-in for the native server: requests are submitted at their
Poisson arrival times, the loop ends exactly when every submitted request
has left the server (done or failed), it sleeps through gaps in which
nothing is resident or queued, and the record is built from the server's
own counters."""
import numpy as np

from vortex_b200 import multibody as MB


class FakeServer:
    """Admits up to max_active requests; each tick advances every resident
    request one step; a request asking for 0 steps fails at admission."""
    instances = []

    def __init__(self, budget, max_active=4, device=0):
        self.max_active = max_active
        self.queue, self.resident, self.res = [], [], {}
        self.ticks = 0
        self.body_steps = 0
        FakeServer.instances.append(self)

    def set_batched(self, on):
        self.batched = bool(on)

    def submit(self, conf, pan, x, y, g, nsteps):
        rid = len(self.res) + 1
        self.res[rid] = {"state": "queued", "steps": 0, "want": nsteps}
        self.queue.append(rid)
        return rid

    def tick(self):
        while self.queue and len(self.resident) < self.max_active:
            rid = self.queue.pop(0)
            if self.res[rid]["want"] == 0:
                self.res[rid]["state"] = "failed"
                continue
            self.res[rid]["state"] = "resident"
            self.resident.append(rid)
        for rid in list(self.resident):
            r = self.res[rid]
            r["steps"] += 1
            self.body_steps += 1
            if r["steps"] == r["want"]:
                r["state"] = "done"
                self.resident.remove(rid)
        self.ticks += 1
        return len(self.resident), len(self.queue)

    def result(self, rid):
        r = self.res[rid]
        out = {"state": r["state"], "steps": r["steps"], "forces": np.zeros((r["steps"], 4)), "n_final": 0}
        if r["state"] == "failed":
            out["error"] = "creation: out of memory"
        return out

    def stats(self):
        return {"finished": sum(r["state"] == "done" for r in self.res.values()), "step_ms_p50": 1.0,
                "step_ms_p99": 2.0, "ttc_s_p50": 0.5, "ttc_s_p99": 0.9, "mean_resident": 1.5,
                "body_steps": self.body_steps, "particle_steps": 10.0 * self.body_steps, "ticks": self.ticks}

    def close(self):
        pass


def test_serve_loop_submits_on_arrival_and_ends_when_all_have_left(monkeypatch):
    FakeServer.instances.clear()
    monkeypatch.setattr(MB.N, "Server", FakeServer)
    monkeypatch.setattr(MB.wl, "make_body", lambda spec, prec: (None, None, None, None, None))
    out = MB.run_serve(requests=12, rate=200.0, steps_lo=3, steps_hi=9, seed=5)
    srv = FakeServer.instances[-1]
    assert len(srv.res) == 12                          # every request was submitted
    assert all(r["state"] == "done" for r in srv.res.values())
    assert out["body_steps"] == out["steps_requested"] == sum(r["want"] for r in srv.res.values())
    assert out["failed"] == 0 and out["ticks"] == srv.ticks
    assert out["wall_s"] > 0 and out["body_steps_per_s"] == out["body_steps"] / out["wall_s"]


def test_serve_loop_counts_failed_requests(monkeypatch):
    FakeServer.instances.clear()
    monkeypatch.setattr(MB.N, "Server", FakeServer)
    monkeypatch.setattr(MB.wl, "make_body", lambda spec, prec: (None, None, None, None, None))
    # steps_lo = steps_hi = 0: every request fails at admission, none is ever resident
    out = MB.run_serve(requests=5, rate=500.0, steps_lo=0, steps_hi=0, seed=6)
    assert out["failed"] == 5 and out["body_steps"] == 0
    assert len(FakeServer.instances[-1].res) == 5
