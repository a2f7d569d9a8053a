"""Seeded workloads: the SplitMix64 stream against the generator's published
first outputs, the derived uniform / normal draws, and the multi-body
population's ranges."""
import numpy as np

from vortex_b200 import workloads as wl


def test_splitmix64_known_answer():
    # first outputs of SplitMix64 seeded with 1234567 (the generator's published test values)
    assert [int(v) for v in wl.splitmix64(1234567, 3)] == [6457827717110365317, 3203168211198807973,
                                                            9817491932198370423]
    # a stream can be resumed at any offset
    assert np.array_equal(wl.splitmix64(99, 10)[4:], wl.splitmix64(99, 6, offset=4))


def test_uniform_and_normal_draws():
    u = wl.uniforms(3, 200000)
    assert u.min() >= 0.0 and u.max() < 1.0 and abs(u.mean() - 0.5) < 0.005
    z = wl.normals(3, 200001)
    assert len(z) == 200001 and abs(z.mean()) < 0.01 and abs(z.std() - 1.0) < 0.01


def test_body_population_ranges():
    specs = [wl.body_spec(7, i) for i in range(256)]
    P = np.array([s["panels"] for s in specs])
    n = np.array([s["n0"] for s in specs])
    re = np.array([s["re"] for s in specs])
    assert P.min() >= 200 and P.max() <= 3320 and n.min() >= 1000 and n.max() <= 500000
    assert re.min() >= 500 and re.max() <= 2e4
    assert 64 < sum(s["kind"] == "plate" for s in specs) < 192
    assert all(abs(s["dt"] - 1.0 / s["panels"]) < 1e-12 for s in specs)
    assert specs[3] == wl.body_spec(7, 3)     # deterministic


def test_make_body_cloud():
    sp = dict(wl.body_spec(7, 0), n0=20000)
    conf, pan, x, y, g = wl.make_body(sp, 1)
    assert len(x) == 20000 and x.min() >= 0.55 and x.max() <= 4.55 and y.min() >= -1 and y.max() <= 1
    assert abs(g.std() - 1e-3) < 5e-5
    assert abs(conf.ve_size - pan["length"].mean()) < 1e-15
