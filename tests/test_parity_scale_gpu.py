"""Stage-by-stage parity of the plain FP64 form with the CPU oracle on the
configurations' own bodies, through the C ABI: the 1000-panel cylinder of
the benchmark and the 2576-panel rounded plate at 20 degrees of incidence,
each with a seeded wake-like cloud of 16 000 vortices around and behind it.

Bounds: new-vortex positions, the 3-nearest distance d, convection with
absorption, compaction (every slot, the dead tail included), collapse
pairing and merges bit-exact; velocities within 1e-12 of the field's
largest component (the sums run in another order than the oracle's
sequential ones: at 16 000 sources and fields of order 1 to 30 the
differences are a few 1e-14 of the field); birth strengths within 1e-10 of
the largest; wall diffusion 1e-13.
The panel system: the device's Gauss-Jordan (the reference's pivot rule)
against the oracle's.  Both are inverses with a residual R = L M - I of
their own (1e-14 for the circle; of order 1e-4 for the plate, the
reference's own result with its pivot rule), so they can differ by
|M_dev - M| <= |M|_inf (|R_dev| + |R|) (max norms, |M|_inf the largest row
sum): the test holds the difference to twice that, and the device's
residual to ten times the oracle's.  The birth strengths are compared with
the device's matrix.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import body_cloud, oracle_params, rel_err, scale_body, with_tail
from vortex_b200 import native as N

pytestmark = pytest.mark.gpu

BODIES = ["circle1000", "plate2576"]
VEL_REL = 1e-12
N_CLOUD = 16000


def make(name, **kw):
    pan, ck = scale_body(name)
    ck = dict(ck, **kw)
    sim = N.Sim(N.default_conf(**ck), pan)
    return sim, pan, ck, oracle_params(pan, ck)


@pytest.mark.parametrize("name", BODIES)
def test_panel_matrix_and_birth(name):
    sim, pan, ck, p = make(name)
    P = len(pan)
    L, M = O.panel_matrix(pan)
    Mg = sim.matrix()
    eye = np.eye(len(M))
    res_o = np.abs(L @ M - eye).max()
    res_d = np.abs(L @ Mg - eye).max()
    bound = 2.0 * np.abs(M).sum(axis=1).max() * (res_d + res_o)
    assert np.abs(Mg - M).max() <= bound, (np.abs(Mg - M).max(), bound)
    assert res_d <= 10.0 * res_o + 1e-13, (res_d, res_o)
    if name == "circle1000":
        assert rel_err(Mg, M) < 1e-11, rel_err(Mg, M)
    x, y, g = with_tail(*body_cloud(pan, N_CLOUD, seed=1), extra=96)
    n = N_CLOUD
    sim.set_slots(x, y, g, n)
    sim.set_dg(2.5e-3)
    sim.stage("birth")
    assert sim.count() == n + P
    gx, gy, gg = sim.get_slots(n + P)
    R = O.birth_rhs(p, pan, x[:n], y[:n], g[:n])
    gam = O.birth_gamma(Mg, R, 2.5e-3)
    bx, by, bg = O.birth_place(p, pan, gam)
    assert np.array_equal(gx[:n], x[:n]) and np.array_equal(gg[:n], g[:n])
    assert np.array_equal(gx[n:], bx) and np.array_equal(gy[n:], by)
    assert rel_err(gg[n:], bg) < 1e-10
    sim.close()


@pytest.mark.parametrize("name", BODIES)
def test_velocity_nearest_and_diffusion(name):
    sim, pan, ck, p = make(name)
    x, y, g = with_tail(*body_cloud(pan, N_CLOUD, seed=2), extra=64)
    n = N_CLOUD
    sim.set_slots(x, y, g, n)
    sim.stage("velocity")
    vx, vy, d = sim.velocity()
    ovx, ovy, od = O.velocity(p, x, y, g, n)
    assert np.array_equal(d, od), "3-nearest distance must be bit-exact"
    assert rel_err(vx, ovx) < VEL_REL and rel_err(vy, ovy) < VEL_REL
    # vortex diffusion from the oracle's velocities and distances
    sim.set_velocity(ovx, ovy, od)
    sim.stage("diffusion")
    dvx, dvy, _ = sim.velocity()
    evx, evy = O.diffusion(p, x, y, g, n, od, ovx, ovy)
    assert rel_err(dvx, evx) < VEL_REL and rel_err(dvy, evy) < VEL_REL
    sim.close()


@pytest.mark.parametrize("name", BODIES)
def test_wall_diffusion(name):
    sim, pan, ck, p = make(name)
    rng = np.random.default_rng(7)
    n = 6000
    k = rng.integers(0, len(pan), n)
    off = rng.uniform(0.0, 8.0, n) * pan["length"][k]
    off[:60] = 1e-6                    # on top of birth points: the override branch
    x = pan["birth"][k, 0] + off * pan["norm"][k, 0]
    y = pan["birth"][k, 1] + off * pan["norm"][k, 1]
    g = rng.normal(0, 1e-3, n)
    d = rng.uniform(0.2, 3.0, n) * float(pan["length"].mean())
    vx0, vy0 = np.ones(n), np.zeros(n)
    sim.set_particles(x, y, g)
    sim.set_velocity(vx0, vy0, d)
    sim.stage("wall")
    vx, vy, _ = sim.velocity()
    evx, evy = O.wall_diffusion(p, pan, x, y, n, d, vx0, vy0)
    assert np.abs(vx - evx).max() < 1e-13 and np.abs(vy - evy).max() < 1e-13
    assert np.abs(evx - 1).max() > 1e-6
    sim.close()


@pytest.mark.parametrize("name", BODIES)
def test_advect_absorb_and_forces(name):
    sim, pan, ck, p = make(name)
    rng = np.random.default_rng(3)
    x, y, g = body_cloud(pan, N_CLOUD, seed=3)
    n = N_CLOUD
    dt = ck["dt"]
    vx = rng.normal(0, 2.0, n)
    vy = rng.normal(0, 2.0, n)
    k = rng.choice(n, 800, replace=False)          # driven through the wall
    cx, cy = pan["contr"][:, 0].mean(), pan["contr"][:, 1].mean()
    vx[k] = (cx - x[k]) / dt * 0.9
    vy[k] = (cy - y[k]) / dt * 0.9
    x[:30] = 9.999
    vx[:30] = 50.0                                  # out of the window
    sim.set_particles(x, y, g)
    sim.set_velocity(vx, vy, np.ones(n))
    sim.stage("advect")
    gx, gy, gg = sim.get_slots(n)
    ox, oy, og, t = O.advect(p, pan, x, y, g, vx, vy, n, len(pan))
    assert np.array_equal(gx, ox) and np.array_equal(gy, oy) and np.array_equal(gg, og)
    assert (og == 0).sum() > 200
    dg, fx, fy, m = O.sums(p, t)
    f = sim.forces()
    assert abs(f[0] - dg) <= 1e-13 * max(1.0, abs(dg))
    for a, b in ((f[1], fx), (f[2], fy), (f[3], m)):
        assert abs(a - b) <= 1e-10 * max(1.0, abs(b))
    sim.close()


@pytest.mark.parametrize("name", BODIES)
def test_compaction_exact(name):
    sim, pan, ck, p = make(name)
    rng = np.random.default_rng(4)
    x, y, g = body_cloud(pan, N_CLOUD, seed=4)
    n = N_CLOUD
    g[rng.random(n) < 0.3] = 0.0
    g[rng.random(n) < 0.01] = 1e-13
    xs, ys, gs = with_tail(x, y, g, extra=64)
    sim.set_slots(xs, ys, gs, n)
    sim.stage("compact")
    ox, oy, og, m = O.compact(xs, ys, gs, n)
    assert sim.count() == m
    gx, gy, gg = sim.get_slots(len(xs))
    assert np.array_equal(gx, ox) and np.array_equal(gy, oy) and np.array_equal(gg, og)
    sim.close()


@pytest.mark.parametrize("name", BODIES)
@pytest.mark.parametrize("pas", [1, 2])
def test_collapse_exact(name, pas):
    sim, pan, ck, p = make(name, r_col_diff_sign=0.8, r_col_same_sign=0.6, max_ve_g=3e-3, n_col=3)
    rng = np.random.default_rng(11 + pas)
    n = N_CLOUD
    eps = ck["ve_size"]
    # clusters of vortices a fraction of eps apart, so chains of candidates form
    cx, cy, _ = body_cloud(pan, 800, seed=20 + pas)
    idx = rng.integers(0, 800, n)
    x = cx[idx] + rng.normal(0, 0.6 * eps, n)
    y = cy[idx] + rng.normal(0, 0.6 * eps, n)
    g = rng.normal(0, 1e-3, n)
    xs, ys, gs = with_tail(x, y, g, extra=32)
    sim.set_slots(xs, ys, gs, n)
    sim.stage("collapse1" if pas == 1 else "collapse2")
    ox, oy, og, m = O.collapse(p, pas, xs, ys, gs, n)
    assert m < n - 200, "the scene must exercise merging"
    assert sim.count() == m
    gx, gy, gg = sim.get_slots(len(xs))
    assert np.array_equal(gx, ox) and np.array_equal(gy, oy) and np.array_equal(gg, og)
    sim.close()


@pytest.mark.parametrize("name", BODIES)
def test_whole_steps_track_oracle(name):
    """Five whole steps from the seeded cloud: the count follows the oracle
    exactly and positions and strengths stay within 1e-9."""
    sim, pan, ck, p = make(name, birth_offset_mode=2)
    M = sim.matrix()
    x, y, g = body_cloud(pan, 6000, seed=5)
    sim.set_particles(x, y, g)
    osim = O.OracleSim(p, pan, M)
    osim.load(x, y, g)
    for k in range(5):
        sim.step(1)
        osim.step()
        assert sim.count() == osim.n, f"step {k}"
    gx, gy, gg = sim.particles()
    ox, oy, og = osim.particles()
    assert np.abs(gx - ox).max() < 1e-9 and np.abs(gy - oy).max() < 1e-9
    assert np.abs(gg - og).max() < 1e-9 * np.abs(og).max()
    sim.close()
