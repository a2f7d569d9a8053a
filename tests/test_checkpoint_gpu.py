"""Binary checkpoints (vx_checkpoint_save / vx_checkpoint_load): a body
continued from a checkpoint in a fresh handle steps bit for bit as the body
that wrote it went on stepping, in both forms, with the V_inf ramp half way
through at the checkpoint; a checkpoint of another body, or a damaged file,
is refused."""
import numpy as np
import pytest

from tests.helpers import conf_kwargs, wake_cloud
from vortex_b200 import native as N
from vortex_b200 import profiles

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [N.PREC_FP64, N.PREC_FP32])
def test_checkpoint_continues_bit_identically(tmp_path, prec):
    ck = conf_kwargs(200, precision=prec, v_inf_incr_steps=10)
    pan = profiles.circle(200)
    x, y, g = wake_cloud(4000 if prec == N.PREC_FP64 else 20000, seed=17)
    path = str(tmp_path / "body.ckpt")
    a = N.Sim(N.default_conf(**ck), pan)
    a.set_particles(x, y, g)
    a.step(5)
    a.checkpoint_save(path)
    a.step(5)
    b = N.Sim(N.default_conf(**ck), pan)
    b.checkpoint_load(path)
    b.step(5)
    for u, w in zip(a.particles(), b.particles()):
        assert np.array_equal(u, w)
    assert np.array_equal(a.forces(), b.forces())
    assert np.array_equal(a.state(), b.state())
    a.close()
    b.close()


def test_checkpoint_refuses_another_body(tmp_path):
    ck = conf_kwargs(200)
    a = N.Sim(N.default_conf(**ck), profiles.circle(200))
    a.set_particles(*wake_cloud(500, seed=3))
    a.step(1)
    path = str(tmp_path / "body.ckpt")
    a.checkpoint_save(path)
    other = N.Sim(N.default_conf(**conf_kwargs(100)), profiles.circle(100))
    with pytest.raises(N.VxError):
        other.checkpoint_load(path)
    bulk = N.Sim(N.default_conf(**dict(ck, precision=N.PREC_FP32)), profiles.circle(200))
    with pytest.raises(N.VxError):
        bulk.checkpoint_load(path)
    bad = tmp_path / "bad.ckpt"
    bad.write_bytes(open(path, "rb").read()[:200])
    with pytest.raises(N.VxError):
        a.checkpoint_load(str(bad))
    for s in (a, other, bulk):
        s.close()
