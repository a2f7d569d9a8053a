"""Profile generators: the rounded plate reproduces the layout of the shipped
2576-panel plate (20 panels per quarter end circle, 1248 per flat side,
every panel about pi * 0.01 / 40 long, clockwise from the leading point), other
panel counts keep the panel lengths nearly equal, and the reference's text
format round-trips."""
import math

import numpy as np

from vortex_b200 import profiles


def test_rounded_plate_matches_shipped_layout():
    pan = profiles.rounded_plate(2576)
    assert len(pan) == 2576
    assert np.abs(pan["length"] - math.pi * 0.01 / 40).max() < 5e-7   # chords of the end arcs
    assert np.allclose(pan["left"][0], [-0.5, 0.0]) and pan["left"][1][1] > 0   # up the leading edge first
    assert np.allclose(pan["left"][20], [-0.49, 0.01])                            # end of the first quarter
    for P in (200, 201, 655, 3320):
        p = profiles.rounded_plate(P)
        assert len(p) == P
        assert p["length"].min() / p["length"].max() > 0.5


def test_profile_round_trip(tmp_path):
    pan = profiles.rotate(profiles.rounded_plate(400), -20.0)
    f = tmp_path / "plate.txt"
    profiles.write_profile(str(f), pan)
    back = profiles.read_profile(str(f))
    for k in ("left", "right", "contr", "birth", "norm", "tang", "length"):
        assert np.array_equal(back[k], pan[k]), k
