"""Record the reference's shipped 1000-panel circle profile
(profiles/Profile_file_krug_1000.txt of the reference checkout) as a small
fixture, so the profile generator can be checked against it without the
checkout:

    VX_REFERENCE_DIR=<reference checkout> python tests/golden/make_profile_golden.py

Writes tests/golden/krug_1000_profile.npz (the panel columns as printed in
the file, 6 decimals for the geometry).
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

from vortex_b200 import profiles  # noqa: E402


def main():
    ref = os.environ.get("VX_REFERENCE_DIR", "/root/reference")
    pan = profiles.read_profile(os.path.join(ref, "profiles", "Profile_file_krug_1000.txt"))
    out = {f: np.asarray(pan[f]) for f in ("left", "right", "contr", "birth", "norm", "tang", "length", "nl", "nr")}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "krug_1000_profile.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path))


if __name__ == "__main__":
    main()
