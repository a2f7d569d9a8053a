"""Golden panel matrices from the reference's own matr_creation.

Calls matr_creation (src/unit_1.cu:256-402, host code) in the reference
build oracle/_ref/libvortex_ref.so (made by oracle/build_ref.sh) on circles of
40 and 200 panels from vortex_b200.profiles.circle and stores the unpadded
(P+1)^2 inverse:

    python tests/golden/make_ref_matrix.py
"""
import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

from oracle import refdrv  # noqa: E402
from vortex_b200 import profiles  # noqa: E402

if __name__ == "__main__":
    out = {}
    for P in (40, 200):
        M = refdrv.matr_creation(profiles.circle(P))
        out[f"circle{P}"] = M[:P + 1, :P + 1]
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_matrix.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path))
