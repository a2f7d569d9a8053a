"""Body profiles: generators, rotation and the reference's text format.

The profile format is the one the reference's loader reads
(src/main.c:220-256): two header lines, the panel count P, then P records
``n lx ly rx ry cx cy bx by nx ny tx ty len nL nR``; anything after the last
record is ignored.  Conventions follow the shipped profiles
(profiles/Profile_file_krug_1000.txt): panels run clockwise, the normal is the
outward chord normal, the tangent is the normal turned by +90 degrees, the
control point is the panel midpoint and the birth column is the left endpoint
moved 1e-4 along the normal.

``rotate`` restates turn.py:13-42 (rotation of every vector column about the
origin; lengths and neighbour indices unchanged).
"""
from __future__ import annotations

import math

import numpy as np

# 120-byte record with the layout of the reference's tPanel
# (include/definitions.h:82-103); shared with the C ABI (vx_panel).
PANEL_DTYPE = np.dtype([
    ("n", "<u4"), ("pad", "<u4"),
    ("left", "<f8", 2), ("right", "<f8", 2), ("contr", "<f8", 2),
    ("birth", "<f8", 2), ("norm", "<f8", 2), ("tang", "<f8", 2),
    ("length", "<f8"), ("nl", "<u4"), ("nr", "<u4"),
])
assert PANEL_DTYPE.itemsize == 120

BIRTH_OFFSET = 1e-4


def panels_from_polygon(pts: np.ndarray) -> np.ndarray:
    """Closed polygon (P,2) traversed clockwise -> panel records."""
    pts = np.asarray(pts, dtype=np.float64)
    P = len(pts)
    pan = np.zeros(P, dtype=PANEL_DTYPE)
    left = pts
    right = np.roll(pts, -1, axis=0)
    ch = right - left
    length = np.hypot(ch[:, 0], ch[:, 1])
    norm = np.stack([-ch[:, 1], ch[:, 0]], axis=1) / length[:, None]
    tang = np.stack([-norm[:, 1], norm[:, 0]], axis=1)
    pan["n"] = np.arange(P)
    pan["left"] = left
    pan["right"] = right
    pan["contr"] = 0.5 * (left + right)
    pan["birth"] = left + BIRTH_OFFSET * norm
    pan["norm"] = norm
    pan["tang"] = tang
    pan["length"] = length
    pan["nl"] = (np.arange(P) - 1) % P
    pan["nr"] = (np.arange(P) + 1) % P
    return pan


def circle(P: int, R: float = 0.5) -> np.ndarray:
    """Circle of radius R with P equal panels, starting at (-R, 0), clockwise."""
    th = math.pi - 2.0 * math.pi * np.arange(P) / P
    return panels_from_polygon(np.stack([R * np.cos(th), R * np.sin(th)], axis=1))


def ellipse(P: int, a: float = 0.5, b: float = 0.25) -> np.ndarray:
    """Ellipse with semi-axes a (x) and b (y), P panels, clockwise from (-a,0)."""
    th = math.pi - 2.0 * math.pi * np.arange(P) / P
    return panels_from_polygon(np.stack([a * np.cos(th), b * np.sin(th)], axis=1))


def rounded_plate(P: int, chord: float = 1.0, thickness: float = 0.02,
                  n_end: int | None = None) -> np.ndarray:
    """Flat plate with semicircular ends (the shape of
    profiles/Profile_file_plas_2576.txt): n_end panels per quarter of each
    end circle (four quarters in all), the rest split between the two flat
    sides (the upper side takes the odd one).  By default n_end makes the
    end panels as long as the flat ones, as in the shipped plate (P = 2576,
    chord 1, thickness 0.02: 20 per quarter, 1248 per side, every panel
    pi * 0.01 / 40 long); strongly unequal panel lengths make the panel
    system singular.  Clockwise from the leading edge."""
    r = 0.5 * thickness
    if n_end is None:
        ell = (2.0 * (chord - 2.0 * r) + 2.0 * math.pi * r) / P
        n_end = max(1, int(round(0.5 * math.pi * r / ell)))
    n_rest = P - 4 * n_end
    n_top, n_bot = (n_rest + 1) // 2, n_rest // 2
    if n_bot < 1:
        raise ValueError("P too small for the end panels")
    xl, xr = -0.5 * chord + r, 0.5 * chord - r
    pts = []
    for k in range(n_end):                      # leading edge, pi -> pi/2
        a = math.pi - 0.5 * math.pi * k / n_end
        pts.append((xl + r * math.cos(a), r * math.sin(a)))
    for k in range(n_top):                      # upper side, left -> right
        pts.append((xl + (xr - xl) * k / n_top, r))
    for k in range(2 * n_end):                  # trailing edge, pi/2 -> -pi/2
        a = 0.5 * math.pi - math.pi * k / (2 * n_end)
        pts.append((xr + r * math.cos(a), r * math.sin(a)))
    for k in range(n_bot):                      # lower side, right -> left
        pts.append((xr - (xr - xl) * k / n_bot, -r))
    for k in range(n_end):                      # back to the leading edge
        a = -0.5 * math.pi - 0.5 * math.pi * k / n_end
        pts.append((xl + r * math.cos(a), r * math.sin(a)))
    return panels_from_polygon(np.array(pts))


def rotate(pan: np.ndarray, angle_deg: float) -> np.ndarray:
    """Rotate every vector column about the origin (turn.py:13-42)."""
    c, s = math.cos(math.radians(angle_deg)), math.sin(math.radians(angle_deg))
    m = np.array([[c, -s], [s, c]])
    out = pan.copy()
    for f in ("left", "right", "contr", "birth", "norm", "tang"):
        out[f] = pan[f] @ m.T
    return out


def write_profile(path, pan: np.ndarray, fmt: str = "%.17g") -> None:
    with open(path, "w") as fh:
        fh.write("--profile-vortex-b200--\n--panel-records--\n")
        fh.write(f"{len(pan)}\n")
        for p in pan:
            vals = [p["left"][0], p["left"][1], p["right"][0], p["right"][1],
                    p["contr"][0], p["contr"][1], p["birth"][0], p["birth"][1],
                    p["norm"][0], p["norm"][1], p["tang"][0], p["tang"][1], p["length"]]
            fh.write(f"{int(p['n'])} " + " ".join(fmt % v for v in vals)
                     + f" {int(p['nl'])} {int(p['nr'])}\n")


def read_profile(path) -> np.ndarray:
    """Parse like src/main.c:226-240 (two header lines skipped, then P)."""
    with open(path, "rb") as fh:
        lines = fh.read().split(b"\n")
    toks = b" ".join(lines[2:]).split()
    P = int(toks[0])
    pan = np.zeros(P, dtype=PANEL_DTYPE)
    for i in range(P):
        r = toks[1 + 16 * i: 1 + 16 * (i + 1)]
        pan[i]["n"] = int(r[0])
        v = [float(t) for t in r[1:14]]
        pan[i]["left"] = v[0:2]
        pan[i]["right"] = v[2:4]
        pan[i]["contr"] = v[4:6]
        pan[i]["birth"] = v[6:8]
        pan[i]["norm"] = v[8:10]
        pan[i]["tang"] = v[10:12]
        pan[i]["length"] = v[12]
        pan[i]["nl"] = int(r[14])
        pan[i]["nr"] = int(r[15])
    return pan


def profile_bbox(pan: np.ndarray, window=(-1e300, 1e300, -1e300, 1e300)):
    """Profile bounding box from the LEFT endpoints only, started from the
    window's opposite edges (src/main.c:235-254).  window = (x_min, x_max,
    y_min, y_max).  Returns (x_min, x_max, y_min, y_max)."""
    x_min, x_max = window[1], window[0]
    y_min, y_max = window[3], window[2]
    for lx, ly in pan["left"]:
        if lx < x_min: x_min = lx
        if lx > x_max: x_max = lx
        if ly < y_min: y_min = ly
        if ly > y_max: y_max = ly
    return x_min, x_max, y_min, y_max
