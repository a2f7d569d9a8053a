"""The C-ABI library loads, exports every function its headers declare, and
its host-only entry points (config and profile parsing) work without a GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from vortex_b200 import native as N
from vortex_b200 import profiles

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared_functions():
    names = set()
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        txt = re.sub(r"//[^\n]*", "", txt)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", txt, flags=re.M):
            nm = m.group(1)
            if nm not in ("if", "while", "for", "return", "sizeof", "defined"):
                names.add(nm)
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = N.lib()
    missing = [nm for nm in declared_functions() if not hasattr(lib, nm)]
    assert not missing, missing
    assert len(declared_functions()) >= 20


def test_conf_parser_follows_reference_rules(tmp_path):
    f = tmp_path / "run.conf"
    f.write_text(
        "steps 400                 # comment after the value\n"
        "saving_step 50\n"
        "dt 0.005\n"
        "ve_size 0.0157\n"
        "r_col_same_sign 0.3\n"
        "stepsX 9\n"                    # not a key: no space after 'steps'
        "unknown_key 12\n"
        "pr_file profiles/x.txt  # file\n"
        "matrix_load 1\n"
        "precision fp32\n"
        "birth_offset_mode half_panel\n"
        "drop_eps 1e-8\n")
    c = N.read_conf(str(f))
    assert c.steps == 400 and c.saving_step == 50 and c.dt == 0.005
    assert c.ve_size == 0.0157 and c.r_col_same_sign == 0.3
    assert c.pr_file == b"profiles/x.txt" and c.matrix_load == 1
    assert c.precision == N.PREC_FP32 and c.birth_offset_mode == N.BIRTH_HALF_PANEL
    assert c.drop_eps == 1e-8
    assert c.v_inf_incr_steps == 0   # default_conf baseline in this binding


def test_conf_defaults_match_reference_main():
    c = N.Conf()
    assert N.lib().vx_conf_default(C.byref(c)) == 0
    assert c.log_level == 3 and c.v_inf_incr_steps == 1 and c.drop_eps == 1e-12


def test_profile_reader_round_trip(tmp_path):
    pan = profiles.rotate(profiles.ellipse(333, 0.5, 0.1), 12.5)
    p = tmp_path / "prof.txt"
    profiles.write_profile(p, pan)
    with open(p, "a") as fh:
        fh.write("0.098\n--trailer--\n-0.5 -0.5 0.5 0.5\n")   # trailer lines are ignored
    rd = N.read_profile(str(p))
    assert len(rd) == 333
    for f in ("left", "right", "contr", "birth", "norm", "tang", "length", "nl", "nr"):
        assert np.array_equal(rd[f], pan[f])


def test_profile_reader_errors(tmp_path):
    p = tmp_path / "bad.txt"
    p.write_text("h1\nh2\n3\n0 1 2 3\n")
    with pytest.raises(N.VxError):
        N.read_profile(str(p))
    with pytest.raises(N.VxError):
        N.read_profile(str(tmp_path / "missing.txt"))
