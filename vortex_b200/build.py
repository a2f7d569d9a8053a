"""Build libvortex_b200.so (all CUDA sources for sm_100a) and the vortex CLI.

    python -m vortex_b200.build          # incremental
    python -m vortex_b200.build --force

Every .cu/.cpp under csrc/ is compiled with nvcc for sm_100a with
-fmad=false (fused multiply-adds are written out explicitly; see
csrc/vx_internal.cuh) and linked into vortex_b200/libvortex_b200.so, in tree,
so the built library travels with the source tree.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libvortex_b200.so")
CLI = os.path.join(HERE, "bin", "vortex")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=default", "-I" + os.path.join(HERE, "..", "include")]
# Build knobs for measuring kernel variants, e.g.
#   VX_NVCC_DEFS="-DVX_DIFF_POLY_EVERY=4" python -m vortex_b200.build --force
FLAGS += os.environ.get("VX_NVCC_DEFS", "").split()
CLI_SOURCES = {"vortex_cli.cpp"}


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")) and f not in CLI_SOURCES)


def _headers_mtime():
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    paths += [os.path.join(HERE, "..", "include", f) for f in os.listdir(os.path.join(HERE, "..", "include"))]
    return max(os.path.getmtime(p) for p in paths)


def _compile(src, force, hdr_mtime, verbose):
    s = os.path.join(CSRC, src)
    o = os.path.join(OBJ, src + ".o")
    if not force and os.path.exists(o) and os.path.getmtime(o) >= max(os.path.getmtime(s), hdr_mtime):
        return o
    cmd = [NVCC, *FLAGS, *ARCH, "-c", s, "-o", o]
    if src.endswith(".cpp"):
        cmd = [NVCC, *FLAGS, "-x", "c++", "-c", s, "-o", o]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return o


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hm = _headers_mtime()
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, hm, verbose), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        tmp = LIB + ".tmp"          # linked aside, then renamed: the library is never seen half written
        cmd = [NVCC, "-shared", "--cudart", "shared", *ARCH, "-o", tmp, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stderr)
        os.replace(tmp, LIB)
    cli_src = os.path.join(CSRC, "vortex_cli.cpp")
    if os.path.exists(cli_src):
        os.makedirs(os.path.dirname(CLI), exist_ok=True)
        if force or not os.path.exists(CLI) or os.path.getmtime(CLI) < max(os.path.getmtime(cli_src),
                                                                             os.path.getmtime(LIB)):
            cmd = ["g++", "-O2", "-std=c++17", "-I" + os.path.join(HERE, "..", "include"), cli_src,
                   "-o", CLI, "-L" + HERE, "-lvortex_b200", "-Wl,-rpath,$ORIGIN/..",
                   "-L/usr/local/cuda/lib64", "-lcudart"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError("CLI build failed:\n" + r.stderr)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true", help="print ptxas register/spill info")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
