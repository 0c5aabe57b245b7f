"""Build libxpgi.so (the C-ABI kernel library) in-tree with nvcc for sm_100a.

    python -m xpg_b200.csrc.build [--verbose]

-fmad=false: float expressions are not contracted into fused multiply-adds (the kernels place fmaf() where the
reference's arithmetic fuses); division and square root stay IEEE (-prec-div / -prec-sqrt default to true).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
LIB_DIR = HERE.parent / "_lib"
LIB = LIB_DIR / "libxpgi.so"
SOURCES = [HERE / "xpgi.cu", HERE / "xpgi_plan.cu", HERE / "xpgi_adapt.cu", HERE / "xpgi_synth.cu",
           HERE / "xpgi_forward.cu", HERE / "xpgi_frames.cu", HERE / "xpgi_spot.cu", HERE / "xpgi_pack.cpp"]
DEPS = SOURCES + [HERE / "xpgi_device.cuh", HERE / "xpgi_internal.h", HERE / "xpgi_synth.h", ROOT / "include" / "xpgi.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def stale():
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in DEPS)


def build(force=False, verbose=False):
    if not force and not stale():
        return LIB
    LIB_DIR.mkdir(exist_ok=True)
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-fmad=false", "-std=c++17", "--shared", "-Xcompiler", "-fPIC",
           "-I", str(ROOT / "include"), "-I", str(HERE), "-o", str(LIB) + ".tmp", *map(str, SOURCES)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stderr[-8000:])
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(str(LIB) + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose="--verbose" in sys.argv))
