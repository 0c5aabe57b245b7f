"""C-ABI checks that need no GPU: the library loads, exports every entry point include/xpgi.h declares, and the
ctypes mirrors of the header's structs have the C layout (sizes and field offsets compiled with gcc)."""
from __future__ import annotations

import re
import subprocess
from pathlib import Path

import pytest

from xpg_b200 import native as N

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "xpgi.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(xi_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = N.load()
    names = declared_functions()
    assert names, "no xi_* declarations found"
    for name in names:
        assert hasattr(lib, name), name
    assert lib.xi_version() >= 1


def test_struct_layouts_match_header(tmp_path):
    structs = {"XiDetector": N.XiDetector, "XiRows": N.XiRows, "XiRowSet": N.XiRowSet, "XiGatherStep": N.XiGatherStep, "XiPackedFrame": N.XiPackedFrame, "XiBlock": N.XiBlock, "XiPass1Out": N.XiPass1Out,
               "XiPass2In": N.XiPass2In, "XiPass2Out": N.XiPass2Out, "XiGatherRows": N.XiGatherRows,
               "XiFrames": N.XiFrames, "XiPlanDetector": N.XiPlanDetector, "XiPredict": N.XiPredict,
               "XiPredictOut": N.XiPredictOut, "XiBoxRules": N.XiBoxRules, "XiBoxOut": N.XiBoxOut, "XiKnn": N.XiKnn,
               "XiRocking": N.XiRocking, "XiFmBoxes": N.XiFmBoxes, "XiFmWindow": N.XiFmWindow}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "xpgi.h"', "int main(void) {"]
    for name, cls in structs.items():
        lines.append(f'printf("{name} %zu\\n", sizeof({name}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{name}.{fname} %zu\\n", offsetof({name}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    r = subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], capture_output=True, text=True)
    if r.returncode != 0:
        pytest.skip("gcc unavailable: " + r.stderr[-200:])
    out = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split("\n") if line)
    for name, cls in structs.items():
        import ctypes
        assert int(out[name]) == ctypes.sizeof(cls), name
        for fname, _ in cls._fields_:
            assert int(out[f"{name}.{fname}"]) == getattr(cls, fname).offset, f"{name}.{fname}"


def test_no_device_without_cuda():
    """The product has no CPU path: without a CUDA device the integration refuses to run."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(RuntimeError):
        N.require_cuda()
