"""The ctypes mirror of the C ABI (ptir_b200/_native.py) has the layout of include/ptir_b200.h.

A small C program compiled against the header prints the size of every struct the Python side
passes by pointer and the offset of each of its fields. The ctypes structs must agree field by
field, in the same order, so that adding a field on one side only fails here and not as silently
misread arguments. CPU only (gcc).
"""
import ctypes as C
import os
import shutil
import subprocess

import pytest

from ptir_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STRUCTS = {
    "ptir_config": N.PtirConfig,
    "ptir_trace_args": N.PtirTraceArgs,
    "ptir_trace_outputs": N.PtirTraceOutputs,
    "ptir_bwd_args": N.PtirBwdArgs,
    "ptir_bwd_outputs": N.PtirBwdOutputs,
    "ptir_counters": N.PtirCounters,
    "ptir_stage_times": N.PtirStageTimes,
    "ptir_view": N.PtirView,
}


def _c_layout(tmp_path) -> dict:
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "ptir_b200.h"', "int main(void) {"]
    for name, cls in STRUCTS.items():
        lines.append(f'    printf("{name} size %zu\\n", sizeof({name}));')
        for field, _ in cls._fields_:
            lines.append(f'    printf("{name} {field} %zu\\n", offsetof({name}, {field}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    layout = {}
    for line in out.splitlines():
        struct, key, value = line.split()
        layout.setdefault(struct, {})[key] = int(value)
    return layout


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc is needed to read the header's layout")
def test_ctypes_structs_match_the_header(tmp_path):
    layout = _c_layout(tmp_path)
    for name, cls in STRUCTS.items():
        c = layout[name]
        assert C.sizeof(cls) == c["size"], (name, C.sizeof(cls), c["size"])
        for field, _ in cls._fields_:
            assert getattr(cls, field).offset == c[field], (name, field, getattr(cls, field).offset, c[field])
