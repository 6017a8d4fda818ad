"""Record the order in which nvcc evaluates the draws of the reference sampler's 3-vector draw
(Sampler::next_3d, sampler.cuh:80-82) and of a two-argument call whose arguments each draw
(the shape of environment.cuh:245-250). Runs oracle/_ref/libref_probe.so (built by
oracle/Makefile from the reference header) on cuda:0 and prints JSON; the result is committed
as tests/golden/draw_order.json."""
import ctypes
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_probe.so"))
out = (ctypes.c_float * 10)()
rc = lib.ref_probe_draw_order(out)
if rc != 0:
    sys.exit(f"probe failed: {rc}")
v = list(out)
seq = v[3:6]
res = {"next_3d": v[0:3], "sequential": seq, "two_args": v[6:8], "two_args_sequential": v[8:10]}
res["next_3d_order"] = "first_component_first" if v[0:3] == seq else (
    "last_component_first" if v[0:3] == seq[::-1] else "other")
res["two_args_order"] = "first_argument_first" if v[6:8] == v[8:10] else "other"
print(json.dumps(res))
