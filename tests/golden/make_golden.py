"""Generate the golden fixtures of tests/golden (run in a checkout that has the reference).

  sampler_kat.json   PCG32 streams printed by oracle/_ref/sampler_kat, a host build of the
                     reference's own sampler (threedgptir_tracer/include/3dgptir/kernels/cuda/sampler.cuh)
  alias_tables.npz   environment importance tables from the reference's own
                     threedgrut/model/aliastable.py on seeded environments
  oracle_small.npz   FP64 oracle render of a tiny seeded scene (pins the oracle against regressions)

Usage: python tests/golden/make_golden.py [--reference /root/reference]
"""
import argparse
import importlib.util
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def sampler_kat(reference):
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={reference}"], check=True)
    out = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "sampler_kat")], check=True, capture_output=True, text=True)
    data = json.loads(out.stdout)
    with open(os.path.join(HERE, "sampler_kat.json"), "w") as f:
        json.dump(data, f, indent=1)


ALIAS_CASES = {"eq64x128": (64, 128, "2d", 3), "eq256x512": (256, 512, "2d", 5), "eq40x70": (40, 70, "2d", 6),
               "cube16": (96, 16, "cube", 4)}


def alias_case_env(name):
    """The seeded environment of an alias-table case (regenerated by the tests)."""
    from ptir_b200 import synthetic

    h, w, kind, seed = ALIAS_CASES[name]
    env = synthetic.make_environment(h, w, seed=seed)
    if name == "eq40x70":  # some dark and non-finite texels
        env[3:7, 10:20, :3] = 0.0
        env[0, 0, 0] = float("nan")
    return env, kind


def alias_tables(reference):
    import torch

    path = os.path.join(reference, "threedgrut", "model", "aliastable.py")
    spec = importlib.util.spec_from_file_location("ref_aliastable", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    arrays = {}
    for name in ALIAS_CASES:
        env, kind = alias_case_env(name)
        t = mod.build_environment_alias_table(env, environment_type=kind)
        arrays[f"{name}_prob"] = t.prob.numpy()
        arrays[f"{name}_alias"] = t.alias.numpy()
        arrays[f"{name}_pdf"] = t.pdf.numpy()
        arrays[f"{name}_hw"] = np.array([t.height, t.width])
    np.savez_compressed(os.path.join(HERE, "alias_tables.npz"), **arrays)


def oracle_small():
    from oracle import oracle as O
    from tests.scenes import small_scene

    s = small_scene(n=600, w=20, h=16, spp=2, max_bounces=3, env_hw=(16, 32), seed=5)
    out, vis, st = O.trace(O.OracleConfig(), s, "f64", threads=1)
    rng = np.random.default_rng(3)
    zhw = s["ray_ori"].shape[:3]
    grads = dict(pbr=rng.standard_normal(zhw + (3,)).astype(np.float32),
                 light=rng.standard_normal(zhw + (3,)).astype(np.float32),
                 material=rng.standard_normal(zhw + (5,)).astype(np.float32))
    mg, eg, _ = O.trace_bwd(O.OracleConfig(), s, out, grads, "f64", threads=1)
    np.savez_compressed(os.path.join(HERE, "oracle_small.npz"), visibility=vis, material_grad=mg, env_grad=eg,
                        segments=np.array([st.segments]), **{f"out_{k}": v for k, v in out.items()},
                        **{f"grad_{k}": v for k, v in grads.items()})


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    a = ap.parse_args()
    sampler_kat(a.reference)
    alias_tables(a.reference)
    oracle_small()
    print("golden fixtures written to", HERE)
