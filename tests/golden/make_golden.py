"""Generate the golden fixtures of tests/golden (run in a checkout that has the reference).

  sampler_kat.json   PCG32 streams printed by oracle/_ref/sampler_kat, a host build of the
                     reference's own sampler (threedgptir_tracer/include/3dgptir/kernels/cuda/sampler.cuh)
  alias_tables.npz   environment importance tables from the reference's own
                     threedgrut/model/aliastable.py on seeded environments
  oracle_small.npz   FP64 oracle render of a tiny seeded scene (pins the oracle against regressions)
  light_tables.npz   packed point / sphere / mesh light tables and top-level light alias tables
                     from the reference's own threedgrut/model/light.py (its image-loading import,
                     imageio, is absent here and unused by these functions, so it is stubbed)

Usage: python tests/golden/make_golden.py --reference REFERENCE_CHECKOUT   (or $PTIR_REFERENCE_ROOT)
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


def light_case(name):
    """Light descriptions and environment of a light-table case (regenerated by the tests)."""
    from ptir_b200 import synthetic

    quad = dict(type="mesh", vertices=[[-0.5, 2.0, -0.5], [0.5, 2.0, -0.5], [0.5, 2.0, 0.5], [-0.5, 2.0, 0.5]],
                triangles=[[0, 1, 2], [0, 2, 3]], radiance=(4.0, 3.5, 3.0), two_sided=False)
    strip = dict(type="mesh", vertices=[[1.0, -1.0, 0.0], [1.5, -1.0, 0.2], [1.2, -0.4, 0.1], [1.9, -0.5, 0.4],
                                        [1.2, -0.4, 0.1]],
                 triangles=[[0, 1, 2], [1, 3, 2], [2, 2, 4]], radiance=(0.5, 1.0, 2.0), two_sided=True)
    if name == "mixed":
        lights = [dict(type="point", position=(0.3, 1.5, -0.2), intensity=(2.0, 1.5, 1.0)),
                  dict(type="sphere", center=(-1.0, 1.2, 0.5), radius=0.25, radiance=(3.0, 3.0, 2.5)),
                  dict(type="point", position=(-0.4, -1.1, 0.9), intensity=(0.0, 0.0, 0.0)),
                  dict(type="sphere", center=(0.8, 0.9, 1.3), radius=0.1, radiance=(10.0, 2.0, 1.0), two_sided=True),
                  quad, strip]
        return lights, synthetic.make_environment(32, 64, seed=11), "2d"
    if name == "point_only":
        return [dict(type="point", position=(0.0, 2.0, 0.0), intensity=(5.0, 5.0, 5.0))], None, "2d"
    if name == "cube_sphere":
        return ([dict(type="sphere", center=(0.0, 0.0, 3.0), radius=0.5, radiance=(1.0, 0.5, 0.25))],
                synthetic.make_environment(48, 8, seed=12), "cube")
    raise KeyError(name)


LIGHT_CASES = ("mixed", "point_only", "cube_sphere")


def _reference_light_module(reference):
    import types

    for m in ("imageio", "imageio.plugins", "imageio.plugins.freeimage"):
        if m not in sys.modules:
            mod = types.ModuleType(m)
            mod.__path__ = []
            sys.modules[m] = mod
    sys.modules["imageio"].plugins = sys.modules["imageio.plugins"]
    sys.modules["imageio.plugins"].freeimage = sys.modules["imageio.plugins.freeimage"]
    sys.path.insert(0, reference)
    import threedgrut.model.light as L  # noqa: E402

    return L


def light_tables(reference):
    import torch

    L = _reference_light_module(reference)
    arrays = {}
    for name in LIGHT_CASES:
        lights, env, kind = light_case(name)
        analytic = [L.Light.from_dict(d) for d in lights if d["type"] != "mesh"]
        meshes = [L.Light.from_dict(d) for d in lights if d["type"] == "mesh"]
        packed = L.Light.pack_lights(analytic, dtype=torch.float32)
        pack = L.pack_mesh_lights(meshes, dtype=torch.float32)
        table = L.build_light_alias_table(environment=None if env is None else torch.as_tensor(env),
                                          environment_type=kind, lights=packed, mesh_powers=pack.powers)
        arrays[f"{name}_lights"] = packed.numpy()
        arrays[f"{name}_table"] = (np.zeros((5, 0), np.float32) if table is None else table.pack().numpy())
        arrays[f"{name}_mesh_vertices"] = pack.vertices.numpy()
        arrays[f"{name}_mesh_triangles"] = pack.triangles.numpy()
        arrays[f"{name}_mesh_lights"] = pack.params.numpy()
        arrays[f"{name}_mesh_tri_table"] = pack.triangle_alias_table.numpy()
        arrays[f"{name}_mesh_powers"] = pack.powers.numpy()
    np.savez_compressed(os.path.join(HERE, "light_tables.npz"), **arrays)


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
    ap.add_argument("--reference", default=os.environ.get("PTIR_REFERENCE_ROOT"),
                    help="the reference checkout (default: $PTIR_REFERENCE_ROOT)")
    a = ap.parse_args()
    sampler_kat(a.reference)
    alias_tables(a.reference)
    light_tables(a.reference)
    oracle_small()
    print("golden fixtures written to", HERE)
