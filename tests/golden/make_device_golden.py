"""Generate tests/golden/device_kat.npz: known-answer vectors of the reference's own device
functions, evaluated on a GPU by kernels compiled from the reference's headers with its NVRTC
options (oracle/ref_device_kat.cu, compiled by oracle/ref_kat.py to oracle/_ref/ref_device_kat.cubin
where the reference checkout is present).

    python tests/golden/make_device_golden.py OUT.npz        # on a machine with a GPU and the cubin

Functions pinned (the reference's file:line): processHit (gaussianParticles.cuh:343-440),
intersectInstanceParticle (gaussianParticles.cuh:484-500), sample_fast_brdf_throughput,
eval_fast_brdf_light_sample and sample_fast_brdf_throughput_with_grads (material.cuh:230-286,
448-492, 343-425), getBackgroundColor / environmentAliasPdf / getBackgroundColorBwd with the
direction gradient / sampleEnvironmentAliasDirection (environment.cuh:361-369, 303-328, 456-473,
421-445, 227-255) on an equirect and a cube map, sampleLight and lightSamplerPdf
(lightSampler.cuh:359-406) over point, sphere and mesh lights and the environment. Inputs are seeded;
every case's inputs and outputs are stored.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

N_CASES = 4096


def _unit(rng, n):
    v = rng.standard_normal((n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def particles(seed=5, n=64):
    from ptir_b200 import synthetic

    f = synthetic.make_field(n, seed=seed, scale_range=(0.05, 0.3), sh_full=True)
    return dict(density=synthetic.density_tensor(f).numpy(), material=synthetic.material_tensor(f).numpy(),
                sph=f["sph"].numpy(), shading_normal=f["snrm"].numpy())


def hit_cases(P, rng, n=N_CASES):
    """Rays from 2.5 away toward points scattered around random Gaussians (inside and outside their
    supports), with a random transmittance before the hit: o.xyz d.xyz id T."""
    m = P["density"].shape[0]
    ids = rng.integers(0, m, n)
    pos = P["density"][ids, 0:3].astype(np.float64)
    scl = P["density"][ids, 8:11].astype(np.float64)
    o = pos + _unit(rng, n) * 2.5
    target = pos + rng.standard_normal((n, 3)) * scl * rng.uniform(0.2, 3.0, (n, 1))
    d = target - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([o, d, ids[:, None], rng.uniform(0.05, 1.0, (n, 1))], 1).astype(np.float32)


def intersect_cases(rng, n=N_CASES):
    o = rng.uniform(-3.0, 3.0, (n, 3))
    d = rng.standard_normal((n, 3)) * rng.uniform(0.2, 3.0, (n, 1))
    tmin = rng.uniform(-1.0, 0.5, (n, 1))
    tmax = tmin + rng.uniform(0.1, 10.0, (n, 1))
    return np.concatenate([o, d, tmin, tmax], 1).astype(np.float32)


def brdf_cases(rng, n=N_CASES, light=False):
    """wo.xyz, normal.xyz, albedo.xyz, metallic, roughness, then rand.xyz (or a light direction),
    padded to 16 floats per case."""
    nrm = _unit(rng, n)
    wo = _unit(rng, n)
    flip = (np.sum(wo * nrm, 1) < 0) & (rng.random(n) < 0.85)
    wo[flip] *= -1.0
    rough = np.where(rng.random(n) < 0.1, rng.uniform(0.0, 0.05, n), rng.uniform(0.05, 1.0, n))
    if light:
        last = _unit(rng, n)
        fl = (np.sum(last * nrm, 1) < 0) & (rng.random(n) < 0.75)
        last[fl] *= -1.0
    else:
        last = rng.random((n, 3))
    return np.concatenate([wo, nrm, rng.random((n, 3)), rng.random((n, 1)), rough[:, None], last, np.zeros((n, 2))],
                          1).astype(np.float32)


def dir_cases(rng, n=N_CASES):
    axes = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], np.float64)
    return np.concatenate([axes, _unit(rng, n - 6)], 0).astype(np.float32)


def seed_cases(rng, n=N_CASES):
    return np.stack([rng.integers(0, 2048, n), rng.integers(0, 2048, n), rng.integers(0, 16, n),
                     rng.integers(0, 8, n)], 1).astype(np.float32)


def environments():
    """(name, env [h,w,4], alias [3,ah,aw]) for a 32x64 equirect map (its table area-resized to the
    reference's 64x128) and a 16x16-face cube map."""
    from ptir_b200 import envmap, synthetic

    out = []
    for name, (h, w), cube, seed in (("equirect", (32, 64), False, 5), ("cube", (96, 16), True, 6)):
        e = synthetic.make_environment(h, w, seed=seed)
        out.append((name, e.numpy(), envmap.pack(envmap.build(e, cube=cube)).numpy()))
    return out


def main(path):
    import torch

    from oracle.ref_kat import RefKat
    from ptir_b200.lights import light_buffers
    from tests.golden.make_golden import light_case

    kat = RefKat()
    rng = np.random.default_rng(2024)
    res = {}
    P = particles()
    res.update({f"particles_{k}": v for k, v in P.items()})
    dev = {k: torch.from_numpy(v).cuda() for k, v in P.items()}
    import ctypes as C

    x = hit_cases(P, rng)
    res["process_hit_in"] = x
    res["process_hit_out"] = kat.run("ref_process_hit", x, 18, extra=(
        (dev["density"].data_ptr(), C.c_void_p), (dev["material"].data_ptr(), C.c_void_p),
        (dev["sph"].data_ptr(), C.c_void_p), (dev["shading_normal"].data_ptr(), C.c_void_p),
        (0.0113, C.c_float), (1.0 / 255.0, C.c_float), (3, C.c_int)))
    x = intersect_cases(rng)
    res["intersect_in"], res["intersect_out"] = x, kat.run("ref_intersect", x, 2)
    for name, cols, light in (("brdf_sample", 7, False), ("brdf_eval", 4, True), ("brdf_grads", 19, False)):
        x = brdf_cases(rng, light=light)
        res[f"{name}_in"], res[f"{name}_out"] = x, kat.run(f"ref_{name}", x, cols)
    for ename, env, alias in environments():
        e_t, a_t = torch.from_numpy(env).cuda(), torch.from_numpy(alias).cuda()
        kat.set_scene(e_t, a_t)
        res[f"env_{ename}"], res[f"alias_{ename}"] = env, alias
        x = dir_cases(rng)
        res[f"env_lookup_{ename}_in"], res[f"env_lookup_{ename}_out"] = x, kat.run("ref_env_lookup", x, 4)
        xb = np.concatenate([dir_cases(rng, 2048), rng.standard_normal((2048, 3)).astype(np.float32)], 1)
        grad = torch.zeros(env.shape, dtype=torch.float32, device="cuda")
        res[f"env_bwd_{ename}_in"] = xb
        res[f"env_bwd_{ename}_out"] = kat.run("ref_env_bwd", xb, 6, extra=(
            (grad.data_ptr(), C.c_void_p), (int(env.shape[0]), C.c_int), (int(env.shape[1]), C.c_int)))
        res[f"env_bwd_{ename}_grad"] = grad.cpu().numpy()
        x = seed_cases(rng)
        res[f"env_sample_{ename}_in"], res[f"env_sample_{ename}_out"] = x, kat.run("ref_env_sample", x, 4)
    # lights: the mixed case (point, sphere, mesh lights and the environment in the top-level table)
    lights, env_l, etype = light_case("mixed")
    from ptir_b200 import envmap

    lb = light_buffers(lights, environment=env_l, environment_type=etype)
    tables = [t.contiguous().cuda() for t in lb.tensors()]
    alias_l = envmap.pack(envmap.build(env_l)).numpy()
    kat.set_scene(env_l.cuda(), torch.from_numpy(alias_l).cuda(), tables)
    for k, t in zip(("lights", "light_alias_table", "mesh_light_vertices", "mesh_light_triangles", "mesh_lights",
                     "mesh_light_triangle_alias_table"), lb.tensors()):
        res[f"lightscene_{k}"] = t.numpy()
    res["lightscene_env"], res["lightscene_alias"] = env_l.numpy(), alias_l
    pos = rng.uniform(-1.0, 1.0, (N_CASES, 3)).astype(np.float32)
    x = np.concatenate([pos, seed_cases(rng)[:, :3], rng.integers(0, 8, (N_CASES, 1))], 1).astype(np.float32)
    res["light_sample_in"], res["light_sample_out"] = x, kat.run("ref_light_sample", x, 10)
    # pdf directions: half toward points of the lights' bounding region, half random
    toward = rng.uniform([-1.2, 0.5, -0.6], [1.0, 2.1, 1.5], (N_CASES, 3)) - pos
    toward /= np.linalg.norm(toward, axis=1, keepdims=True)
    dirs = np.where(rng.random((N_CASES, 1)) < 0.5, toward, _unit(rng, N_CASES))
    x = np.concatenate([pos, dirs], 1).astype(np.float32)
    res["light_pdf_in"], res["light_pdf_out"] = x, kat.run("ref_light_pdf", x, 1)
    np.savez_compressed(path, **res)
    print(f"wrote {path}: {len(res)} arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden", "device_kat.npz"))
