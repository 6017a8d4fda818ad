"""Light tables and the oracle's light sampler, on the CPU.

* ptir_b200.lights builds the packed tables of the reference's threedgrut/model/light.py
  (Light.pack_lights, pack_mesh_lights, build_light_alias_table): they equal the tables the
  reference built for the same lights (tests/golden/light_tables.npz, made by
  tests/golden/make_golden.py).
* The oracle's light sampler (lightSampler.cuh:12-406, meshLight.cuh:11-101): point-light samples
  carry the selection pdf and I / d^2; a planar one-sided mesh light's sampling pdf equals the pdf
  its MIS evaluation gives the same direction; sphere samples on the near side do too (samples on
  the far side keep the area pdf of the point drawn, as in the reference, so their evaluated pdf
  is the near side's); light types are drawn in proportion to their selection pdfs; and the
  mesh-light estimate of irradiance matches quadrature of the area integral.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from ptir_b200 import lights as PL
from tests.golden.make_golden import LIGHT_CASES, light_case
from tests.scenes import small_scene, with_lights

GOLDEN = np.load("tests/golden/light_tables.npz")


@pytest.mark.parametrize("name", LIGHT_CASES)
def test_tables_match_reference(name):
    lights, env, kind = light_case(name)
    analytic = [d for d in lights if d["type"] != "mesh"]
    meshes = [d for d in lights if d["type"] == "mesh"]
    packed = PL.pack_lights(analytic)
    mesh = PL.pack_mesh_lights(meshes)
    table = PL.build_light_alias_table(None if env is None else torch.as_tensor(env), kind, packed, mesh.powers)
    ours = {"lights": packed, "table": table, "mesh_vertices": mesh.vertices, "mesh_triangles": mesh.triangles,
            "mesh_lights": mesh.params, "mesh_tri_table": mesh.triangle_alias_table, "mesh_powers": mesh.powers}
    for key, value in ours.items():
        ref = GOLDEN[f"{name}_{key}"]
        got = value.numpy()
        assert got.shape == ref.shape, (key, got.shape, ref.shape)
        assert got.dtype == ref.dtype, (key, got.dtype, ref.dtype)
        if key == "table":
            np.testing.assert_array_equal(got[1:4], ref[1:4])  # alias, type, index
            np.testing.assert_allclose(got[[0, 4]], ref[[0, 4]], rtol=1e-6, atol=1e-7)
        else:
            np.testing.assert_allclose(got, ref, rtol=1e-6, atol=1e-7, err_msg=key)


def test_empty_and_degenerate_tables():
    assert tuple(PL.build_light_alias_table().shape) == (5, 0)
    assert tuple(PL.pack_lights(None).shape) == (0, 9)
    dark = PL.pack_lights([dict(type="point", position=(0, 0, 0), intensity=(0, 0, 0))])
    assert tuple(PL.build_light_alias_table(lights=dark).shape) == (5, 0)
    flat = PL.pack_mesh_lights([dict(type="mesh", vertices=[[0, 0, 0], [1, 0, 0], [2, 0, 0]], triangles=[[0, 1, 2]])])
    assert flat.params.shape[0] == 0 and tuple(flat.triangle_alias_table.shape) == (3, 0)
    with pytest.raises(ValueError):
        PL.pack_lights([dict(type="sphere", radius=0.0)])
    with pytest.raises(NotImplementedError):
        PL.pack_lights([dict(type="spot")])


def _scene(lights, environment=False):
    return with_lights(small_scene(n=50, w=8, h=4), lights, environment=environment)


def test_point_light_samples():
    lights, _, _ = light_case("point_only")
    s = _scene(lights)
    rng = np.random.default_rng(0)
    pos = rng.uniform(-1, 1, (64, 3)).astype(np.float32)
    wi, Li, pdf, dist, kind, ev = O.light_samples(O.OracleConfig(), s, pos)
    p = np.array(lights[0]["position"], np.float64)
    to = p - pos.astype(np.float64)
    d = np.linalg.norm(to, axis=1)
    assert np.all(kind == 1) and np.all(pdf == 1.0)
    np.testing.assert_allclose(dist, d, rtol=1e-12)
    np.testing.assert_allclose(wi, to / d[:, None], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(Li, np.array(lights[0]["intensity"])[None, :] / (d * d)[:, None], rtol=1e-12)
    assert np.all(ev == 0.0)  # a delta light adds nothing to the MIS pdf


QUAD = dict(type="mesh", vertices=[[-0.5, 2.0, -0.5], [0.5, 2.0, -0.5], [0.5, 2.0, 0.5], [-0.5, 2.0, 0.5]],
            triangles=[[0, 1, 2], [0, 2, 3]], radiance=(4.0, 3.5, 3.0), two_sided=False)


def test_mesh_light_pdf_consistency_and_irradiance():
    s = _scene([QUAD])
    m = 40000
    p = np.array([0.1, 0.0, 0.2], np.float32)
    pos = np.tile(p, (m, 1))
    wi, Li, pdf, dist, kind, ev = O.light_samples(O.OracleConfig(), s, pos)
    assert np.all(kind == 3) and np.all(pdf > 0)
    np.testing.assert_allclose(ev, pdf, rtol=1e-9)
    # irradiance on a surface facing +y: Monte Carlo vs midpoint quadrature of the area integral
    est = float(np.mean(Li[:, 0] * np.maximum(wi[:, 1], 0.0) / pdf))
    g = (np.arange(800) + 0.5) / 800 - 0.5
    X, Z = np.meshgrid(g, g, indexing="ij")
    to = np.stack([X - p[0], np.full_like(X, 2.0 - p[1]), Z - p[2]], -1)
    d2 = np.sum(to * to, -1)
    cos_s = to[..., 1] / np.sqrt(d2)
    cos_l = cos_s  # light normal is -y
    ref = 4.0 * float(np.sum(cos_s * cos_l / d2)) / 800 ** 2
    assert abs(est - ref) <= 0.01 * ref, (est, ref)


def test_sphere_light_near_side_pdf():
    sphere = dict(type="sphere", center=(0.3, 1.8, -0.2), radius=0.4, radiance=(2.0, 2.0, 2.0))
    s = _scene([sphere])
    m = 4000
    pos = np.zeros((m, 3), np.float32)
    wi, Li, pdf, dist, kind, ev = O.light_samples(O.OracleConfig(), s, pos)
    c = s["lights"][0, 1:4].astype(np.float64)  # the float32 table values the sampler read
    r = float(s["lights"][0, 4])
    b = wi @ (-c)
    disc = b * b - (c @ c - r * r)
    t_near = -b - np.sqrt(np.maximum(disc, 0.0))
    near = np.abs(dist - t_near) <= 1e-9 * dist
    assert 0.3 < near.mean() < 0.6  # the cap seen from the origin is less than half the sphere
    well = near & (disc > 1e-7)  # grazing directions are ill-conditioned in the intersection
    np.testing.assert_allclose(ev[well], pdf[well], rtol=1e-6)
    assert np.all(ev[~near] > 0)


def test_light_types_drawn_by_selection_pdf():
    lights, _, _ = light_case("mixed")
    s = with_lights(small_scene(n=50, w=8, h=4), lights, environment=True)
    table = s["light_alias_table"]
    m = 20000
    pos = np.zeros((m, 3), np.float32)
    _, _, pdf, _, kind, _ = O.light_samples(O.OracleConfig(), s, pos)
    assert np.all(pdf > 0)
    for t in (0, 1, 2, 3):
        expect = float(table[4][table[2] == t].sum())
        got = float(np.mean(kind == t))
        sigma = np.sqrt(max(expect * (1 - expect), 1e-12) / m)
        assert abs(got - expect) <= 5 * sigma + 1e-9, (t, got, expect)
