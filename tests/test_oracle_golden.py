"""The oracle and the host-side table builder against golden vectors of the reference."""
import json
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from ptir_b200 import envmap
from tests.golden.make_golden import ALIAS_CASES, alias_case_env
from tests.scenes import small_scene

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_sampler_matches_reference_kat():
    """PCG32 streams of the oracle equal the reference sampler's own host build."""
    with open(os.path.join(GOLDEN, "sampler_kat.json")) as f:
        kat = json.load(f)
    assert len(kat["cases"]) >= 8
    for c in kat["cases"]:
        x, y, z, fr = c["launch"]
        assert O.launch_seed(x, y, z, fr) == c["seed"]
        assert O.sampler_stream(x, y, z, fr, 16).tolist() == c["u32"]
        u = O.sampler_stream(x, y, z, fr, 8)
        ref_1d = np.array(c["next_1d"], np.float32)
        ours = (u & 0xFFFFFF).astype(np.float32) * np.float32(1.0 / 16777216.0)
        assert np.array_equal(ours, ref_1d)


@pytest.mark.parametrize("name", list(ALIAS_CASES))
def test_alias_table_matches_reference(name):
    """envmap.build reproduces threedgrut/model/aliastable.py bit for bit."""
    g = np.load(os.path.join(GOLDEN, "alias_tables.npz"))
    env, kind = alias_case_env(name)
    t = envmap.build(env, cube=(kind == "cube"))
    assert [t["height"], t["width"]] == g[f"{name}_hw"].tolist()
    assert np.array_equal(t["prob"].numpy(), g[f"{name}_prob"])
    assert np.array_equal(t["alias"].numpy(), g[f"{name}_alias"])
    assert np.array_equal(t["pdf"].numpy(), g[f"{name}_pdf"])
    packed = envmap.pack(t)
    assert packed.shape == (3, t["height"], t["width"]) and packed.dtype == torch.float32


def test_alias_table_samples_its_pdf():
    """Walker sampling from the table reproduces the cell probabilities (table self-consistency)."""
    env, _ = alias_case_env("eq64x128")
    t = envmap.build(env)
    prob, alias = t["prob"].numpy().astype(np.float64), t["alias"].numpy()
    n = prob.size
    implied = prob / n
    np.add.at(implied, alias, (1.0 - prob) / n)
    from ptir_b200.envmap import _solid_angles_equirect

    sa = _solid_angles_equirect(t["height"], t["width"]).numpy().reshape(-1).astype(np.float64)
    target = t["pdf"].numpy().astype(np.float64) * sa
    assert np.allclose(implied, target / target.sum(), rtol=1e-4, atol=1e-9)


def test_oracle_regression_fixture():
    """The FP64 oracle still produces the committed render and gradients of a tiny scene."""
    g = np.load(os.path.join(GOLDEN, "oracle_small.npz"))
    s = small_scene(n=600, w=20, h=16, spp=2, max_bounces=3, env_hw=(16, 32), seed=5)
    out, vis, st = O.trace(O.OracleConfig(), s, "f64", threads=1)
    for k in O.FWD_KEYS:
        assert np.array_equal(out[k], g[f"out_{k}"]), k
    assert np.array_equal(vis, g["visibility"])
    assert st.segments == int(g["segments"][0])
    grads = {k: g[f"grad_{k}"] for k in ("pbr", "light", "material")}
    mg, eg, _ = O.trace_bwd(O.OracleConfig(), s, out, grads, "f64", threads=1)
    assert np.allclose(mg, g["material_grad"], rtol=1e-12, atol=1e-15)
    assert np.allclose(eg, g["env_grad"], rtol=1e-12, atol=1e-15)


def test_draw_order_matches_nvcc():
    """The oracle (and the kernels) take the draws of a 3-vector and of the alias sampler's
    (u, v) jitter first-argument-first, the order nvcc gives the reference's code
    (tests/golden/draw_order.json, recorded by tests/golden/probe_draw_order.py on a B200)."""
    with open(os.path.join(GOLDEN, "draw_order.json")) as f:
        d = json.load(f)
    assert d["next_3d_order"] == "first_component_first"
    assert d["two_args_order"] == "first_argument_first"
    assert O.OracleConfig().draw_order == 0
