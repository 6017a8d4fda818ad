"""The tracer's per-ray device functions against the reference's own: both evaluate the cases of
tests/golden/device_kat.npz on a B200 (the reference's processHit, intersectInstanceParticle, BRDF
sample / eval / gradients, environment lookup / gradient scatter / alias sampling, light sampling
and pdf, compiled from its headers with its NVRTC options by tests/golden/make_device_golden.py),
the tracer's through oracle/libptir_kat.so, built from ptir_b200/csrc with the library's flags.

Both compute in float32 with fast math, so they agree to a few float32 ulps, widened where the
function loses bits in float (the BRDF at low roughness: tests/device_kat.py case_rtol); each
check bounds the share of cases outside the tolerance. The finite-difference outputs (over eps =
1e-3) are compared as vectors.
"""
import numpy as np
import pytest

from tests.device_kat import CASES, FD_COLUMNS, PtirKat, case_rtol, close, fd_report, load, value_columns

pytestmark = pytest.mark.gpu

ATOL, RTOL = 1e-6, 1e-5
MIN_SHARE = {"process_hit": 0.999, "intersect": 0.9995, "brdf_sample": 0.999, "brdf_eval": 0.999, "brdf_grads": 0.999,
             "env_lookup": 0.999, "env_bwd": 0.999, "env_sample": 0.9995, "light_sample": 0.999, "light_pdf": 0.999}


@pytest.mark.parametrize("entry,key,cols,scene", CASES, ids=[c[1] for c in CASES])
def test_device_function_matches_the_reference(cuda_device, entry, key, cols, scene):
    g = load()
    x, ref = g[f"{key}_in"], g[f"{key}_out"][:, :cols]
    out, eg = PtirKat().run(entry, g, scene, x, cols)
    vc = value_columns(entry, cols)
    ok = close(out[:, vc], ref[:, vc], ATOL, case_rtol(entry, x, RTOL))
    exact = np.all(out[:, :cols] == ref, axis=1).mean()
    print(f"{key}: {ok.mean():.5f} of {len(ok)} cases within {ATOL} + {RTOL} |ref|, {exact:.5f} bit-identical")
    assert ok.mean() >= MIN_SHARE[entry], (key, ok.mean())
    if entry in FD_COLUMNS:
        fd = FD_COLUMNS[entry]
        rep = fd_report(out[:, fd], ref[:, fd])
        print(f"{key} finite differences: {rep}")
        assert rep["rel_l2"] <= 1e-3 and rep["cos"] >= 0.99999 and rep["share"] >= 0.99, (key, rep)
    if entry in ("process_hit", "intersect"):
        assert (out[:, 0] == ref[:, 0]).mean() >= 0.9995
    if entry == "light_sample":
        assert (out[:, 8] == ref[:, 8]).mean() >= 0.9995
    if entry == "env_bwd":
        ref_g = g[f"{key}_grad"][..., :3].astype(np.float64)
        rel = np.linalg.norm(eg[..., :3] - ref_g) / np.linalg.norm(ref_g)
        assert rel <= 1e-5, rel
