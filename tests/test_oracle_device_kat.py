"""The oracle's restatement of the reference's per-ray device functions, pinned to the reference
itself: tests/golden/device_kat.npz holds the outputs of the reference's own processHit,
intersectInstanceParticle, BRDF sample / eval / gradients, environment lookup / gradient scatter /
alias sampling and light sampling / pdf, compiled from its headers with its NVRTC options and run
on a B200 (tests/golden/make_device_golden.py). The oracle evaluates the same cases in FP64.

The reference computes in float32 with fast math. Values agree to float32 precision, widened where
the function itself loses bits in float: the BRDF functions at low roughness, where the GGX terms
cancel (tests/device_kat.py: case_rtol), and a branch taken at a threshold, which the share bounds
cover. The two outputs that are finite differences over eps = 1e-3 of float evaluations (the
sampled direction's roughness derivative and the environment lookup's direction gradient) carry
that rounding times 1 / eps and are compared as vectors. CPU only.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.device_kat import CASES, FD_COLUMNS, case_rtol, close, fd_report, load, oracle_scene, value_columns

ATOL, RTOL = 1e-5, 1e-4
# share of cases whose value columns all agree within ATOL + case_rtol |ref|, per function
MIN_SHARE = {"process_hit": 0.999, "intersect": 0.999, "brdf_sample": 0.999, "brdf_eval": 0.999, "brdf_grads": 0.995,
             "env_lookup": 0.999, "env_bwd": 0.999, "env_sample": 0.999, "light_sample": 0.999, "light_pdf": 0.998}


@pytest.mark.parametrize("entry,key,cols,scene", CASES, ids=[c[1] for c in CASES])
def test_oracle_matches_the_reference_function(entry, key, cols, scene):
    g = load()
    x, ref = g[f"{key}_in"], g[f"{key}_out"][:, :cols]
    out, eg = O.kat(O.OracleConfig(), oracle_scene(g, scene), entry, x)
    vc = value_columns(entry, cols)
    ok = close(out[:, vc], ref[:, vc], ATOL, case_rtol(entry, x, RTOL))
    print(f"{key}: {ok.mean():.5f} of {len(ok)} cases within {ATOL} + {RTOL} |ref| (conditioning-widened)")
    assert ok.mean() >= MIN_SHARE[entry], (key, ok.mean())
    if entry in FD_COLUMNS:
        fd = FD_COLUMNS[entry]
        rep = fd_report(out[:, fd], ref[:, fd])
        print(f"{key} finite differences: {rep}")
        assert rep["rel_l2"] <= 1e-2 and rep["cos"] >= 0.9999 and rep["share"] >= 0.95, (key, rep)
    if entry in ("process_hit", "intersect"):
        assert (out[:, 0] == ref[:, 0]).mean() >= 0.999  # accepted / hit or not
    if entry == "light_sample":
        assert (out[:, 8] == ref[:, 8]).mean() >= 0.999  # the light type sampled
    if entry == "env_bwd":
        ref_g = g[f"{key}_grad"][..., :3].astype(np.float64)
        rel = np.linalg.norm(eg[..., :3] - ref_g) / np.linalg.norm(ref_g)
        assert rel <= 1e-4, rel
