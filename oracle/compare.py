"""ORACLE — TEST INFRASTRUCTURE ONLY.

Comparison of a tracer's outputs with the oracle's, split by path decisions. Only the tests and
the accuracy leg of ``bench.py`` use this module.

Both the GPU tracer and the oracle write a per-path decision signature (an FNV-1a hash of every
discrete branch a path takes: accepted-hit counts, interaction and escape flags, NEE shadow ray
cast and occluded, continuation after each BRDF sample). Paths with equal signatures took the
same branches, so their outputs differ only by rounding; paths with different signatures took
another branch somewhere (a hit accepted at the response threshold, a stochastic draw against a
transmittance or alpha, a grazing candidate kept or not) and differ by whole contributions.
"""
from __future__ import annotations

import numpy as np

TOL_ABS = 1e-3
TOL_REL = 1e-3


def rel_cos(a, b):
    """(relative L2 distance of a from b, cosine of a and b) over all elements, in FP64."""
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    nb = max(float(np.linalg.norm(b)), 1e-30)
    na = max(float(np.linalg.norm(a)), 1e-30)
    return float(np.linalg.norm(a - b) / nb), float(a @ b / (na * nb))


def within(x, ref, tol_abs=TOL_ABS, tol_rel=TOL_REL):
    """Per sample: every channel within tol_abs + tol_rel * |ref|."""
    x, ref = np.asarray(x, np.float64), np.asarray(ref, np.float64)
    return np.all(np.abs(x - ref) <= tol_abs + tol_rel * np.abs(ref), axis=-1)


def image_report(x, ref, sig_x, sig_ref) -> dict:
    """Error of image x ([...,C]) against ref, over all paths and over the paths whose signatures
    agree."""
    x, ref = np.asarray(x, np.float64), np.asarray(ref, np.float64)
    agree = np.asarray(sig_x) == np.asarray(sig_ref)
    err = np.abs(x - ref)
    ok = within(x, ref)
    out = {"paths": int(agree.size), "flipped_paths": int((~agree).sum()),
           "flipped_fraction": float((~agree).mean()),
           "all": {"within_tol": float(ok.mean()), "max_abs": float(err.max(initial=0.0)),
                   "mean_abs": float(err.mean()) if err.size else 0.0, "rel_l2": rel_cos(x, ref)[0]}}
    if agree.any():
        ea = err[agree]
        out["agree"] = {"within_tol": float(ok[agree].mean()), "max_abs": float(ea.max(initial=0.0)),
                        "max_rel": float((ea / (np.abs(ref[agree]) + TOL_ABS)).max(initial=0.0)),
                        "rel_l2": rel_cos(x[agree], ref[agree])[0]}
    return out


def grad_report(mat, env, mat_ref, env_ref) -> dict:
    """Relative L2 and cosine of the material (albedo + roughness columns) and environment (RGB)
    gradients against the reference's."""
    m_rel, m_cos = rel_cos(np.asarray(mat)[:, :4], np.asarray(mat_ref)[:, :4])
    out = {"material_rel_l2": m_rel, "material_cos": m_cos}
    if env is not None and env_ref is not None:
        e_rel, e_cos = rel_cos(np.asarray(env)[..., :3], np.asarray(env_ref)[..., :3])
        out.update(env_rel_l2=e_rel, env_cos=e_cos)
    return out


def masked_grad(g, sig_x, sig_ref):
    """The incoming per-sample gradient with the paths whose signatures differ set to zero: the
    adjoint over the paths on which both evaluations took the same branches."""
    agree = (np.asarray(sig_x) == np.asarray(sig_ref))[..., None]
    return np.where(agree, g, 0.0).astype(np.float32)
