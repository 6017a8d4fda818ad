"""Generate tests/golden/render_host.npz: the reference's own tracer.py
(threedgptir_tracer/tracer.py), driven with the stand-in plugin of tests/render_host.py, on the
cases listed there.

    PTIR_REFERENCE_ROOT=<reference checkout> python tests/golden/make_render_golden.py [OUT.npz]

The reference module is loaded from its file with the threedgrut modules it imports replaced:
``threedgrut.datasets.protocols`` (only the ``Batch`` type annotation is used), the rich logger and
the CUDA timer by small stand-ins, while the a-trous ``Filter`` (threedgrut/model/filters.py) and
the mask ``post_processing`` (threedgrut/model/ptir_helper.py) are the reference's own files, loaded
the same way. Its ``_threedgptir_plugin`` global is set to a namespace holding
``RecordingPlugin``, which ``load_threedgptir_plugin`` (tracer.py:122-131) then keeps: the swap of
the native plugin that the drop-in relies on.
"""
from __future__ import annotations

import importlib.util
import logging
import os
import sys
import types

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
REF = os.environ.get("PTIR_REFERENCE_ROOT", "/root/reference")


def _module(name, **attrs):
    m = types.ModuleType(name)
    m.__dict__.update(attrs)
    sys.modules[name] = m
    return m


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    m = importlib.util.module_from_spec(spec)
    sys.modules[name] = m
    spec.loader.exec_module(m)
    return m


def load_reference_tracer():
    class _Logger:
        def __getattr__(self, _):
            return lambda *a, **k: None

    class _CudaTimer:  # only built when render.enable_kernel_timings is set
        pass

    _module("threedgrut", __path__=[])
    _module("threedgrut.datasets", __path__=[])
    _module("threedgrut.datasets.protocols", Batch=object)
    _module("threedgrut.utils", __path__=[])
    _module("threedgrut.utils.logger", logger=_Logger())
    _module("threedgrut.utils.timer", CudaTimer=_CudaTimer)
    _module("threedgrut.utils.normal", normal_mae=None)
    _module("threedgrut.model", __path__=[])
    _load("threedgrut.model.filters", os.path.join(REF, "threedgrut", "model", "filters.py"))
    _load("threedgrut.model.ptir_helper", os.path.join(REF, "threedgrut", "model", "ptir_helper.py"))
    _module("threedgptir_tracer", __path__=[])
    return _load("threedgptir_tracer.tracer", os.path.join(REF, "threedgptir_tracer", "tracer.py"))


def main(path):
    import torch

    from tests import render_host as H

    logging.disable(logging.WARNING)
    ref = load_reference_tracer()
    ref._threedgptir_plugin = types.SimpleNamespace(OptixTracer=H.RecordingPlugin)
    res = {}
    for case in H.CASES:
        for k, v in H.run_case(ref.Tracer, case).items():
            res[f"{case[0]}__{k}"] = v.numpy()
    for k, v in H.run_build_sequence(ref.Tracer).items():
        res[f"build__{k}"] = v.numpy()
    res["ctor_args"] = np.array([str(a) for a in H.constructor_args(ref.Tracer)])
    res["torch_version"] = np.array(torch.__version__)
    np.savez_compressed(path, **res)
    print(f"wrote {path}: {len(res)} arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden", "render_host.npz"))
