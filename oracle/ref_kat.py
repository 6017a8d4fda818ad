"""ORACLE — TEST INFRASTRUCTURE ONLY.

Known-answer kernels compiled from the reference's own device headers (oracle/ref_device_kat.cu).

``compile_cubin(reference_root)`` compiles them here, with NVRTC and the reference's own options
(threedgptir_tracer/include/3dgptir/cuoptixMacros.h:69-71) and JIT defines
(src/optixTracer.cpp:240-272), to ``oracle/_ref/ref_device_kat.cubin`` (git-ignored; it travels to
the GPU box with the other built files). ``RefKat`` loads that cubin through the CUDA driver API
and runs its kernels on torch CUDA tensors. Only tests/golden/make_device_golden.py uses it, to
produce the fixtures tests/golden/device_kat.npz.
"""
from __future__ import annotations

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CUBIN = os.path.join(HERE, "_ref", "ref_device_kat.cubin")
SOURCE = os.path.join(HERE, "ref_device_kat.cu")

# the reference's NVRTC options (cuoptixMacros.h:69-71) for sm_100a instead of compute_75, without
# -rdc (one self-contained module), and the defines of its default tracer
# (optixTracer.cpp:240-272: degree-4 kernel, normals, hit counts, MIS, SH degree 3, instances,
# density clamping)
NVRTC_OPTIONS = ["-std=c++17", "-arch=sm_100a", "-use_fast_math", "--extra-device-vectorization", "-default-device",
                 "-D__OPTIX__", "-DPARTICLE_KERNEL_DEGREE=4", "-DENABLE_NORMALS", "-DENABLE_HIT_COUNTS",
                 "-DENABLE_MIS", "-DSPH_MAX_NUM_COEFFS=16", "-DPARTICLE_PRIMITIVE_CLAMPED=1"]


def _check(res, what):
    err = res[0]
    if int(err) != 0:
        raise RuntimeError(f"{what} failed: {err}")
    return res[1:] if len(res) > 2 else (res[1] if len(res) == 2 else None)


def compile_cubin(reference_root: str, out: str = CUBIN) -> str:
    """Compile oracle/ref_device_kat.cu against the reference checkout at `reference_root` (no GPU
    needed)."""
    from cuda.bindings import nvrtc

    inc = os.path.join(reference_root, "threedgptir_tracer", "include")
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    with open(SOURCE, "rb") as f:
        src = f.read()
    prog = _check(nvrtc.nvrtcCreateProgram(src, b"ref_device_kat.cu", 0, [], []), "nvrtcCreateProgram")
    opts = [o.encode() for o in NVRTC_OPTIONS + [f"-I{inc}", f"-I{os.path.join(HERE, 'ref_stub')}", f"-I{cuda_inc}"]]
    res = nvrtc.nvrtcCompileProgram(prog, len(opts), opts)
    size = _check(nvrtc.nvrtcGetProgramLogSize(prog), "log size")
    log = b" " * size
    nvrtc.nvrtcGetProgramLog(prog, log)
    if int(res[0]) != 0:
        raise RuntimeError("NVRTC compile of ref_device_kat.cu failed:\n" + log.decode(errors="replace"))
    n = _check(nvrtc.nvrtcGetCUBINSize(prog), "cubin size")
    cubin = b" " * n
    _check(nvrtc.nvrtcGetCUBIN(prog, cubin), "get cubin")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    with open(out, "wb") as f:
        f.write(cubin)
    return out


class RefKat:
    """The reference's known-answer kernels on the current CUDA context (torch's)."""

    def __init__(self, cubin: str = CUBIN):
        import torch
        from cuda.bindings import driver

        torch.zeros(1, device="cuda")  # the primary context, current on this thread
        self._drv = driver
        with open(cubin, "rb") as f:
            self._image = f.read()
        self._mod = _check(driver.cuModuleLoadData(self._image), "cuModuleLoadData")
        self._fn = {}

    def _func(self, name):
        if name not in self._fn:
            self._fn[name] = _check(self._drv.cuModuleGetFunction(self._mod, name.encode()), f"get {name}")
        return self._fn[name]

    def launch(self, name, n_threads, args):
        """Launch kernel `name` over n_threads threads; args: (value, ctypes type) pairs."""
        import ctypes as C

        import torch

        vals = tuple(a for a, _ in args)
        types = tuple(t for _, t in args)
        blocks = max(1, (n_threads + 127) // 128)
        torch.cuda.synchronize()
        _check(self._drv.cuLaunchKernel(self._func(name), blocks, 1, 1, 128, 1, 1, 0, 0, (vals, types), 0),
               f"launch {name}")
        torch.cuda.synchronize()
        del C

    # -- scene ------------------------------------------------------------------------------
    def set_scene(self, env, alias, lights=None):
        """env [eh, ew, 4], alias [3, ah, aw] CUDA float tensors (or None); lights: the six
        LightBuffers tensors (or None). Keeps references so the pointers stay valid."""
        import ctypes as C

        self._scene = (env, alias, lights)
        p = lambda t: 0 if t is None or t.numel() == 0 else t.data_ptr()  # noqa: E731
        eh, ew = (int(env.shape[0]), int(env.shape[1])) if env is not None else (0, 0)
        ah, aw = (int(alias.shape[1]), int(alias.shape[2])) if alias is not None else (0, 0)
        lt = lights or (None,) * 6
        cnt = lambda t, ax: 0 if t is None else int(t.shape[ax])  # noqa: E731
        V, I = C.c_void_p, C.c_int  # noqa: E741
        args = [(p(env), V), (eh, I), (ew, I), (p(alias), V), (ah, I), (aw, I),
                (p(lt[0]), V), (cnt(lt[0], 0), I), (p(lt[1]), V), (cnt(lt[1], 1), I), (p(lt[2]), V), (cnt(lt[2], 0), I),
                (p(lt[3]), V), (cnt(lt[3], 0), I), (p(lt[4]), V), (cnt(lt[4], 0), I), (p(lt[5]), V), (cnt(lt[5], 1), I)]
        self.launch("ref_set_scene", 1, args)

    def run(self, name, inputs: np.ndarray, out_cols: int, extra=()):
        """Kernel `name` on inputs [n, IN] (float32); returns outputs [n, out_cols] (numpy)."""
        import ctypes as C

        import torch

        x = torch.from_numpy(np.ascontiguousarray(inputs, np.float32)).cuda()
        n = x.shape[0]
        y = torch.zeros((n, out_cols), dtype=torch.float32, device="cuda")
        self.launch(name, n, [(n, C.c_int), (x.data_ptr(), C.c_void_p), (y.data_ptr(), C.c_void_p), *extra])
        return y.cpu().numpy()


if __name__ == "__main__":
    import sys

    print(compile_cubin(sys.argv[1]))
