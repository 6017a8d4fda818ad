"""``OptixTracer``: the native tracer object with the reference's pybind11 surface.

Same constructor arguments and the same ``trace`` / ``trace_bwd`` / ``build_bvh`` methods,
argument order, tensor layouts and return tuples as the reference class
(threedgptir_tracer/bindings.cpp:32-38, include/3dgptir/optixTracer.h:130-217), backed by
``libptir_b200.so`` through its C ABI instead of OptiX.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _native as N


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _f32(t: torch.Tensor, name: str) -> torch.Tensor:
    """Contiguous float32 CUDA view of `t`; other dtypes are rejected like the reference's getPtr
    (tensorBuffering.h:30-39)."""
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name}: expected a torch.Tensor")
    if t.dtype != torch.float32:
        raise TypeError(f"{name}: unsupported dtype {t.dtype} (float32 required)")
    if not t.is_cuda:
        raise ValueError(f"{name}: CUDA tensor required")
    return t.contiguous()


def _f32_strided(t: torch.Tensor, name: str) -> torch.Tensor:
    """A per-sample float32 CUDA tensor passed with its own strides, as the reference's
    PackedTensorAccessor32 reads it (tensorBuffering.h:41-45): no copy, whatever its layout."""
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name}: expected a torch.Tensor")
    if t.dtype != torch.float32:
        raise TypeError(f"{name}: unsupported dtype {t.dtype} (float32 required)")
    if not t.is_cuda:
        raise ValueError(f"{name}: CUDA tensor required")
    return t


def _strides4(t: torch.Tensor | None):
    """The element strides of a [Z,H,W,C] (or [1,1,T,C]) tensor for a `*_strides[4]` field (an
    absent tensor's are zeros, unused)."""
    s = (0, 0, 0, 0) if t is None else tuple(int(v) for v in t.stride())
    return (C.c_int64 * 4)(*s)


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _light_tables(lights, light_alias_table, mesh_light_vertices, mesh_light_triangles, mesh_lights,
                  mesh_light_triangle_alias_table) -> list:
    """The six LightBuffers tensors (threedgptir_tracer/tracer.py:40-119) as contiguous CUDA tensors,
    None where a table is absent or empty; shapes are checked as the kernels index them."""
    specs = ((lights, "lights", 9, None, torch.float32), (light_alias_table, "light_alias_table", None, 5, torch.float32),
             (mesh_light_vertices, "mesh_light_vertices", 3, None, torch.float32),
             (mesh_light_triangles, "mesh_light_triangles", 3, None, torch.int32),
             (mesh_lights, "mesh_lights", 8, None, torch.float32),
             (mesh_light_triangle_alias_table, "mesh_light_triangle_alias_table", None, 3, torch.float32))
    out = []
    for t, name, cols, rows, dtype in specs:
        if t is None or t.numel() == 0:
            out.append(None)
            continue
        if t.dim() != 2 or (cols is not None and t.shape[1] != cols) or (rows is not None and t.shape[0] != rows):
            shape = f"[{rows}, K]" if rows is not None else f"[K, {cols}]"
            raise ValueError(f"{name} must be {shape}, got {tuple(t.shape)}")
        if t.dtype != dtype:
            raise TypeError(f"{name}: unsupported dtype {t.dtype} ({dtype} required)")
        if not t.is_cuda:
            raise ValueError(f"{name}: CUDA tensor required")
        out.append(t.contiguous())
    return out


def split_views(flat: torch.Tensor, views) -> list:
    """Per-view [Z,H,W,C...] views of a flat per-sample tensor [T,C...] of trace_views()."""
    out, start = [], 0
    for _, _, z, h, w in views:
        n = int(z) * int(h) * int(w)
        out.append(flat[start:start + n].reshape(int(z), int(h), int(w), *flat.shape[1:]))
        start += n
    return out


class OptixTracer:
    """Drop-in for ``libthreedgptir_cc.OptixTracer``.

    The keyword arguments after the reference's own set the B200 launch shape (no counterpart in
    the reference): ``schedule`` ("wavefront" or "megakernel"), and for the wavefront
    ``chunk_tiles`` (8x4 pixel tiles per chunk), ``kbuffer`` (8, 16 or 32 candidates per
    traversal; 16 and 32 composite in the reference's rounds of 16, a 32-entry traversal standing
    for two rounds when its second half is the next round's candidates), ``refill_lanes`` (waiting lanes before an intersection warp refills, 1..32) and
    ``block_size`` (64, 128 or 256); 0 keeps the default. ``collect_timings`` records CUDA events
    around every kernel launch for ``stage_times()``; ``sort_rays`` intersects bounce rays in
    (direction octant, origin cell, direction cell) order (the results do not change); ``exact_replay`` lets the
    backward re-traversals include each segment's last composited Gaussian, which the
    reference's float epsilon leaves out; ``compensated_grads``
    accumulates the gradient atomics as Kahan pairs (off: plain float atomics, as the
    reference). ``storage`` ("fp32",
    "bf16" or "fp16") sets how the tracer holds the Gaussians' attributes: in 16-bit storage
    geometry, material, shading normals and SH are rounded once per call (and by ``build_bvh``)
    and widened on load, all arithmetic staying FP32. ``warp_aggregate`` sums the gradient terms
    that lanes of a warp add to the same Gaussian or texel before the atomics (off: one atomic
    per lane and term). ``shadow_kbuffer`` (8, 16 or 32; 0 = 16) sets the k-buffer of the NEE
    shadow rays apart from ``kbuffer``. ``exact_candidates`` makes every traversal return exactly
    the K nearest candidates (off: subtrees are culled by their box entry as the reference's
    traversal culls them, which keeps a grazing Gaussian or not depending on the order), so that
    the results depend on neither the traversal order nor ``kbuffer``. ``resume_rounds`` (k-buffer 8
    or 16) picks the traversals whose next k-buffer round starts from what the previous round set
    aside against its K-th distance instead of from the root: 0 the backward replay's (default), 1
    none, 2 the replay's and the intersection stage's. ``bvh_builder`` picks the hierarchy of a
    rebuild: "morton" (the Karras hierarchy over the sorted keys), "ploc" (agglomerative clustering
    by surface area over the same sorted leaves: a better tree and a slower build, which
    synchronises the stream, so a rebuild cannot be captured in a CUDA graph) or "default" (PLOC)."""

    def __init__(
        self,
        path: str,
        cuda_path: str,
        pipeline: str,
        backward_pipeline: str,
        primitive: str,
        particle_kernel_degree: float,
        particle_kernel_min_response: float,
        particle_kernel_density_clamping: bool,
        particle_radiance_sph_degree: int,
        enable_normals: bool,
        enable_hit_counts: bool,
        enable_mis: bool,
        enable_metallic: bool,
        visualize_lights: bool = False,
        collect_counters: bool = True,
        schedule: str = "wavefront",
        chunk_tiles: int = 0,
        kbuffer: int = 16,
        refill_lanes: int = 0,
        block_size: int = 0,
        collect_timings: bool = False,
        sort_rays: bool = True,
        exact_replay: bool = False,
        compensated_grads: bool = True,
        storage: str = "fp32",
        warp_aggregate: bool = True,
        shadow_kbuffer: int = 0,
        exact_candidates: bool = False,
        resume_rounds: int = 0,
        bvh_builder: str = "default",
    ):
        if pipeline not in ("reference",):
            raise ValueError(f"pipeline '{pipeline}' is not available (only 'reference')")
        if backward_pipeline not in ("referenceBwd",):
            raise ValueError(f"backward pipeline '{backward_pipeline}' is not available (only 'referenceBwd')")
        if primitive not in ("instances",):
            raise ValueError(f"primitive type '{primitive}' is not available (only 'instances')")
        if storage not in N.STORAGES:
            raise ValueError(f"storage '{storage}' is not one of {sorted(N.STORAGES)}")
        if bvh_builder not in N.BVH_BUILDERS:
            raise ValueError(f"bvh_builder '{bvh_builder}' is not one of {sorted(N.BVH_BUILDERS)}")
        self._lib = N.load()
        self.sph_degree = int(particle_radiance_sph_degree)
        self.enable_normals = bool(enable_normals)
        cfg = N.PtirConfig(
            float(particle_kernel_degree), float(particle_kernel_min_response), int(bool(particle_kernel_density_clamping)),
            self.sph_degree, int(bool(enable_normals)), int(bool(enable_hit_counts)), int(bool(enable_mis)),
            int(bool(enable_metallic)), int(bool(visualize_lights)), int(bool(collect_counters)),
            N.SCHEDULES[schedule], int(chunk_tiles), int(kbuffer), int(refill_lanes), int(block_size),
            int(bool(collect_timings)), 0 if sort_rays else 1, int(bool(exact_replay)), 0 if compensated_grads else 1,
            N.STORAGES[storage], 0 if warp_aggregate else 1, int(shadow_kbuffer), int(bool(exact_candidates)),
            int(resume_rounds), N.BVH_BUILDERS[bvh_builder])
        handle = C.c_void_p()
        rc = self._lib.ptir_create(C.byref(cfg), C.byref(handle))
        if rc != N.PTIR_OK:
            raise N.PtirError(rc, "ptir_create failed (check the construction options)")
        self._h = handle
        self._n = -1

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.ptir_destroy(h)
            self._h = None

    # --------------------------------------------------------------------------------
    def build_bvh(self, mog_pos, mog_rot, mog_scl, mog_dns, rebuild, allow_update=True):
        """buildBVH (optixTracer.cpp:633-907): instance boxes -> LBVH (rebuild) or refit."""
        pos, rot = _f32(mog_pos, "mog_pos"), _f32(mog_rot, "mog_rot")
        scl, dns = _f32(mog_scl, "mog_scl"), _f32(mog_dns, "mog_dns")
        n = pos.shape[0]
        if rot.shape != (n, 4) or scl.shape != (n, 3) or dns.numel() != n:
            raise ValueError("build_bvh: expected pos [N,3], rot [N,4], scl [N,3], dns [N,1]")
        rc = self._lib.ptir_build_bvh(self._h, _ptr(pos), _ptr(rot), _ptr(scl), _ptr(dns), int(n), int(bool(rebuild)),
                                      int(bool(allow_update)), _stream())
        N.check(self._h, rc, "build_bvh")
        self._n = n

    # --------------------------------------------------------------------------------
    def _args(self, frame, ray_to_world, ray_ori, ray_dir, particle_density, particle_material, particle_radiance,
              particle_shading_normal, environment, environment_alias_table, lights, light_alias_table,
              mesh_light_vertices, mesh_light_triangles, mesh_lights, mesh_light_triangle_alias_table, sh_indirect,
              sph_degree, min_transmittance, max_bounces):
        keep = []
        t2w = _f32(ray_to_world, "ray_to_world")
        if t2w.numel() < 12:
            raise ValueError("ray_to_world must hold at least one 3x4 (or 4x4) transform")
        ori, dirs = _f32_strided(ray_ori, "ray_ori"), _f32_strided(ray_dir, "ray_dir")
        if ori.dim() != 4 or ori.shape[-1] != 3 or dirs.shape != ori.shape:
            raise ValueError("ray_ori / ray_dir must be [Z,H,W,3]")
        dens = _f32(particle_density, "particle_density")
        mat = _f32(particle_material, "particle_material")
        rad = _f32(particle_radiance, "particle_radiance")
        n = dens.shape[0]
        if dens.shape != (n, 12) or mat.shape != (n, 5):
            raise ValueError("particle_density must be [N,12] and particle_material [N,5]")
        coeffs = (self.sph_degree + 1) ** 2 * 3
        if rad.shape != (n, coeffs):
            raise ValueError(f"particle_radiance must be [N,{coeffs}]")
        snrm = _f32(particle_shading_normal, "particle_shading_normal") if particle_shading_normal is not None else None
        if snrm is not None and snrm.numel() != 3 * n:
            raise ValueError("particle_shading_normal must be [N,3]")
        env = environment
        env_ok = (isinstance(env, torch.Tensor) and env.dim() >= 3 and env.shape[0] > 0 and env.shape[1] > 0
                  and env.shape[2] == 4 and env.numel() > 0)
        env = _f32(env, "environment") if env_ok else None
        alias = environment_alias_table
        alias_ok = (isinstance(alias, torch.Tensor) and alias.dim() == 3 and alias.shape[0] == 3 and alias.shape[1] > 0
                    and alias.shape[2] > 0)
        alias = _f32(alias, "environment_alias_table") if alias_ok else None
        lt = _light_tables(lights, light_alias_table, mesh_light_vertices, mesh_light_triangles, mesh_lights,
                           mesh_light_triangle_alias_table)
        keep += [t2w, ori, dirs, dens, mat, rad, snrm, env, alias, *lt]
        a = N.PtirTraceArgs()
        a.frame = int(frame) & 0xFFFFFFFF
        a.ray_to_world = _ptr(t2w)
        a.ray_origin, a.ray_direction = _ptr(ori), _ptr(dirs)
        a.use_strides = 1
        a.ray_origin_strides, a.ray_direction_strides = _strides4(ori), _strides4(dirs)
        a.z, a.h, a.w = int(ori.shape[0]), int(ori.shape[1]), int(ori.shape[2])
        a.particle_density, a.particle_material, a.particle_radiance = _ptr(dens), _ptr(mat), _ptr(rad)
        a.particle_shading_normal = _ptr(snrm)
        a.n = int(n)
        a.environment = _ptr(env)
        a.env_h, a.env_w = (int(env.shape[0]), int(env.shape[1])) if env is not None else (0, 0)
        a.environment_alias = _ptr(alias)
        a.alias_h, a.alias_w = (int(alias.shape[1]), int(alias.shape[2])) if alias is not None else (0, 0)
        lgt, table, verts, tris, mesh, tri_table = lt
        a.lights, a.light_alias, a.mesh_light_vertices = _ptr(lgt), _ptr(table), _ptr(verts)
        a.mesh_light_triangles, a.mesh_lights, a.mesh_light_alias = _ptr(tris), _ptr(mesh), _ptr(tri_table)
        a.num_lights = int(lgt.shape[0]) if lgt is not None else 0
        a.num_light_entries = int(table.shape[1]) if table is not None else 0
        a.num_mesh_light_vertices = int(verts.shape[0]) if verts is not None else 0
        a.num_mesh_light_triangles = int(tris.shape[0]) if tris is not None else 0
        a.num_mesh_lights = int(mesh.shape[0]) if mesh is not None else 0
        a.mesh_light_alias_cols = int(tri_table.shape[1]) if tri_table is not None else 0
        a.sh_indirect = int(sh_indirect)
        a.sph_eval_degree = int(sph_degree)
        a.min_transmittance = float(min_transmittance)
        a.max_bounces = int(max_bounces)
        return a, keep, ori.shape[:3], n, env

    def trace(self, frame, ray_to_world, ray_ori, ray_dir, particle_density, particle_material, particle_radiance,
              particle_shading_normal, environment, environment_alias_table, lights, light_alias_table,
              mesh_light_vertices, mesh_light_triangles, mesh_lights, mesh_light_triangle_alias_table, sh_indirect,
              sph_degree, min_transmittance, max_bounces, _views=None, path_signature=None):
        """trace (optixTracer.cpp:909-1013). Returns (rayRad, rayDns, rayHit[...,2], rayHitSecondMoment,
        rayDepthDistortion, rayNrm, rayShadingNrm, rayMaterial, rayHitsCount, particleVisibility, rayPbr,
        rayLight, rayPbrComponents). `path_signature` (not in the reference): an int32 CUDA tensor of
        Z*H*W elements, contiguous, filled with each path's decision signature (a hash of its
        discrete branches, include/ptir_b200.h), for parity diagnostics."""
        a, keep, zhw, n, _ = self._args(frame, ray_to_world, ray_ori, ray_dir, particle_density, particle_material,
                                        particle_radiance, particle_shading_normal, environment, environment_alias_table,
                                        lights, light_alias_table, mesh_light_vertices, mesh_light_triangles,
                                        mesh_lights, mesh_light_triangle_alias_table, sh_indirect, sph_degree,
                                        min_transmittance, max_bounces)
        dev = particle_density.device
        e = lambda c: torch.empty((*zhw, c), dtype=torch.float32, device=dev)  # noqa: E731
        out = dict(radiance=e(3), density=e(1), hit=e(2), hit2=e(1), distortion=e(1), normal=e(3), snormal=e(3),
                   material=e(5), hits=e(1))
        vis = torch.empty((n, 1), dtype=torch.float32, device=dev)
        pbr, light = e(3), e(3)
        comps = torch.empty((*zhw, 2, 3), dtype=torch.float32, device=dev)
        sig = None
        if path_signature is not None:
            sig = path_signature
            if (sig.dtype != torch.int32 or not sig.is_cuda or not sig.is_contiguous()
                    or sig.numel() != int(zhw[0]) * int(zhw[1]) * int(zhw[2])):
                raise ValueError("path_signature must be a contiguous int32 CUDA tensor with one element per sample")
        o = N.PtirTraceOutputs(
            _ptr(out["radiance"]), _ptr(out["density"]), _ptr(out["hit"]), _ptr(out["hit2"]), _ptr(out["distortion"]),
            _ptr(out["normal"]), _ptr(out["snormal"]), _ptr(out["material"]), _ptr(out["hits"]), _ptr(pbr),
            _ptr(light), _ptr(comps), _ptr(vis), _ptr(sig))
        if _views is None:
            rc = self._lib.ptir_trace(self._h, C.byref(a), C.byref(o), _stream())
        else:
            rc = self._lib.ptir_trace_views(self._h, C.byref(a), _views, len(_views), C.byref(o), _stream())
        N.check(self._h, rc, "trace")
        del keep
        return (out["radiance"], out["density"], out["hit"], out["hit2"], out["distortion"], out["normal"],
                out["snormal"], out["material"], out["hits"], vis, pbr, light, comps)

    def trace_bwd(self, frame, ray_to_world, ray_ori, ray_dir, ray_rad, ray_dns, ray_hit, ray_hit_second_moment,
                  ray_depth_distortion, ray_nrm, ray_shading_nrm, ray_material, ray_pbr, ray_light, particle_density,
                  particle_material, particle_radiance, particle_shading_normal, environment, environment_alias_table,
                  lights, light_alias_table, mesh_light_vertices, mesh_light_triangles, mesh_lights,
                  mesh_light_triangle_alias_table, ray_rad_grd, ray_dns_grd, ray_hit_grd, ray_hit_second_moment_grd,
                  ray_depth_distortion_grd, ray_nrm_grd, ray_shading_nrm_grd, ray_material_grd, ray_pbr_grd,
                  ray_light_grd, sh_indirect, sph_degree, min_transmittance, max_bounces, _views=None):
        """traceBwd (optixTracer.cpp:1015-1145). Returns (densityGrad [N,12], materialGrad [N,5],
        radianceGrad [N,C], shadingNormalGrad [N,3], environmentGrad like environment); as in the
        reference only the material and environment gradients are non-zero."""
        a, keep, zhw, n, env = self._args(frame, ray_to_world, ray_ori, ray_dir, particle_density, particle_material,
                                          particle_radiance, particle_shading_normal, environment,
                                          environment_alias_table, lights, light_alias_table, mesh_light_vertices,
                                          mesh_light_triangles, mesh_lights, mesh_light_triangle_alias_table,
                                          sh_indirect, sph_degree, min_transmittance, max_bounces)
        dev = particle_density.device

        def g(t, c, name):
            if t is None:
                return None
            t = _f32_strided(t, name)
            if t.dim() != 4 or tuple(t.shape[:3]) != tuple(zhw) or t.shape[-1] != c:
                raise ValueError(f"{name} must be [Z,H,W,{c}]")
            return t

        pbr, light = g(ray_pbr, 3, "ray_pbr"), g(ray_light, 3, "ray_light")
        pbr_g, light_g = g(ray_pbr_grd, 3, "ray_pbr_grd"), g(ray_light_grd, 3, "ray_light_grd")
        mat_g = g(ray_material_grd, 5, "ray_material_grd")
        keep += [pbr, light, pbr_g, light_g, mat_g]
        density_grad = torch.zeros((n, 12), dtype=torch.float32, device=dev)
        material_grad = torch.empty((n, 5), dtype=torch.float32, device=dev)
        radiance_grad = torch.zeros_like(particle_radiance)
        snrm_grad = (torch.zeros_like(particle_shading_normal) if particle_shading_normal is not None
                     else torch.zeros((n, 3), dtype=torch.float32, device=dev))
        env_grad = torch.zeros_like(environment)
        b = N.PtirBwdArgs(_ptr(pbr), _ptr(light), _ptr(pbr_g), _ptr(light_g), _ptr(mat_g), 1, _strides4(pbr),
                          _strides4(light), _strides4(pbr_g), _strides4(light_g), _strides4(mat_g))
        o = N.PtirBwdOutputs(_ptr(material_grad), _ptr(env_grad) if env is not None else None)
        if _views is None:
            rc = self._lib.ptir_trace_bwd(self._h, C.byref(a), C.byref(b), C.byref(o), _stream())
        else:
            rc = self._lib.ptir_trace_bwd_views(self._h, C.byref(a), _views, len(_views), C.byref(b), C.byref(o),
                                                _stream())
        N.check(self._h, rc, "trace_bwd")
        del keep
        return density_grad, material_grad, radiance_grad, snrm_grad, env_grad

    # --------------------------------------------------------------------------------
    # batched views (not in the reference): several views of their own extent in one launch sequence
    def _view_table(self, views):
        """views: sequence of (frame, ray_to_world [>=1,4,4], z, h, w). Returns the C table, the
        tensors to keep alive, and the total launch count."""
        if not 1 <= len(views) <= N.MAX_VIEWS:
            raise ValueError(f"between 1 and {N.MAX_VIEWS} views per batch")
        table = (N.PtirView * len(views))()
        keep, total = [], 0
        for k, (frame, t2w, z, h, w) in enumerate(views):
            t2w = _f32(t2w, "ray_to_world")
            if t2w.numel() < 12:
                raise ValueError("ray_to_world must hold at least one 3x4 (or 4x4) transform")
            keep.append(t2w)
            table[k] = N.PtirView(int(z), int(h), int(w), int(frame) & 0xFFFFFFFF, _ptr(t2w))
            total += int(z) * int(h) * int(w)
        return table, keep, total

    def trace_views(self, views, ray_ori, ray_dir, particle_density, particle_material, particle_radiance,
                    particle_shading_normal, environment, environment_alias_table, lights, light_alias_table,
                    mesh_light_vertices, mesh_light_triangles, mesh_lights, mesh_light_triangle_alias_table,
                    sh_indirect, sph_degree, min_transmittance, max_bounces, path_signature=None):
        """trace() over a batch of views of their own extent and sample count, in one launch
        sequence. `views` lists (frame, ray_to_world, z, h, w); ray_ori / ray_dir are the views'
        [Z,H,W,3] rays concatenated in view order, [T,3]. Returns the 13 outputs of trace() with
        every per-sample output flat, [T,C] (split_views() cuts them per view); each view's
        values are those of its own trace() call."""
        table, keep_t, total = self._view_table(views)
        ori = _f32_strided(ray_ori, "ray_ori").reshape(1, 1, -1, 3)
        dirs = _f32_strided(ray_dir, "ray_dir").reshape(1, 1, -1, 3)
        if ori.shape[2] != total or dirs.shape != ori.shape:
            raise ValueError(f"ray_ori / ray_dir must hold the {total} rays of the views")
        out = self.trace(views[0][0], keep_t[0], ori, dirs, particle_density, particle_material, particle_radiance,
                         particle_shading_normal, environment, environment_alias_table, lights, light_alias_table,
                         mesh_light_vertices, mesh_light_triangles, mesh_lights, mesh_light_triangle_alias_table,
                         sh_indirect, sph_degree, min_transmittance, max_bounces, _views=table,
                         path_signature=path_signature)
        flat = [t if k == 9 else t.reshape(total, *t.shape[3:]) for k, t in enumerate(out)]
        del keep_t
        return tuple(flat)

    def trace_bwd_views(self, views, ray_ori, ray_dir, ray_rad, ray_dns, ray_hit, ray_hit_second_moment,
                        ray_depth_distortion, ray_nrm, ray_shading_nrm, ray_material, ray_pbr, ray_light,
                        particle_density, particle_material, particle_radiance, particle_shading_normal, environment,
                        environment_alias_table, lights, light_alias_table, mesh_light_vertices, mesh_light_triangles,
                        mesh_lights, mesh_light_triangle_alias_table, ray_rad_grd, ray_dns_grd, ray_hit_grd,
                        ray_hit_second_moment_grd, ray_depth_distortion_grd, ray_nrm_grd, ray_shading_nrm_grd,
                        ray_material_grd, ray_pbr_grd, ray_light_grd, sh_indirect, sph_degree, min_transmittance,
                        max_bounces):
        """trace_bwd() over a batch of views; per-sample inputs flat [T,C] as trace_views() returns them."""
        table, keep_t, total = self._view_table(views)
        r = lambda t: None if t is None else t.reshape(1, 1, total, -1)  # noqa: E731
        ori, dirs = r(_f32_strided(ray_ori, "ray_ori")), r(_f32_strided(ray_dir, "ray_dir"))
        res = self.trace_bwd(views[0][0], keep_t[0], ori, dirs, r(ray_rad), r(ray_dns), r(ray_hit),
                             r(ray_hit_second_moment), r(ray_depth_distortion), r(ray_nrm), r(ray_shading_nrm),
                             r(ray_material), r(ray_pbr), r(ray_light), particle_density, particle_material,
                             particle_radiance, particle_shading_normal, environment, environment_alias_table, lights,
                             light_alias_table, mesh_light_vertices, mesh_light_triangles, mesh_lights,
                             mesh_light_triangle_alias_table, r(ray_rad_grd), r(ray_dns_grd), r(ray_hit_grd),
                             r(ray_hit_second_moment_grd), r(ray_depth_distortion_grd), r(ray_nrm_grd),
                             r(ray_shading_nrm_grd), r(ray_material_grd), r(ray_pbr_grd), r(ray_light_grd),
                             sh_indirect, sph_degree, min_transmittance, max_bounces, _views=table)
        del keep_t
        return res

    # --------------------------------------------------------------------------------
    # extensions (not in the reference): counters and device status for tests and benchmarks
    def counters(self, stage: str | None = None) -> dict:
        """Device counters of the last trace / trace_bwd, of all kernels or of one stage
        ("intersect", "shadow", "replay", "shading", "megakernel", "sort")."""
        c = N.PtirCounters()
        if stage is None:
            rc = self._lib.ptir_get_counters(self._h, C.byref(c), _stream())
        else:
            rc = self._lib.ptir_get_stage_counters(self._h, N.STAGES.index(stage), C.byref(c), _stream())
        N.check(self._h, rc, "counters")
        return c.as_dict()

    def set_collect_timings(self, on: bool) -> None:
        """Launch timing on or off (keep it off while capturing a CUDA graph)."""
        N.check(self._h, self._lib.ptir_set_collect_timings(self._h, int(bool(on))), "set_collect_timings")

    def stage_times(self) -> dict:
        """{stage: (milliseconds, launches)} recorded since the previous call (collect_timings=True):
        CUDA events around every launch, on the launch stream."""
        t = N.PtirStageTimes()
        N.check(self._h, self._lib.ptir_get_stage_times(self._h, C.byref(t)), "stage_times")
        return {name: (float(t.ms[k]), int(t.launches[k])) for k, name in enumerate(N.STAGES)}

    def device_status(self) -> int:
        w = C.c_uint32(0)
        self._lib.ptir_device_status(self._h, C.byref(w), _stream())
        return int(w.value)

    def scene_bounds(self) -> torch.Tensor:
        out = (C.c_float * 6)()
        N.check(self._h, self._lib.ptir_scene_bounds(self._h, out, _stream()), "scene_bounds")
        return torch.tensor(list(out), dtype=torch.float32)

    def debug_accel(self):
        """(nodes [N-1,16], leaves [N,16]) float32 host copies of the acceleration structure."""
        n = max(self._n, 0)
        nodes = torch.zeros((max(n - 1, 0), 16), dtype=torch.float32)
        leaves = torch.zeros((n, 16), dtype=torch.float32)
        rc = self._lib.ptir_debug_accel(self._h, nodes.data_ptr() if n > 1 else None, leaves.data_ptr() if n else None,
                                        _stream())
        N.check(self._h, rc, "debug_accel")
        return nodes, leaves
