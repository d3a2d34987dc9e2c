"""myrt_b200: B200-native wavefront path-tracing core behind myrt's interfaces.

Python front end over the C ABI (include/myrt_cuda.h). The compute path is the
in-tree CUDA library libmyrt_b200.so. It is loaded on first use (a Context,
a host BVH build, ...), not at import, so the pure-numpy scene generators in
``myrt_b200.scenes`` can be used by processes that must not map it; every
call that needs it raises when it has not been built (there is no CPU
fallback).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import ISECT_REFERENCE, ISECT_WATERTIGHT, MYRT_ERR_DEVICE_ABORT, MYRT_ERR_UNSUPPORTED, MYRT_OK  # noqa: F401

HIT_DTYPE = np.dtype([("prim", np.int32), ("t", np.float32), ("u", np.float32), ("v", np.float32)])


class MyrtError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"myrt error {code}: {message}")
        self.code = code


def _ptr(a) -> int | None:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if isinstance(a, C.Array):
        return C.addressof(a)
    return int(a.data_ptr())  # torch tensor


def bvh_info_dict(info: _abi.myrt_bvh_info) -> dict:
    return {f: getattr(info, f) for f, _ in _abi.myrt_bvh_info._fields_ if f != "pad"}


def forward_default_shadow():
    """The light camera of forward_renderer::pass_shadow as the library builds
    it: (view, projection), numpy [4, 4] in math layout."""
    v = np.zeros(16, np.float32)
    p = np.zeros(16, np.float32)
    _abi.lib().myrt_forward_default_shadow(v.ctypes.data, p.ctypes.data)
    return v.reshape(4, 4).T.copy(), p.reshape(4, 4).T.copy()


def build_bvh8(positions: np.ndarray):
    """Host-only BVH build. positions: float32 [T, 3, 3] (or [T, 9]).
    Returns (nodes uint32 [N, 20], triangles float32 [M, 12], info dict)."""
    pos = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 9)
    L = _abi.lib()
    h = C.c_void_p()
    rc = L.myrt_bvh8_build(pos.ctypes.data, pos.shape[0], C.byref(h))
    if rc != MYRT_OK:
        raise MyrtError(rc, "myrt_bvh8_build failed")
    try:
        info = _abi.myrt_bvh_info()
        L.myrt_bvh8_get_info(h, C.byref(info))
        nodes = np.zeros((info.wide_nodes, 20), np.uint32)
        tris = np.zeros((info.triangles, 12), np.float32)
        L.myrt_bvh8_copy(h, nodes.ctypes.data, tris.ctypes.data)
        return nodes, tris, bvh_info_dict(info)
    finally:
        L.myrt_bvh8_free(h)


class Context:
    """One CUDA device, one stream, one resident scene (myrt_ctx)."""

    def __init__(self, device: int = 0):
        self._L = _abi.lib()
        self._h = C.c_void_p()
        opts = _abi.myrt_device_opts(device, 0)
        rc = self._L.myrt_ctx_create(C.byref(opts), C.byref(self._h))
        if rc != MYRT_OK:
            raise MyrtError(rc, "myrt_ctx_create failed")
        self._keep = []

    # -- lifecycle --
    def close(self):
        if self._h:
            self._L.myrt_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str):
        if rc != MYRT_OK:
            buf = C.create_string_buffer(512)
            self._L.myrt_get_last_error(self._h, buf, 512)
            raise MyrtError(rc, f"{what}: {buf.value.decode(errors='replace')}")

    def set_tuning(self, trace_persistent: int = 0, refill: int = 1, blocks_per_sm: int = 0,
                   trace_min_blocks: int = 0, trace_unit_steps: int = 0, wave_paths: int = 0,
                   pt_blocks_per_sm: int = 0, trace_smem_stack: int = 0, trace_order: int = 0,
                   bvh_builder: int = 0, sdf_cells: int = 0, guide_poll_limit: int = 0, guide_stall_test: int = 0,
                   instancing: int = 0, pt_grid: int = 0, ref_frames: int = 0):
        t = _abi.myrt_tuning(trace_persistent, refill, blocks_per_sm, trace_min_blocks, trace_unit_steps,
                             wave_paths, pt_blocks_per_sm, trace_smem_stack, bvh_builder, trace_order, sdf_cells,
                             guide_poll_limit, guide_stall_test, instancing, pt_grid, ref_frames)
        self._check(self._L.myrt_set_tuning(self._h, C.byref(t)), "myrt_set_tuning")

    def set_transforms(self, drawables):
        """myrt_scene_set_transforms: new transforms / material indices for the
        uploaded drawables (a ctypes array of myrt_drawable); re-bake and rebuild
        on the device. Returns bvh_info()."""
        self._check(self._L.myrt_scene_set_transforms(self._h, C.cast(drawables, C.c_void_p), len(drawables)),
                    "myrt_scene_set_transforms")
        return self.bvh_info()

    def scene_bvh(self):
        """The scene's device tree: (nodes uint32 [N, 20], triangles float32 [T, 12])."""
        info = self.bvh_info()
        nodes = np.empty((int(info["wide_nodes"]), 20), np.uint32)
        tris = np.empty((int(info["triangles"]), 12), np.float32)
        self._check(self._L.myrt_scene_copy_bvh(self._h, nodes.ctypes.data, tris.ctypes.data), "myrt_scene_copy_bvh")
        return nodes, tris

    def set_phase_timing(self, enable: bool = True):
        """Device-time accounting of the ray queries (ordering, traversal)."""
        self._check(self._L.myrt_set_phase_timing(self._h, int(enable)), "myrt_set_phase_timing")

    def phase_times(self) -> dict:
        """Summed device milliseconds of the queries since the last call: order_ms
        (ray keys + radix sort), traverse_ms (traversal kernel), queries."""
        o, t, q = C.c_double(), C.c_double(), C.c_uint64()
        self._check(self._L.myrt_get_phase_times(self._h, C.byref(o), C.byref(t), C.byref(q)),
                    "myrt_get_phase_times")
        return dict(order_ms=o.value, traverse_ms=t.value, queries=q.value)

    def get_tuning(self) -> dict:
        t = _abi.myrt_tuning()
        self._check(self._L.myrt_get_tuning(self._h, C.byref(t)), "myrt_get_tuning")
        return {f: getattr(t, f) for f, _ in _abi.myrt_tuning._fields_}

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        self._check(self._L.myrt_get_stream(self._h, C.byref(s)), "myrt_get_stream")
        return s.value or 0

    # -- scene --
    def upload_scene(self, indices: np.ndarray, vertices: np.ndarray, normals: np.ndarray | None = None,
                     uvs: np.ndarray | None = None, drawables: np.ndarray | None = None,
                     materials: np.ndarray | None = None, material_data: np.ndarray | None = None) -> dict:
        """Mirror of scene::prepare's uploads. vertices/normals: float32 [V, 3|4]."""
        idx = np.ascontiguousarray(indices, dtype=np.uint32).ravel()

        def pad4(a):
            a = np.asarray(a, np.float32)
            if a.shape[1] == 4:
                return np.ascontiguousarray(a)
            out = np.zeros((a.shape[0], 4), np.float32)
            out[:, :3] = a
            return out

        verts = pad4(vertices)
        nrm = pad4(normals) if normals is not None else None
        uv = np.ascontiguousarray(uvs, np.float32) if uvs is not None else None
        mats = np.ascontiguousarray(materials, np.int32).reshape(-1, 2) if materials is not None else None
        mdata = np.ascontiguousarray(material_data, np.float32).ravel() if material_data is not None else None
        view = _abi.myrt_scene_view(
            idx.ctypes.data, idx.size, verts.ctypes.data, verts.shape[0], _ptr(nrm), _ptr(uv),
            _ptr(drawables), 0 if drawables is None else len(drawables), _ptr(mats),
            0 if mats is None else mats.shape[0], _ptr(mdata), 0 if mdata is None else mdata.size)
        self._check(self._L.myrt_scene_upload(self._h, C.byref(view)), "myrt_scene_upload")
        return self.bvh_info()

    def upload_sdf(self, instrs, programs, params, drawables):
        """SDF programs + drawables (myrt_sdf_upload). drawables: float32 [N, 36]
        (myrt_b200.sdf.sdf_drawables); an empty array removes all SDF drawables."""
        ins = np.ascontiguousarray(instrs, np.int32).reshape(-1, 2)
        prs = np.ascontiguousarray(programs, np.int32).reshape(-1, 2)
        par = np.ascontiguousarray(params, np.float32).ravel()
        dr = np.ascontiguousarray(drawables, np.float32).reshape(-1, 36)
        view = _abi.myrt_sdf_view(ins.ctypes.data, ins.shape[0], prs.ctypes.data, prs.shape[0], par.ctypes.data,
                                  par.size, dr.ctypes.data, dr.shape[0])
        self._check(self._L.myrt_sdf_upload(self._h, C.byref(view)), "myrt_sdf_upload")

    def trace_sdf(self, rays, steps: int, eps: float, any_hit: bool = False, rng_states=None) -> dict:
        """SDF closest / any hit for host rays (myrt_trace_sdf)."""
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        out = np.empty((r.shape[0], 8), np.float32)
        rs = None if rng_states is None else np.ascontiguousarray(rng_states, np.uint32)
        self._check(self._L.myrt_trace_sdf(self._h, r.ctypes.data, r.shape[0], steps, eps, int(any_hit),
                                           _ptr(rs), out.ctypes.data), "myrt_trace_sdf")
        return dict(hit=out[:, 0].astype(np.int32), t=out[:, 1].copy(), normal=out[:, 2:5].copy(),
                    uv=out[:, 5:7].copy(), material=out[:, 7].copy().view(np.int32))

    def bvh_info(self) -> dict:
        info = _abi.myrt_bvh_info()
        self._check(self._L.myrt_scene_bvh_info(self._h, C.byref(info)), "myrt_scene_bvh_info")
        return bvh_info_dict(info)

    # -- host-memory queries (copies inside the call) --
    def trace_closest(self, rays: np.ndarray, intersector: int = ISECT_REFERENCE, out: np.ndarray | None = None):
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        hits = out if out is not None else np.empty(r.shape[0], HIT_DTYPE)
        self._check(self._L.myrt_trace_closest(self._h, r.ctypes.data, r.shape[0], hits.ctypes.data, intersector),
                    "myrt_trace_closest")
        return hits

    def trace_any(self, rays: np.ndarray, intersector: int = ISECT_REFERENCE):
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        occ = np.empty(r.shape[0], np.uint8)
        self._check(self._L.myrt_trace_any(self._h, r.ctypes.data, r.shape[0], occ.ctypes.data, intersector),
                    "myrt_trace_any")
        return occ

    # -- device-memory queries (torch tensors; asynchronous on `stream`) --
    def trace_closest_device(self, rays, hits, intersector: int = ISECT_REFERENCE, stream: int | None = None):
        n = rays.numel() // 8
        self._check(self._L.myrt_trace_closest_device(self._h, _ptr(rays), n, _ptr(hits), intersector, stream),
                    "myrt_trace_closest_device")

    def trace_any_device(self, rays, occluded, intersector: int = ISECT_REFERENCE, stream: int | None = None):
        n = rays.numel() // 8
        self._check(self._L.myrt_trace_any_device(self._h, _ptr(rays), n, _ptr(occluded), intersector, stream),
                    "myrt_trace_any_device")

    def trace_closest_stats_device(self, rays, hits, nodes, tris, intersector: int = ISECT_REFERENCE,
                                   stream: int | None = None):
        n = rays.numel() // 8
        self._check(self._L.myrt_trace_closest_stats_device(self._h, _ptr(rays), n, _ptr(hits), _ptr(nodes),
                                                            _ptr(tris), intersector, stream),
                    "myrt_trace_closest_stats_device")

    def sync(self):
        self._check(self._L.myrt_sync(self._h), "myrt_sync")

    GLSL_FUNCTIONS = {"sin": 0, "cos": 1, "atan": 2, "exp": 3, "pow": 4}

    def glsl_builtin(self, name: str, x, y=None) -> np.ndarray:
        """myrt_glsl_builtins: the library's GLSL built-in `name` on the device."""
        xs = np.ascontiguousarray(x, np.float32).ravel()
        ys = None if y is None else np.ascontiguousarray(np.broadcast_to(np.float32(y) if np.isscalar(y) else y,
                                                                          xs.shape), np.float32).ravel()
        out = np.empty_like(xs)
        self._check(self._L.myrt_glsl_builtins(self._h, self.GLSL_FUNCTIONS[name], xs.ctypes.data,
                                               None if ys is None else ys.ctypes.data, xs.size, out.ctypes.data),
                    "myrt_glsl_builtins")
        return out

    # -- wavefront rendering (sequential_pathtracer::run) --
    def render(self, inverse_view, inverse_projection, width: int, height: int, num_bounces: int = 10,
               frames: int = 1, shading: int = _abi.SHADE_REFERENCE, sdf_marching_steps: int = 400,
               sdf_marching_epsilon: float = 1e-5, dof: bool = False, lens_size=(0.2, 0.2), focus: float = 1.0,
               bokeh_slot: int = -1):
        cam = _abi.myrt_camera()
        cam.inverse_view[:] = np.asarray(inverse_view, np.float32).ravel().tolist()
        cam.inverse_projection[:] = np.asarray(inverse_projection, np.float32).ravel().tolist()
        p = _abi.myrt_render_params(width, height, num_bounces, frames, shading, 0, sdf_marching_steps,
                                    sdf_marching_epsilon)
        p.dof_active = int(dof)
        p.lens_size[:] = [float(lens_size[0]), float(lens_size[1])]
        p.focus = float(focus)
        p.bokeh_texture = bokeh_slot + 1 if bokeh_slot >= 0 else 0
        self._check(self._L.myrt_render(self._h, C.byref(cam), C.byref(p)), "myrt_render")

    def upload_texture(self, slot: int, rgba, wrap: int = 0):
        """myrt_texture_upload: rgba float32 [H, W, 4] (None empties the slot)."""
        if rgba is None:
            self._check(self._L.myrt_texture_upload(self._h, slot, None, 0, 0, wrap), "myrt_texture_upload")
            return
        a = np.ascontiguousarray(rgba, np.float32)
        self._check(self._L.myrt_texture_upload(self._h, slot, a.ctypes.data, a.shape[1], a.shape[0], wrap),
                    "myrt_texture_upload")

    def upload_cubemap(self, faces):
        """myrt_cubemap_upload: faces float32 [6, S, S, 4] (+x, -x, +y, -y, +z, -z); None removes it."""
        if faces is None:
            self._check(self._L.myrt_cubemap_upload(self._h, None, 0), "myrt_cubemap_upload")
            return
        a = np.ascontiguousarray(faces, np.float32)
        self._check(self._L.myrt_cubemap_upload(self._h, a.ctypes.data, a.shape[1]), "myrt_cubemap_upload")

    def forward_render(self, view, projection, width: int, height: int, random_seed: int = 0,
                       shadow_size: int = 0, shadow_view=None, shadow_projection=None):
        """myrt_forward_run (forward_renderer::run): view / projection are
        column-major 4x4 (numpy [4, 4] in math layout is transposed for you
        when given as a 2-D array); shadow_view / shadow_projection replace the
        reference's light camera when both are given."""
        p = _abi.myrt_forward_params()
        p.width, p.height = width, height

        def colmajor(m):
            a = np.asarray(m, np.float32)
            return (a.T if a.ndim == 2 else a).ravel()

        p.view[:] = colmajor(view).tolist()
        p.projection[:] = colmajor(projection).tolist()
        p.random_seed = int(random_seed) & 0xFFFFFFFF
        p.shadow_size = shadow_size
        if shadow_view is not None and shadow_projection is not None:
            p.custom_shadow = 1
            p.shadow_view[:] = colmajor(shadow_view).tolist()
            p.shadow_projection[:] = colmajor(shadow_projection).tolist()
        self._check(self._L.myrt_forward_run(self._h, C.byref(p)), "myrt_forward_run")

    def forward_read(self, width: int, height: int, shadow_size: int = 2048) -> dict:
        """myrt_forward_read: result / gbuffer as float32 (from their half
        bits), shadow_map float32, visibility uint64."""
        res = np.empty((height, width, 4), np.uint16)
        gb = np.empty((3, height, width, 4), np.uint16)
        sm = np.empty((shadow_size, shadow_size, 4), np.float32)
        vis = np.empty((height, width), np.uint64)
        self._check(self._L.myrt_forward_read(self._h, width, height, shadow_size, res.ctypes.data, gb.ctypes.data,
                                              sm.ctypes.data, vis.ctypes.data), "myrt_forward_read")
        return {"result": res.view(np.float16).astype(np.float32), "gbuffer": gb.view(np.float16).astype(np.float32),
                "shadow_map": sm, "visibility": vis}

    def forward_result(self, width: int, height: int, shadow_size: int = 2048, out=None) -> np.ndarray:
        """The last forward run's RGBA16F result as half bits (uint16 [H, W, 4]),
        copied into `out` when given."""
        res = out if out is not None else np.empty((height, width, 4), np.uint16)
        self._check(self._L.myrt_forward_read(self._h, width, height, shadow_size, res.ctypes.data, None, None,
                                              None), "myrt_forward_read")
        return res

    def forward_buffers(self) -> dict:
        """Device pointers of the last forward run's images."""
        ptrs = [C.c_void_p() for _ in range(4)]
        self._check(self._L.myrt_forward_buffers(self._h, *[C.byref(q) for q in ptrs]), "myrt_forward_buffers")
        return dict(zip(("result", "gbuffer", "shadow_map", "visibility"), [q.value for q in ptrs]))

    def set_area_lights(self, lights):
        """myrt_set_area_lights: lights [n, 12] float32 rows (corner, edge_u,
        edge_v, emission)."""
        L = np.ascontiguousarray(lights, np.float32).reshape(-1, 12)
        arr = (_abi.myrt_area_light * max(1, L.shape[0]))()
        C.memmove(arr, L.ctypes.data, L.nbytes)
        self._check(self._L.myrt_set_area_lights(self._h, arr, L.shape[0]), "myrt_set_area_lights")

    def render_physical(self, inverse_view, inverse_projection, width: int, height: int, spp: int = 1,
                        max_depth: int = 8, rr_start: int = 3, seed: int = 0, env=(0.0, 0.0, 0.0),
                        fp64: bool = False, guided: bool = False, wave_paths: int = 0,
                        sdf_marching_steps: int = 256, sdf_marching_epsilon: float = 1e-4):
        """Physical (or guided) shading: `spp` samples per pixel accumulated
        into the context's images."""
        cam = _abi.myrt_camera()
        cam.inverse_view[:] = np.asarray(inverse_view, np.float32).ravel().tolist()
        cam.inverse_projection[:] = np.asarray(inverse_projection, np.float32).ravel().tolist()
        p = _abi.myrt_render_params()
        p.width, p.height, p.num_bounces, p.frames = width, height, 0, spp
        p.shading = _abi.SHADE_GUIDED if guided else _abi.SHADE_PHYSICAL
        p.sdf_marching_steps, p.sdf_marching_epsilon = sdf_marching_steps, sdf_marching_epsilon
        p.max_depth, p.rr_start, p.seed, p.accum_fp64 = max_depth, rr_start, seed, int(fp64)
        p.env_radiance[:] = [float(x) for x in env]
        p.wave_paths = wave_paths
        self._check(self._L.myrt_render(self._h, C.byref(cam), C.byref(p)), "myrt_render")

    def render_stats(self) -> dict:
        """Cumulative camera / extension / shadow ray counts of the physical wavefront."""
        st = _abi.myrt_render_stats()
        self._check(self._L.myrt_get_render_stats(self._h, C.byref(st)), "myrt_get_render_stats")
        return dict(paths=st.paths, extension_rays=st.extension_rays, shadow_rays=st.shadow_rays)

    # ---- learned path guiding ----
    def guide_configure(self, **kw):
        """myrt_guide_configure; keys: fraction, learning_rate, train_steps,
        batch, train, warmup_waves, seed (unset keys keep their values)."""
        p = _abi.myrt_guide_params()
        self._check(self._L.myrt_guide_get_config(self._h, C.byref(p)), "myrt_guide_get_config")
        for k, v in kw.items():
            if not hasattr(p, k):
                raise KeyError(k)
            setattr(p, k, v)
        self._check(self._L.myrt_guide_configure(self._h, C.byref(p)), "myrt_guide_configure")

    def guide_config(self) -> dict:
        p = _abi.myrt_guide_params()
        self._check(self._L.myrt_guide_get_config(self._h, C.byref(p)), "myrt_guide_get_config")
        return {f: getattr(p, f) for f, _ in _abi.myrt_guide_params._fields_}

    def guide_reset(self):
        self._check(self._L.myrt_guide_reset(self._h), "myrt_guide_reset")

    def guide_params(self) -> np.ndarray:
        out = np.empty(_abi.GUIDE_PARAM_COUNT, np.float32)
        self._check(self._L.myrt_guide_get_params(self._h, out.ctypes.data), "myrt_guide_get_params")
        return out

    def guide_set_params(self, params):
        p = np.ascontiguousarray(params, np.float32).ravel()
        assert p.size == _abi.GUIDE_PARAM_COUNT
        self._check(self._L.myrt_guide_set_params(self._h, p.ctypes.data), "myrt_guide_set_params")

    def guide_eval(self, points) -> np.ndarray:
        """points [n, 12] (position, 1, normal, 0, view, 0) -> lobes [n, 64]."""
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 12)
        out = np.empty((pts.shape[0], 64), np.float32)
        self._check(self._L.myrt_guide_eval(self._h, pts.ctypes.data, pts.shape[0], out.ctypes.data),
                    "myrt_guide_eval")
        return out

    def guide_gradients(self, samples):
        """samples [n, 16] (position, w, normal, 0, view, 0, direction, 0) -> (grads, loss)."""
        smp = np.ascontiguousarray(samples, np.float32).reshape(-1, 16)
        g = np.empty(_abi.GUIDE_PARAM_COUNT, np.float32)
        loss = C.c_float()
        self._check(self._L.myrt_guide_gradients(self._h, smp.ctypes.data, smp.shape[0], g.ctypes.data,
                                                 C.byref(loss)), "myrt_guide_gradients")
        return g, loss.value

    def guide_train(self, samples, steps: int) -> np.ndarray:
        smp = np.ascontiguousarray(samples, np.float32).reshape(-1, 16)
        loss = np.zeros(max(steps, 1), np.float32)
        self._check(self._L.myrt_guide_train(self._h, smp.ctypes.data, smp.shape[0], steps, loss.ctypes.data),
                    "myrt_guide_train")
        return loss[:steps]

    def guide_stats(self) -> dict:
        st = _abi.myrt_guide_stats()
        self._check(self._L.myrt_guide_get_stats(self._h, C.byref(st)), "myrt_guide_get_stats")
        return {f: getattr(st, f) for f, _ in _abi.myrt_guide_stats._fields_ if f != "pad"}

    def begin_samples(self, first_sample: int):
        """myrt_begin_samples: the next render starts a new accumulation whose
        (physical / guided) samples are numbered from first_sample."""
        self._check(self._L.myrt_begin_samples(self._h, int(first_sample)), "myrt_begin_samples")

    def render_buffer_f64(self) -> int:
        """Device pointer of the FP64 accumulation (myrt_render_buffer_f64)."""
        p = C.c_void_p()
        self._check(self._L.myrt_render_buffer_f64(self._h, C.byref(p)), "myrt_render_buffer_f64")
        return p.value

    def render_size(self) -> tuple[int, int]:
        """(width, height) of the context's render images (myrt_render_size)."""
        w, h = C.c_uint32(), C.c_uint32()
        self._check(self._L.myrt_render_size(self._h, C.byref(w), C.byref(h)), "myrt_render_size")
        return w.value, h.value

    def _check_size(self, width: int, height: int):
        if (width, height) != self.render_size():
            raise MyrtError(_abi.MYRT_ERR_INVALID_ARGUMENT,
                            f"images are {self.render_size()}, not {(width, height)}")

    def read_accumulation_f64(self, width: int, height: int):
        self._check_size(width, height)
        acc = np.empty((height, width, 4), np.float64)
        self._check(self._L.myrt_read_accumulation_f64(self._h, acc.ctypes.data), "myrt_read_accumulation_f64")
        return acc

    def render_noalloc(self, inverse_view, inverse_projection, width: int, height: int, accum, display,
                       sample_index: int = 0, num_bounces: int = 10, frames: int = 1,
                       shading: int = _abi.SHADE_REFERENCE, stream: int | None = None,
                       sdf_marching_steps: int = 400, sdf_marching_epsilon: float = 1e-5, dof: bool = False,
                       lens_size=(0.2, 0.2), focus: float = 1.0, bokeh_slot: int = -1):
        """myrt_render_noalloc: renders into caller-owned device images (torch
        tensors, float32 [H, W, 4]) with no device allocation by the library.
        Camera and shading options as render()."""
        cam = _abi.myrt_camera()
        cam.inverse_view[:] = np.asarray(inverse_view, np.float32).ravel().tolist()
        cam.inverse_projection[:] = np.asarray(inverse_projection, np.float32).ravel().tolist()
        p = _abi.myrt_render_params(width, height, num_bounces, frames, shading, 0, sdf_marching_steps,
                                    sdf_marching_epsilon)
        p.dof_active = int(dof)
        p.lens_size[:] = [float(lens_size[0]), float(lens_size[1])]
        p.focus = float(focus)
        p.bokeh_texture = bokeh_slot + 1 if bokeh_slot >= 0 else 0
        self._check(self._L.myrt_render_noalloc(self._h, C.byref(cam), C.byref(p), sample_index, _ptr(accum),
                                                _ptr(display), stream), "myrt_render_noalloc")

    def read_accumulation(self, width: int, height: int):
        """(rgb sum + count, display) images as float32 [H, W, 4]."""
        self._check_size(width, height)
        acc = np.empty((height, width, 4), np.float32)
        disp = np.empty((height, width, 4), np.float32)
        self._check(self._L.myrt_read_accumulation(self._h, acc.ctypes.data, disp.ctypes.data),
                    "myrt_read_accumulation")
        return acc, disp

    def reset_accumulation(self):
        self._check(self._L.myrt_reset_accumulation(self._h), "myrt_reset_accumulation")

    def sample_count(self) -> int:
        c = C.c_uint32()
        self._check(self._L.myrt_sample_count(self._h, C.byref(c)), "myrt_sample_count")
        return c.value

    def set_seed(self, seed: int):
        self._check(self._L.myrt_set_seed(self._h, seed), "myrt_set_seed")


class Batch:
    """myrt_batch: physical-mode jobs over several scene contexts, rendered as
    one CUDA graph per frame. jobs: dicts with keys scene, width, height, spp,
    inverse_view, inverse_projection and optionally seed, max_depth, rr_start,
    fp64, env, sdf_marching_steps, sdf_marching_epsilon. The contexts must
    outlive the batch."""

    def __init__(self, contexts, jobs):
        self._L = _abi.lib()
        self._ctxs = list(contexts)
        self._jobs = [dict(j) for j in jobs]
        arr = (_abi.myrt_batch_job * len(jobs))()
        for k, j in enumerate(jobs):
            b = arr[k]
            b.scene, b.width, b.height, b.spp = j["scene"], j["width"], j["height"], j["spp"]
            b.seed, b.max_depth, b.rr_start = j.get("seed", 0), j.get("max_depth", 8), j.get("rr_start", 3)
            b.accum_fp64 = int(j.get("fp64", False))
            b.env_radiance[:] = [float(x) for x in j.get("env", (0.0, 0.0, 0.0))]
            b.sdf_marching_steps = j.get("sdf_marching_steps", 256)
            b.sdf_marching_epsilon = j.get("sdf_marching_epsilon", 1e-4)
            b.camera.inverse_view[:] = np.asarray(j["inverse_view"], np.float32).ravel().tolist()
            b.camera.inverse_projection[:] = np.asarray(j["inverse_projection"], np.float32).ravel().tolist()
        handles = (C.c_void_p * len(self._ctxs))(*[c._h.value for c in self._ctxs])
        self._h = C.c_void_p()
        rc = self._L.myrt_batch_create(handles, len(self._ctxs), arr, len(jobs), C.byref(self._h))
        self._ctxs[0]._check(rc, "myrt_batch_create")

    def _check(self, rc, what):
        self._ctxs[0]._check(rc, what)

    def close(self):
        if self._h:
            self._L.myrt_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return self._ctxs[0].stream

    def set_tuning(self, wave_paths: int = 0, blocks_per_sm: int = 0):
        self._check(self._L.myrt_batch_set_tuning(self._h, wave_paths, blocks_per_sm), "myrt_batch_set_tuning")

    def render(self):
        self._check(self._L.myrt_batch_render(self._h), "myrt_batch_render")

    def reset(self):
        self._check(self._L.myrt_batch_reset(self._h), "myrt_batch_reset")

    def read(self, job: int):
        """Accumulation (rgb sum, count) float32 [H, W, 4]; FP64 jobs: float64."""
        j = self._jobs[job]
        if j.get("fp64", False):
            out = np.empty((j["height"], j["width"], 4), np.float64)
            self._check(self._L.myrt_batch_read(self._h, job, None, out.ctypes.data), "myrt_batch_read")
        else:
            out = np.empty((j["height"], j["width"], 4), np.float32)
            self._check(self._L.myrt_batch_read(self._h, job, out.ctypes.data, None), "myrt_batch_read")
        return out

    def render_stats(self) -> dict:
        st = _abi.myrt_render_stats()
        self._check(self._L.myrt_batch_get_stats(self._h, C.byref(st)), "myrt_batch_get_stats")
        return dict(paths=st.paths, extension_rays=st.extension_rays, shadow_rays=st.shadow_rays)

    def info(self) -> dict:
        i = _abi.myrt_batch_info()
        self._check(self._L.myrt_batch_get_info(self._h, C.byref(i)), "myrt_batch_get_info")
        return {f: getattr(i, f) for f, _ in _abi.myrt_batch_info._fields_ if f != "pad"}
