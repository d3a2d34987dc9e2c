"""ctypes declarations of the C ABI in include/myrt_cuda.h.

The shared library is built in-tree (myrt_b200/build.py) and loaded from the
package directory. There is no fallback: if the library is missing, importing
the package raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libmyrt_b200.so"

MYRT_OK = 0
MYRT_ERR_INVALID_ARGUMENT = -1
MYRT_ERR_CUDA = -2
MYRT_ERR_OUT_OF_MEMORY = -3
MYRT_ERR_NO_SCENE = -4
MYRT_ERR_UNSUPPORTED = -5
MYRT_ERR_DEVICE_ABORT = -6
MYRT_ERR_INTERNAL = -7

ISECT_REFERENCE = 0
ISECT_WATERTIGHT = 1


class myrt_device_opts(C.Structure):
    _fields_ = [("device", C.c_int), ("flags", C.c_uint32)]


class myrt_drawable(C.Structure):
    _fields_ = [("transformation", C.c_float * 16), ("inverse_transformation", C.c_float * 16),
                ("bvh_node_base_index", C.c_uint32), ("bvh_index_base_index", C.c_uint32),
                ("indices_base_index", C.c_uint32), ("points_base_index", C.c_uint32), ("index_count", C.c_uint32),
                ("material_index", C.c_int32), ("geometry_index", C.c_int32), ("pad", C.c_int32)]


class myrt_material_ref(C.Structure):
    _fields_ = [("id", C.c_int32), ("offset", C.c_int32)]


class myrt_scene_view(C.Structure):
    _fields_ = [("indices", C.c_void_p), ("index_count", C.c_size_t), ("vertices", C.c_void_p),
                ("vertex_count", C.c_size_t), ("normals", C.c_void_p), ("uvs", C.c_void_p),
                ("drawables", C.c_void_p), ("drawable_count", C.c_size_t), ("materials", C.c_void_p),
                ("material_count", C.c_size_t), ("material_data", C.c_void_p), ("material_data_count", C.c_size_t)]


class myrt_bvh_info(C.Structure):
    _fields_ = [("triangles", C.c_uint64), ("binary_nodes", C.c_uint64), ("wide_nodes", C.c_uint64),
                ("leaf_slots", C.c_uint64), ("binary_depth", C.c_int32), ("wide_depth", C.c_int32),
                ("max_leaf_size", C.c_int32), ("pad", C.c_int32), ("build_seconds", C.c_double),
                ("node_bytes", C.c_uint64), ("triangle_bytes", C.c_uint64)]


class myrt_camera(C.Structure):
    _fields_ = [("inverse_view", C.c_float * 16), ("inverse_projection", C.c_float * 16)]


class myrt_render_params(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("num_bounces", C.c_int32), ("frames", C.c_uint32),
                ("shading", C.c_int32), ("flags", C.c_uint32), ("sdf_marching_steps", C.c_int32),
                ("sdf_marching_epsilon", C.c_float), ("max_depth", C.c_int32), ("rr_start", C.c_int32),
                ("seed", C.c_uint32), ("accum_fp64", C.c_uint32), ("env_radiance", C.c_float * 3),
                ("wave_paths", C.c_uint32), ("dof_active", C.c_int32), ("lens_size", C.c_float * 2),
                ("focus", C.c_float), ("bokeh_texture", C.c_int32)]


class myrt_forward_params(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("view", C.c_float * 16),
                ("projection", C.c_float * 16), ("random_seed", C.c_uint32), ("shadow_size", C.c_uint32),
                ("custom_shadow", C.c_int32), ("shadow_view", C.c_float * 16),
                ("shadow_projection", C.c_float * 16)]


class myrt_pp_pass(C.Structure):
    _fields_ = [("op", C.c_int32), ("i", C.c_int32 * 3), ("p", C.c_float * 4)]


class myrt_image(C.Structure):
    _fields_ = [("rgba", C.c_void_p), ("width", C.c_uint32), ("height", C.c_uint32)]


PP_DENOISE, PP_BLUR, PP_CUTOFF, PP_ADD, PP_TONEMAP, PP_FXAA, PP_SCALE = range(7)


class myrt_render_stats(C.Structure):
    _fields_ = [("paths", C.c_uint64), ("extension_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("reserved", C.c_uint64)]


class myrt_guide_params(C.Structure):
    _fields_ = [("fraction", C.c_float), ("learning_rate", C.c_float), ("train_steps", C.c_uint32),
                ("batch", C.c_uint32), ("train", C.c_uint32), ("warmup_waves", C.c_uint32), ("seed", C.c_uint32),
                ("weight_clamp", C.c_float), ("target", C.c_uint32), ("reserved", C.c_uint32)]


class myrt_guide_stats(C.Structure):
    _fields_ = [("adam_steps", C.c_uint64), ("waves", C.c_uint64), ("waves_trained", C.c_uint64),
                ("last_samples", C.c_uint32), ("last_loss", C.c_float), ("last_weight_sum", C.c_float),
                ("pad", C.c_uint32)]


GUIDE_PARAM_COUNT = 16640


class myrt_batch_job(C.Structure):
    _fields_ = [("scene", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32),
                ("seed", C.c_uint32), ("max_depth", C.c_int32), ("rr_start", C.c_int32), ("accum_fp64", C.c_uint32),
                ("env_radiance", C.c_float * 3), ("sdf_marching_steps", C.c_int32),
                ("sdf_marching_epsilon", C.c_float), ("pad", C.c_uint32), ("camera", myrt_camera)]


class myrt_batch_info(C.Structure):
    _fields_ = [("waves", C.c_uint32), ("max_wave_paths", C.c_uint32), ("paths_per_frame", C.c_uint64),
                ("graph_nodes", C.c_uint32), ("wave_paths", C.c_uint32), ("blocks_per_sm", C.c_uint32),
                ("pad", C.c_uint32)]


class myrt_area_light(C.Structure):
    _fields_ = [("corner", C.c_float * 3), ("edge_u", C.c_float * 3), ("edge_v", C.c_float * 3),
                ("emission", C.c_float * 3)]


class myrt_sdf_view(C.Structure):
    _fields_ = [("instrs", C.c_void_p), ("instr_count", C.c_size_t), ("programs", C.c_void_p),
                ("program_count", C.c_size_t), ("params", C.c_void_p), ("param_count", C.c_size_t),
                ("drawables", C.c_void_p), ("drawable_count", C.c_size_t)]


class myrt_tuning(C.Structure):
    _fields_ = [("trace_persistent", C.c_uint32), ("refill", C.c_uint32), ("blocks_per_sm", C.c_uint32),
                ("trace_min_blocks", C.c_uint32), ("trace_unit_steps", C.c_uint32), ("wave_paths", C.c_uint32),
                ("pt_blocks_per_sm", C.c_uint32), ("trace_smem_stack", C.c_uint32),
                ("bvh_builder", C.c_uint32), ("trace_order", C.c_uint32),
                ("sdf_cells", C.c_uint32), ("guide_poll_limit", C.c_uint32), ("guide_stall_test", C.c_uint32),
                ("instancing", C.c_uint32), ("pt_grid", C.c_uint32),
                ("ref_frames", C.c_uint32)]


SHADE_REFERENCE = 0
SHADE_PHYSICAL = 1
SHADE_GUIDED = 2

P = C.c_void_p
SZ = C.c_size_t
U32 = C.c_uint32
I = C.c_int

# name -> (restype, argtypes)
SIGNATURES = {
    "myrt_bvh8_build": (I, [P, SZ, C.POINTER(P)]),
    "myrt_bvh8_get_info": (I, [P, C.POINTER(myrt_bvh_info)]),
    "myrt_bvh8_copy": (I, [P, P, P]),
    "myrt_bvh8_free": (I, [P]),
    "myrt_ctx_create": (I, [C.POINTER(myrt_device_opts), C.POINTER(P)]),
    "myrt_ctx_destroy": (I, [P]),
    "myrt_get_last_error": (I, [P, C.c_char_p, SZ]),
    "myrt_get_stream": (I, [P, C.POINTER(P)]),
    "myrt_set_tuning": (I, [P, C.POINTER(myrt_tuning)]),
    "myrt_get_tuning": (I, [P, C.POINTER(myrt_tuning)]),
    "myrt_scene_upload": (I, [P, C.POINTER(myrt_scene_view)]),
    "myrt_scene_bvh_info": (I, [P, C.POINTER(myrt_bvh_info)]),
    "myrt_sdf_upload": (I, [P, C.POINTER(myrt_sdf_view)]),
    "myrt_trace_sdf": (I, [P, P, U32, C.c_int32, C.c_float, I, P, P]),
    "myrt_trace_closest": (I, [P, P, U32, P, I]),
    "myrt_trace_closest_device": (I, [P, P, U32, P, I, P]),
    "myrt_trace_any": (I, [P, P, U32, P, I]),
    "myrt_trace_any_device": (I, [P, P, U32, P, I, P]),
    "myrt_trace_closest_stats_device": (I, [P, P, U32, P, P, P, I, P]),
    "myrt_render": (I, [P, C.POINTER(myrt_camera), C.POINTER(myrt_render_params)]),
    "myrt_read_accumulation": (I, [P, P, P]),
    "myrt_read_accumulation_f64": (I, [P, P]),
    "myrt_set_area_lights": (I, [P, P, U32]),
    "myrt_get_render_stats": (I, [P, C.POINTER(myrt_render_stats)]),
    "myrt_batch_create": (I, [P, U32, P, U32, C.POINTER(P)]),
    "myrt_batch_set_tuning": (I, [P, U32, U32]),
    "myrt_batch_render": (I, [P]),
    "myrt_batch_read": (I, [P, U32, P, P]),
    "myrt_batch_reset": (I, [P]),
    "myrt_batch_get_info": (I, [P, C.POINTER(myrt_batch_info)]),
    "myrt_batch_get_stats": (I, [P, C.POINTER(myrt_render_stats)]),
    "myrt_scene_copy_bvh": (I, [P, P, P]),
    "myrt_texture_upload": (I, [P, U32, P, U32, U32, U32]),
    "myrt_cubemap_upload": (I, [P, P, U32]),
    "myrt_forward_run": (I, [P, C.POINTER(myrt_forward_params)]),
    "myrt_begin_samples": (I, [P, U32]),
    "myrt_render_size": (I, [P, C.POINTER(U32), C.POINTER(U32)]),
    "myrt_render_buffer_f64": (I, [P, C.POINTER(P)]),
    "myrt_forward_read": (I, [P, U32, U32, U32, P, P, P, P]),
    "myrt_forward_buffers": (I, [P, C.POINTER(P), C.POINTER(P), C.POINTER(P), C.POINTER(P)]),
    "myrt_forward_default_shadow": (I, [P, P]),
    "myrt_scene_set_transforms": (I, [P, P, C.c_size_t]),
    "myrt_post_pass": (I, [P, C.POINTER(myrt_pp_pass), C.POINTER(myrt_image), C.POINTER(myrt_image),
                           C.POINTER(myrt_image), P]),
    "myrt_set_phase_timing": (I, [P, C.c_int]),
    "myrt_get_phase_times": (I, [P, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_uint64)]),
    "myrt_batch_destroy": (I, [P]),
    "myrt_guide_configure": (I, [P, C.POINTER(myrt_guide_params)]),
    "myrt_guide_get_config": (I, [P, C.POINTER(myrt_guide_params)]),
    "myrt_guide_reset": (I, [P]),
    "myrt_guide_get_params": (I, [P, P]),
    "myrt_guide_set_params": (I, [P, P]),
    "myrt_guide_eval": (I, [P, P, U32, P]),
    "myrt_guide_gradients": (I, [P, P, U32, P, P]),
    "myrt_guide_train": (I, [P, P, U32, U32, P]),
    "myrt_guide_get_stats": (I, [P, C.POINTER(myrt_guide_stats)]),
    "myrt_render_buffers": (I, [P, C.POINTER(P), C.POINTER(P)]),
    "myrt_reset_accumulation": (I, [P]),
    "myrt_sample_count": (I, [P, C.POINTER(C.c_uint32)]),
    "myrt_set_seed": (I, [P, C.c_uint32]),
    "myrt_render_noalloc": (I, [P, C.POINTER(myrt_camera), C.POINTER(myrt_render_params), C.c_uint32, P, P, P]),
    "myrt_sync": (I, [P]),
    "myrt_glsl_builtins": (I, [P, I, P, P, U32, P]),
}

_lib = None


def lib() -> C.CDLL:
    """Load libmyrt_b200.so (once). Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m myrt_b200.build` "
                               "(or __graft_entry__.build()); there is no CPU fallback")
        h = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _lib = h
    return _lib
