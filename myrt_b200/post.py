"""Post-processing on device images (torch float32 [H, W, 4] tensors on the
context's GPU): the reference's passes (src/pt/pp_*.comp through
myrt_post_pass) and its compositions from src/pathtracer/post_process.cpp
(blur2d, bloom) and src/main.cpp:840-875 (the per-frame chain: down-scale,
bloom, filmic tonemap, FXAA). Every pass writes a new tensor whose values are
half-precision representable, like the reference's RGBA16F targets."""
from __future__ import annotations

import ctypes as C

from . import _abi


def _image(t) -> _abi.myrt_image:
    assert t.is_cuda and t.dtype.is_floating_point and t.dim() == 3 and t.shape[2] == 4 and t.is_contiguous()
    return _abi.myrt_image(t.data_ptr(), t.shape[1], t.shape[0])


def run(ctx, op: int, img, i=(0, 0, 0), p=(0.0, 0.0, 0.0, 0.0), overlay=None, out_size=None, out=None, stream=None):
    """One myrt_post_pass on torch's current stream (or `stream`, a raw CUDA
    stream handle), ordered with the tensors' producers and consumers;
    out_size (h, w) for the scale pass. Returns the output tensor."""
    import torch

    if stream is None:
        stream = torch.cuda.current_stream(img.device).cuda_stream or 1  # 1 = cudaStreamLegacy
    h, w = out_size if out_size else img.shape[:2]
    if out is None:
        out = torch.empty((h, w, 4), dtype=torch.float32, device=img.device)
    ps = _abi.myrt_pp_pass(op, (C.c_int32 * 3)(*i), (C.c_float * 4)(*p))
    ii, oo = _image(img), _image(out)
    ov = _image(overlay) if overlay is not None else None
    ctx._check(ctx._L.myrt_post_pass(ctx._h, C.byref(ps), C.byref(ii), C.byref(ov) if ov else None, C.byref(oo),
                                     C.c_void_p(stream) if stream else None), "myrt_post_pass")
    return out


def denoise(ctx, img, exponent: float = 10.0, strength: float = 0.05):
    """denoise (post_process.hpp defaults exponent 10, strength 0.05)."""
    return run(ctx, _abi.PP_DENOISE, img, p=(exponent, strength, 0.0, 0.0))


def blur(ctx, img, direction: int, step: float = 1.25):
    return run(ctx, _abi.PP_BLUR, img, i=(direction, 0, 0), p=(step, 0.0, 0.0, 0.0))


def blur2d(ctx, img, step: float = 1.25):
    """blur2d::process (post_process.cpp:188-195): x, then y."""
    return blur(ctx, blur(ctx, img, 0, step), 1, step)


def cutoff(ctx, img, value=(1.0, 1.0, 1.0, 1.0), leave_above: bool = True):
    return run(ctx, _abi.PP_CUTOFF, img, i=(int(leave_above), 0, 0), p=tuple(float(v) for v in value))


def add(ctx, img, overlay, factor: float = 1.0):
    return run(ctx, _abi.PP_ADD, img, p=(factor, 0.0, 0.0, 0.0), overlay=overlay)


def tonemap(ctx, img, alpha_one: bool = True):
    """Filmic tonemap; alpha_one as the OpenCL kernel main.cpp runs."""
    return run(ctx, _abi.PP_TONEMAP, img, i=(int(alpha_one), 0, 0))


def fxaa(ctx, img):
    return run(ctx, _abi.PP_FXAA, img)


def scaled_size(h: int, w: int, factor: float) -> tuple[int, int]:
    """linear_scale's target size: width * factor in float, truncated."""
    import numpy as np

    f = np.float32(factor)
    return int(np.float32(h) * f), int(np.float32(w) * f)


def scale(ctx, img, factor: float):
    return run(ctx, _abi.PP_SCALE, img, out_size=scaled_size(img.shape[0], img.shape[1], factor))


def bloom(ctx, img, blur_step: float = 1.25, texture_scaling: float = 2.0, overlay_factor: float = 0.3):
    """bloom::process (post_process.cpp:170-186): cutoff twice, scale down,
    blur2d, scale up, add to the input."""
    r = cutoff(ctx, img)
    r = cutoff(ctx, r)
    r = scale(ctx, r, 1.0 / texture_scaling)
    r = blur2d(ctx, r, blur_step)
    r = scale(ctx, r, texture_scaling)
    return add(ctx, img, r, overlay_factor)


def frame(ctx, img, super_sampling: float = 1.0, blur_step: float = 1.25, texture_scaling: float = 2.0,
          overlay_factor: float = 0.3):
    """The per-frame chain of main.cpp:840-875: down-scale by 1 / super_sampling,
    bloom, filmic tonemap (alpha 1), FXAA."""
    r = scale(ctx, img, 1.0 / super_sampling)
    r = bloom(ctx, r, blur_step, texture_scaling, overlay_factor)
    r = tonemap(ctx, r, alpha_one=True)
    return fxaa(ctx, r)
