"""Forward (raster preview) renderer on the GPU vs the oracle's restated passes.

Bar: bit-exact everywhere -- the visibility keys (24-bit depth, triangle), the
G-buffer (half bits), the shadow map and the resolved image. The rasteriser
and the attribute interpolation use only + * / and sqrt, each rounded
separately on both sides; the resolve's sin / cos / pow are the library's GLSL
built-ins (glmath.hpp), which the oracle evaluates to the same bits when
switched to them (its default, the host libm, pins it to the reference's
compiled resolve.frag).
"""
import numpy as np
import pytest

import pyoracle as po
from myrt_b200 import forward_default_shadow
from myrt_b200.camera import view_projection
from myrt_b200.scenes import icosphere_field

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _library_builtins():
    with po.glsl_math(1):
        yield


def _same(a, b):
    return np.array_equal(a, b, equal_nan=True)


def _close(res, ref):
    assert np.isfinite(res).all()
    same = (res == ref).all(-1).mean()
    assert np.array_equal(res, ref), f"only {same:.4f} of pixels bit-identical"


def _run(ctx, s, W, H, view, proj, seed, S, sv, sp, custom=True, textures=None):
    if custom:
        ctx.forward_render(view, proj, W, H, seed, S, sv, sp)
    else:
        ctx.forward_render(view, proj, W, H, seed, S)
    got = ctx.forward_read(W, H, S)
    ref = po.forward_render(s, W, H, view, proj, seed, S, sv, sp, textures=textures)
    return got, ref


def test_forward_matches_oracle_instanced_spheres(ctx):
    s = icosphere_field(n_spheres=24, subdiv=2, floor_cells=4, seed=4)
    ctx.upload_scene(**s)
    W, H, S = 96, 64, 256
    view, proj = view_projection((0, 1.0, -4.5), (0, -0.3, 0), vfov_deg=50, aspect=W / H, near=0.05, far=50.0)
    sv, sp = view_projection((2.0, 6.0, 3.0), (0, -1.2, 0), vfov_deg=40, aspect=1.0, near=1.0, far=30.0)
    got, ref = _run(ctx, s, W, H, view, proj, 12345, S, sv, sp)
    assert np.array_equal(got["visibility"], ref["visibility"])
    assert _same(got["gbuffer"], ref["gbuffer"])
    assert _same(got["shadow_map"], ref["shadow_map"])
    fg = got["visibility"] != np.uint64(0xFFFFFFFFFFFFFFFF)
    assert 0.2 < fg.mean() < 0.95
    _close(got["result"], ref["result"])


def test_forward_near_plane_default_light_and_texture(ctx):
    """Eye inside the scene: the floor reaches behind it (corners with w <= 0,
    whole-viewport boxes); the reference's light camera at 2048^2; an albedo
    texture on the floor material."""
    s = icosphere_field(n_spheres=12, subdiv=2, floor_cells=6, seed=9)
    ny = s["material_data"].reshape(-1, 7).copy()
    ny[0, 5] = np.array([1], np.uint32).view(np.float32)[0]  # floor: texture slot 0 -> handle (1, 0)
    ny[0, 6] = 0.0
    s["material_data"] = ny.ravel()
    tex = np.zeros((16, 16, 4), np.float32)
    tex[..., 0] = (np.arange(16)[None, :] // 4 % 2) * 0.8 + 0.1
    tex[..., 1] = (np.arange(16)[:, None] // 4 % 2) * 0.6 + 0.2
    tex[..., 2], tex[..., 3] = 0.4, 1.0
    ctx.upload_scene(**s)
    ctx.upload_texture(0, tex, wrap=0)
    W, H = 80, 60
    view, proj = view_projection((0.2, -0.9, -2.2), (0.0, -0.6, 1.0), vfov_deg=70, aspect=W / H, near=0.02, far=40)
    sv, sp = forward_default_shadow()
    got, ref = _run(ctx, s, W, H, view, proj, 77, 2048, sv, sp, custom=False, textures=[(tex, 0)])
    assert np.array_equal(got["visibility"], ref["visibility"])
    assert _same(got["gbuffer"], ref["gbuffer"])
    assert _same(got["shadow_map"], ref["shadow_map"])
    _close(got["result"], ref["result"])
    ctx.upload_texture(0, None)


def test_forward_follows_instance_moves(ctx):
    """After myrt_scene_set_transforms the rasteriser draws the re-baked
    triangles: the same images as uploading the moved scene."""
    s = icosphere_field(n_spheres=8, subdiv=2, floor_cells=2, seed=5)
    ctx.upload_scene(**s)
    W, H, S = 64, 48, 128
    view, proj = view_projection((0, 0.5, -4.0), (0, -0.3, 0), vfov_deg=55, aspect=W / H)
    sv, sp = view_projection((1.0, 5.0, 2.0), (0, -1.2, 0), vfov_deg=45, aspect=1.0, near=1.0, far=20.0)
    d = s["drawables"]
    for k in range(4):
        d[k].transformation[12] += 0.3  # translation only: the normal matrix stays
    ctx.set_transforms(d)
    ctx.forward_render(view, proj, W, H, 5, S, sv, sp)
    moved = ctx.forward_read(W, H, S)
    ref = po.forward_render(s, W, H, view, proj, 5, S, sv, sp)
    assert np.array_equal(moved["visibility"], ref["visibility"])
    assert _same(moved["gbuffer"], ref["gbuffer"])


def test_forward_empty_view_is_background(ctx):
    s = icosphere_field(n_spheres=2, subdiv=1, floor_cells=1, seed=1)
    ctx.upload_scene(**s)
    W, H = 32, 24
    view, proj = view_projection((0, 0, -5), (0, 0, -10), vfov_deg=40, aspect=W / H)  # looking away
    sv, sp = forward_default_shadow()
    got, ref = _run(ctx, s, W, H, view, proj, 3, 64, sv, sp)
    assert (got["visibility"] == np.uint64(0xFFFFFFFFFFFFFFFF)).all()
    assert _same(got["result"], ref["result"])
    assert (got["result"][..., 3] == 1).all()


def test_forward_rejects_bad_sizes(ctx):
    s = icosphere_field(n_spheres=1, subdiv=1, floor_cells=1, seed=1)
    ctx.upload_scene(**s)
    view, proj = view_projection((0, 0, -5), (0, 0, 0))
    from myrt_b200 import MyrtError
    with pytest.raises(MyrtError):
        ctx.forward_render(view, proj, 0, 16, 1)
    with pytest.raises(MyrtError):
        ctx.forward_render(view, proj, 16, 16, 1, shadow_size=20000)
    ctx.forward_render(view, proj, 16, 12, 1, shadow_size=64)
    with pytest.raises(MyrtError):  # host arrays made for another size are refused
        ctx.forward_read(16, 12, 2048)
    with pytest.raises(MyrtError):
        ctx.forward_result(12, 16, 64)
    assert ctx.forward_result(16, 12, 64).shape == (12, 16, 4)
