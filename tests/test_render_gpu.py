"""Wavefront render ("reference shading") on the GPU vs the oracle's restated
passes, with the same host random stream.

Bar: bit-identical accumulation and display images. Closest hits, random draws
and every + and * are reproduced exactly (the device shading is compiled
without FMA contraction), and the transcendentals (sin, cos, atan, pow) are the
library's GLSL built-ins (glmath.hpp), which the oracle evaluates to the same
bits when switched to them (its default, the host libm, is what pins it to the
reference's own shaders compiled in oracle/_ref).
"""
import numpy as np
import pytest

import pyoracle as po
from myrt_b200.camera import look_at
from myrt_b200.scenes import heightfield, icosphere_field

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _library_builtins():
    with po.glsl_math(1):
        yield


def _compare(acc, ref):
    assert np.isfinite(acc).all()
    assert np.array_equal(acc[..., 3], ref[..., 3]), "per-pixel sample counts differ"
    same = (acc == ref).all(-1).mean()
    assert np.array_equal(acc, ref), f"only {same:.4f} of pixels bit-identical"
    return same


def test_reference_render_spheres(ctx):
    s = icosphere_field(n_spheres=24, subdiv=2, floor_cells=4, seed=4)
    ctx.upload_scene(**s)
    W, H = 96, 64
    iv, ip = look_at((0, 1, -4.5), (0, -0.3, 0), vfov_deg=50, aspect=W / H)
    ctx.set_seed(5489)
    ctx.render(iv, ip, W, H, num_bounces=4, frames=2)
    ctx.render(iv, ip, W, H, num_bounces=4, frames=2)  # accumulation continues
    assert ctx.sample_count() == 4
    acc, disp = ctx.read_accumulation(W, H)
    ref, ref_disp = po.render_reference(s, W, H, bounces=4, frames=4, inv_view=iv, inv_proj=ip, seed=5489)
    _compare(acc, ref)
    assert np.array_equal(disp, ref_disp)


def test_reference_render_default_bounces_heightfield(ctx):
    idx, pts = heightfield(32, seed=2)
    rng = np.random.default_rng(0)
    nrm = np.tile(np.array([[0.0, 1.0, 0.0]], np.float32), (pts.shape[0], 1))
    nrm[:, [0, 2]] = rng.normal(0, 0.05, (pts.shape[0], 2))
    mat = np.array([0, 0], np.int32)
    from myrt_b200.scenes import pbr_material

    mdata = pbr_material([0.7, 0.5, 0.3], ior=1.45, roughness=0.3, metallic=0.0, transmission=0.3)
    scene = dict(indices=idx, vertices=pts, normals=nrm, materials=mat, material_data=mdata)
    ctx.upload_scene(**scene)
    W, H = 64, 64
    iv, ip = look_at((0, 1.5, -2.5), (0, 0, 0), vfov_deg=60, aspect=1.0)
    ctx.set_seed(1234)
    ctx.render(iv, ip, W, H, num_bounces=10, frames=3)
    acc, _ = ctx.read_accumulation(W, H)
    ref, _ = po.render_reference(scene, W, H, bounces=10, frames=3, inv_view=iv, inv_proj=ip, seed=1234)
    _compare(acc, ref)


def test_accumulation_restarts(ctx):
    idx, pts = heightfield(8, seed=1)
    ctx.upload_scene(idx, pts)
    W, H = 32, 16
    iv, ip = look_at((0, 1.5, -2.5), (0, 0, 0), aspect=W / H)
    ctx.render(iv, ip, W, H, num_bounces=2, frames=3)
    assert ctx.sample_count() == 3
    iv2, _ = look_at((0.1, 1.5, -2.5), (0, 0, 0), aspect=W / H)
    ctx.render(iv2, ip, W, H, num_bounces=2, frames=1)  # camera change
    assert ctx.sample_count() == 1
    acc, _ = ctx.read_accumulation(W, H)
    assert np.all(acc[..., 3] == 1.0)
    ctx.render(iv2, ip, 16, 16, num_bounces=2, frames=2)  # resolution change
    assert ctx.sample_count() == 2
    ctx.reset_accumulation()
    assert ctx.sample_count() == 0


def test_reference_render_full_scene(ctx):
    """The 655,872-triangle scene at 128^2 with the reference's 10 bounces."""
    s = icosphere_field()
    ctx.upload_scene(**s)
    W, H = 128, 128
    iv, ip = look_at((0, 1, -4.5), (0, -0.3, 0), vfov_deg=50, aspect=1.0)
    ctx.set_seed(77)
    ctx.render(iv, ip, W, H, num_bounces=10, frames=2)
    acc, _ = ctx.read_accumulation(W, H)
    ref, _ = po.render_reference(s, W, H, bounces=10, frames=2, inv_view=iv, inv_proj=ip, seed=77)
    _compare(acc, ref)


def test_reference_render_mesh_and_sdf(ctx):
    """Meshes plus SDF drawables (a 64-primitive smooth-union field and a
    translated Menger sponge) in one frame: the trace pass takes the nearer of
    the mesh hit and the sphere-traced SDF hits, and shadow rays test both."""
    from myrt_b200 import sdf as S

    s = icosphere_field(n_spheres=12, subdiv=2, floor_cells=4, seed=6)
    lib = S.SdfLibrary()
    lib.add(S.random_sdf_field(64, k=0.1, seed=2, extent=0.6))
    lib.add(S.intersection(S.menger_fractal(3), S.box((0.9, 0.9, 0.9), 2)))
    up = np.array([[1, 0, 0, 0.0], [0, 1, 0, 0.2], [0, 0, 1, 0.5], [0, 0, 0, 1]])
    side = np.array([[0.4, 0, 0, 1.3], [0, 0.4, 0, -0.6], [0, 0, 0.4, -0.4], [0, 0, 0, 1]])
    dr = S.sdf_drawables([up, side], [0, 1])
    ctx.upload_scene(**s)
    ctx.upload_sdf(lib.instrs, lib.programs, lib.params, dr)
    W, H = 64, 48
    iv, ip = look_at((0, 1, -4.5), (0, -0.3, 0), vfov_deg=50, aspect=W / H)
    ctx.set_seed(31)
    ctx.render(iv, ip, W, H, num_bounces=4, frames=2, sdf_marching_steps=200, sdf_marching_epsilon=1e-4)
    acc, _ = ctx.read_accumulation(W, H)
    scene = dict(s, sdf=dict(lib=lib, drawables=dr, steps=200, eps=1e-4))
    ref, _ = po.render_reference(scene, W, H, bounces=4, frames=2, inv_view=iv, inv_proj=ip, seed=31)
    ctx.upload_sdf(np.zeros((0, 2)), np.zeros((0, 2)), np.zeros(0), np.zeros((0, 36)))
    _compare(acc, ref)
    # the SDF drawables are visible: the render differs from the meshes-only one
    ref0, _ = po.render_reference(s, W, H, bounces=4, frames=2, inv_view=iv, inv_proj=ip, seed=31)
    assert np.abs(ref0[..., :3] - ref[..., :3]).max(-1).mean() > 1e-2


def _textured_heightfield():
    """32 x 32 height field with uvs from xz, two materials: one with an albedo
    texture (slot 0, a checker in linear [0, 1]), one plain."""
    from myrt_b200.scenes import pbr_material

    idx, pts = heightfield(32, seed=3)
    uvs = np.stack([(pts[:, 0] + 1) * 1.5, (pts[:, 2] + 1) * 1.5], 1).astype(np.float32)  # repeats past 1
    m0 = pbr_material([0.7, 0.5, 0.3], ior=1.5, roughness=0.6)
    m0[5] = np.array([1], np.uint32).view(np.float32)[0]  # handle (slot 0 + 1, 0)
    m1 = pbr_material([0.3, 0.6, 0.8], ior=1.5, roughness=0.3, metallic=1.0)
    mdata = np.concatenate([m0, m1])
    from myrt_b200._abi import myrt_drawable

    n = idx.size
    dr = (myrt_drawable * 2)()
    eye = np.eye(4, dtype=np.float32).ravel().tolist()
    for k in range(2):
        dr[k].transformation[:] = eye
        dr[k].inverse_transformation[:] = eye
        dr[k].points_base_index = 0
        dr[k].material_index = k
    half = (n // 6) * 3
    dr[0].indices_base_index, dr[0].index_count = 0, half
    dr[1].indices_base_index, dr[1].index_count = half, n - half
    scene = dict(indices=idx, vertices=pts, uvs=uvs, drawables=dr, materials=np.array([[0, 0], [0, 7]], np.int32),
                 material_data=mdata)
    g = np.indices((8, 8)).sum(0) % 2
    checker = np.zeros((8, 8, 4), np.float32)
    checker[..., 0] = np.where(g, 0.9, 0.2)
    checker[..., 1] = np.where(g, 0.8, 0.3)
    checker[..., 2] = np.where(g, 0.1, 0.7)
    checker[..., 3] = 1.0
    return scene, checker


def _bokeh_mask():
    """16 x 16 ring with a dark centre: draws inside it trigger bokeh_get's retries."""
    y, x = np.mgrid[0:16, 0:16]
    r = np.hypot(x - 7.5, y - 7.5) / 8.0
    v = np.where((r > 0.35) & (r < 0.95), 1.0, 0.0).astype(np.float32)
    m = np.zeros((16, 16, 4), np.float32)
    m[..., 0], m[..., 1], m[..., 2], m[..., 3] = v, 0.8 * v, 0.6 * v, 1.0
    return m


def _cubemap(size=16):
    f = np.zeros((6, size, size, 4), np.float32)
    s = np.linspace(0, 1, size, dtype=np.float32)
    for k in range(6):
        f[k, ..., 0] = 0.2 + 0.1 * k + 0.5 * s[None, :]
        f[k, ..., 1] = 0.3 + 0.4 * s[:, None]
        f[k, ..., 2] = 0.9 - 0.1 * k
        f[k, ..., 3] = 1.0
    return f


def test_reference_render_textures_cubemap_dof(ctx):
    """Albedo textures (material handle = slot + 1), the environment cube map and
    depth of field with a bokeh mask, against the oracle's restated passes."""
    scene, checker = _textured_heightfield()
    ctx.upload_scene(**scene)
    ctx.upload_texture(0, checker, wrap=0)
    ctx.upload_texture(1, _bokeh_mask(), wrap=0)
    cube = _cubemap()
    ctx.upload_cubemap(cube)
    try:
        W, H = 80, 60
        iv, ip = look_at((0, 1.2, -2.5), (0, 0, 0), vfov_deg=55, aspect=W / H)
        ctx.set_seed(777)
        ctx.render(iv, ip, W, H, num_bounces=4, frames=3, dof=True, lens_size=(0.2, 0.15), focus=2.4, bokeh_slot=1)
        acc, _ = ctx.read_accumulation(W, H)
        ref, _ = po.render_reference(scene, W, H, bounces=4, frames=3, inv_view=iv, inv_proj=ip, seed=777,
                                     textures=[(checker, 0), (_bokeh_mask(), 0)], cubemap=cube, dof=True,
                                     lens_size=(0.2, 0.15), focus=2.4, bokeh_slot=1)
        _compare(acc, ref)
        # without the extras the image changes (the features are in use)
        ref_plain, _ = po.render_reference(scene, W, H, bounces=4, frames=3, inv_view=iv, inv_proj=ip, seed=777)
        assert np.abs(ref_plain[..., :3] - ref[..., :3]).mean() > 1e-2
    finally:
        ctx.upload_texture(0, None)
        ctx.upload_texture(1, None)
        ctx.upload_cubemap(None)


@pytest.mark.parametrize("frames_in_flight", [1, 2, 3])
def test_frames_in_flight_do_not_change_the_images(ctx, frames_in_flight):
    """Frames of one call rendered together (tuning ref_frames), in batches that
    leave a remainder, give the images of frames rendered one at a time -- and
    of the oracle's sequential frames."""
    s = icosphere_field(n_spheres=16, subdiv=2, floor_cells=4, seed=6)
    ctx.upload_scene(**s)
    W, H = 80, 48
    iv, ip = look_at((0, 1, -4.5), (0, -0.3, 0), vfov_deg=50, aspect=W / H)
    try:
        ctx.set_tuning(ref_frames=frames_in_flight)
        ctx.reset_accumulation()
        ctx.set_seed(321)
        ctx.render(iv, ip, W, H, num_bounces=5, frames=5)
        ctx.render(iv, ip, W, H, num_bounces=5, frames=2)
        acc, disp = ctx.read_accumulation(W, H)
    finally:
        ctx.set_tuning()
    assert ctx.sample_count() == 7
    ref, ref_disp = po.render_reference(s, W, H, bounces=5, frames=7, inv_view=iv, inv_proj=ip, seed=321)
    _compare(acc, ref)
    assert np.array_equal(disp, ref_disp)


def test_sorted_trace_passes_do_not_change_the_images(ctx):
    """16 frames in flight of 256 x 256 fill 1 Mi ray slots, so the first two
    trace passes run in the sorted visiting order (trace_order 0); every pass
    sorted (2) and none (1) give the same bits."""
    s = icosphere_field(n_spheres=64, subdiv=2, floor_cells=8, seed=8)
    ctx.upload_scene(**s)
    W = H = 256
    iv, ip = look_at((0, 1, -4.5), (0, -0.3, 0), vfov_deg=50, aspect=1.0)
    out = []
    try:
        for order in (1, 0, 2):
            ctx.set_tuning(trace_order=order)
            ctx.reset_accumulation()
            ctx.set_seed(99)
            ctx.render(iv, ip, W, H, num_bounces=3, frames=16)
            out.append(ctx.read_accumulation(W, H))
    finally:
        ctx.set_tuning()
    for acc, disp in out[1:]:
        assert np.array_equal(acc, out[0][0]) and np.array_equal(disp, out[0][1])
    assert out[0][0][..., 3].min() == 16
