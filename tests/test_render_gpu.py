"""Wavefront render ("reference shading") on the GPU vs the oracle's restated
passes, with the same host random stream.

Tolerance: closest hits, random draws and every + and * are reproduced exactly
(the device shading is compiled without FMA contraction); only CUDA's sinf,
cosf, atanf and powf differ from the host's libm by an ulp or two. A path is
therefore either identical up to those last bits, or diverges at a discrete
decision that such a bit flips (Russian roulette, lobe choice, a grazing hit).
Bar, per test: per-pixel sample counts equal; at least 97 % of pixels within
1e-3 relative (max over rgb); image mean within 1 %.
"""
import numpy as np
import pytest

import pyoracle as po
from myrt_b200.camera import look_at
from myrt_b200.scenes import heightfield, icosphere_field

pytestmark = pytest.mark.gpu


def _compare(acc, ref, frac_bar=0.97, mean_bar=0.01):
    assert np.isfinite(acc).all()
    assert np.array_equal(acc[..., 3], ref[..., 3]), "per-pixel sample counts differ"
    rel = np.abs(acc[..., :3] - ref[..., :3]) / (1e-3 + np.abs(ref[..., :3]))
    close = (rel.max(-1) <= 1e-3).mean()
    m, mr = acc[..., :3].mean(), ref[..., :3].mean()
    assert close >= frac_bar, f"only {close:.4f} of pixels within 1e-3"
    assert abs(m - mr) / mr < mean_bar, (m, mr)
    return close


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
    assert np.abs(disp - ref_disp).mean() < 0.01


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
