"""Physical shading mode: GGX + Lambert BSDF, NEE with the power heuristic to
parallelogram lights, Russian roulette, counter-based random numbers.

The device kernels use only +, -, *, /, sqrt and comparisons (sin / cos come
from a polynomial of the project's own), compiled without FMA contraction, and
the oracle restates them with -ffp-contract=off: images are compared BIT FOR
BIT. Physics checks on the oracle: the direct lighting of a Lambertian plane
under a small light matches the analytic irradiance, and the environment
furnace returns the environment radiance.
"""
import numpy as np
import pytest

import pyoracle as po
from myrt_b200.camera import look_at
from myrt_b200.scenes import area_light, heightfield, icosphere_field, icosphere_field_lit, pbr_material


def _plane(size=2.0, rough=1.0, albedo=0.8, ior=1.0, metallic=0.0):
    idx = np.array([0, 1, 2, 0, 2, 3], np.uint32)
    h = size / 2
    pts = np.array([[-h, 0, -h], [h, 0, -h], [h, 0, h], [-h, 0, h]], np.float32)
    mats = np.array([[0, 0]], np.int32)
    mdata = pbr_material([albedo] * 3, ior=ior, roughness=rough, metallic=metallic)
    return dict(indices=idx, vertices=pts, materials=mats, material_data=mdata)


def test_oracle_env_furnace():
    s = _plane()
    s["vertices"] = s["vertices"] + np.float32([0, -50, 0])  # out of view
    iv, ip = look_at((0, 1, -3), (0, 1, 0), vfov_deg=30, aspect=1.0)
    acc = po.render_physical(s, 8, 8, 4, iv, ip, lights=None, env=(0.25, 0.5, 1.0))
    assert np.array_equal(acc[..., 3], np.full((8, 8), 4.0, np.float32))
    assert np.array_equal(acc[..., :3] / 4, np.broadcast_to(np.float32([0.25, 0.5, 1.0]), (8, 8, 3)))


def test_oracle_direct_light_matches_irradiance():
    """Lambertian plane (ior 1 -> F0 = 0, roughness 1) under a 0.1 x 0.1 light at
    height 1, emission 20, camera looking straight down at the spot below: the
    one-bounce estimate (NEE + BSDF hits of the light, power-heuristic MIS)
    converges to (albedo / pi) * Le * A / d^2."""
    s = _plane(albedo=0.8)
    lights = area_light((0.0, 1.0, 0.0), 0.1, 20.0)[None]
    iv, ip = look_at((0.0, 0.5, 0.0001), (0, 0, 0), vfov_deg=1.0, aspect=1.0, up=(0, 0, 1))
    acc = po.render_physical(s, 4, 4, 4096, iv, ip, lights=lights, max_depth=1, rr_start=99, seed=3)
    est = acc[..., :3].sum() / acc[..., 3].sum() / 3
    expect = 0.8 / np.pi * 20.0 * 0.01 / 1.0
    # Schlick's grazing term adds a little at F0 = 0; the light's finite size removes ~1 %
    assert abs(est - expect) / expect < 0.03, (est, expect)


def test_oracle_depth_zero_sees_only_emitters():
    s, lights = icosphere_field_lit(n_spheres=8, subdiv=1, floor_cells=2, seed=1)
    iv, ip = look_at((0, 0.5, -3), (0, 1.0, 0), vfov_deg=60, aspect=1.0)
    acc = po.render_physical(s, 16, 16, 2, iv, ip, lights=lights, max_depth=0)
    v = acc[..., :3]
    assert set(np.unique(v)).issubset({0.0, 40.0})  # 2 samples x emission 20 where the light is seen


@pytest.mark.gpu
@pytest.mark.parametrize("wave", [0, 2048])
def test_physical_bit_exact_spheres(ctx, wave):
    s, lights = icosphere_field_lit(n_spheres=24, subdiv=2, floor_cells=4, seed=4)
    ctx.upload_scene(**s)
    ctx.set_area_lights(lights)
    W, H = 48, 32
    iv, ip = look_at((0, 1, -4.5), (0, -0.3, 0), vfov_deg=50, aspect=W / H)
    ctx.render_physical(iv, ip, W, H, spp=3, max_depth=8, rr_start=3, seed=11, env=(0.05, 0.06, 0.08),
                        wave_paths=wave)
    ctx.render_physical(iv, ip, W, H, spp=2, max_depth=8, rr_start=3, seed=11, env=(0.05, 0.06, 0.08),
                        wave_paths=wave)
    assert ctx.sample_count() == 5
    acc, disp = ctx.read_accumulation(W, H)
    ref = po.render_physical(s, W, H, 5, iv, ip, lights, env=(0.05, 0.06, 0.08), max_depth=8, rr_start=3, seed=11)
    assert np.array_equal(acc, ref)
    assert np.array_equal(disp[..., :3], (ref[..., :3] / ref[..., 3:4]).astype(np.float32))


@pytest.mark.gpu
def test_physical_fp64_and_heightfield(ctx):
    idx, pts = heightfield(24, seed=5)
    mats = np.array([[0, 0]], np.int32)
    mdata = pbr_material([0.7, 0.6, 0.5], ior=1.5, roughness=0.2, metallic=0.0)
    s = dict(indices=idx, vertices=pts, materials=mats, material_data=mdata)
    lights = np.stack([area_light((0.3, 1.2, 0.1), 0.3, [30.0, 20.0, 10.0]),
                       area_light((-0.5, 0.8, -0.4), 0.1, [5.0, 5.0, 40.0])])
    ctx.upload_scene(**s)
    ctx.set_area_lights(lights)
    W, H = 32, 32
    iv, ip = look_at((0, 1.5, -2.5), (0, 0, 0), vfov_deg=60, aspect=1.0)
    ctx.render_physical(iv, ip, W, H, spp=6, max_depth=5, rr_start=1, seed=2, fp64=True)
    acc = ctx.read_accumulation_f64(W, H)
    ref = po.render_physical(s, W, H, 6, iv, ip, lights, max_depth=5, rr_start=1, seed=2, fp64=True)
    assert np.array_equal(acc, ref)
    assert (acc[..., :3] > 0).mean() > 0.15  # the height field fills about a quarter of the view


@pytest.mark.gpu
@pytest.mark.parametrize("chain", [False, True])
def test_physical_mesh_and_sdf(ctx, chain):
    """Mesh + SDF render bit-identical to the oracle; the chained field runs
    through the evaluator's cell lists and the march's early exit."""
    from myrt_b200 import sdf as S

    s, lights = icosphere_field_lit(n_spheres=12, subdiv=2, floor_cells=4, seed=6)
    lib = S.SdfLibrary()
    lib.add(S.random_sdf_field(64, k=0.1, seed=2, extent=0.6, chain=chain))
    dr = S.sdf_drawables([np.array([[1, 0, 0, 0.0], [0, 1, 0, 0.2], [0, 0, 1, 0.5], [0, 0, 0, 1]])], [0])
    ctx.upload_scene(**s)
    ctx.upload_sdf(lib.instrs, lib.programs, lib.params, dr)
    ctx.set_area_lights(lights)
    W, H = 40, 32
    iv, ip = look_at((0, 1, -4.5), (0, -0.3, 0), vfov_deg=50, aspect=W / H)
    ctx.render_physical(iv, ip, W, H, spp=2, max_depth=6, seed=9, sdf_marching_steps=128, sdf_marching_epsilon=1e-4)
    acc, _ = ctx.read_accumulation(W, H)
    scene = dict(s, sdf=dict(lib=lib, drawables=dr, steps=128, eps=1e-4))
    ref = po.render_physical(scene, W, H, 2, iv, ip, lights, max_depth=6, seed=9)
    ctx.upload_sdf(np.zeros((0, 2)), np.zeros((0, 2)), np.zeros(0), np.zeros((0, 36)))
    assert np.array_equal(acc, ref)


@pytest.mark.gpu
def test_sorted_extension_queues_do_not_change_the_image(ctx):
    """A 1 Mi-path wave (256 x 256 x 16 spp) sorts its vertex-1 and vertex-2
    extension queues by default (trace_order 0); sorting none (1) or every
    vertex after the camera's (2) gives the same bits. A small render of the
    same scene with sorted queues still equals the oracle."""
    s, lights = icosphere_field_lit(n_spheres=64, subdiv=2, floor_cells=8, seed=9)
    ctx.upload_scene(**s)
    ctx.set_area_lights(lights)
    W = H = 256
    iv, ip = look_at((0, 1, -4.5), (0, -0.3, 0), vfov_deg=50, aspect=1.0)
    out = []
    try:
        for order in (1, 0, 2):
            ctx.set_tuning(trace_order=order)
            ctx.reset_accumulation()
            ctx.render_physical(iv, ip, W, H, spp=16, max_depth=6, rr_start=3, seed=21)
            out.append(ctx.read_accumulation(W, H)[0])
        ctx.set_tuning(trace_order=2)
        w, h = 40, 24
        iv2, ip2 = look_at((0, 1, -4.5), (0, -0.3, 0), vfov_deg=50, aspect=w / h)
        ctx.reset_accumulation()
        ctx.render_physical(iv2, ip2, w, h, spp=4, max_depth=6, rr_start=3, seed=5)
        small = ctx.read_accumulation(w, h)[0]
    finally:
        ctx.set_tuning()
    for acc in out[1:]:
        assert np.array_equal(acc, out[0])
    assert out[0][..., 3].min() == 16
    ref = po.render_physical(s, w, h, 4, iv2, ip2, lights, max_depth=6, rr_start=3, seed=5)
    assert np.array_equal(small, ref)
