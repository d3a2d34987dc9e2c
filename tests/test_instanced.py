"""Instanced scenes: the reference's two-level walk (src/pt/pt_trace.comp:98-116,
284-309, visit_object_aabb) -- a tree over the drawables' world boxes, each ray
moved into a drawable's object space by inverse_transformation and tested
against the untransformed geometry.

Golden data (tests/golden/instanced_field.npz) comes from the reference's own
code compiled in oracle/_ref: bvh.cpp trees (split_aabbs per geometry as
scene::push_geometry builds them, dont_split over the drawables' world boxes as
scene::prepare does) walked by the compiled bvh.impl.glsl + visit_object_aabb.

Bar: hit prim ids equal the reference's except on exact ties in t (the
reference keeps the first visited, the library the smaller prim id; where ids
differ, t must be equal and the library's id smaller); t, u, v bit-identical
wherever the ids agree; any-hit answers identical. The agreement fraction is
printed.
"""
import ctypes as C

import numpy as np
import pytest

import myrt_b200 as mb
import pyoracle as po
from myrt_b200._abi import myrt_drawable
from myrt_b200.scenes import icosphere_field, instanced_field, pinhole_rays


def _scene_from_golden(g):
    raw = np.ascontiguousarray(g["drawables"], np.uint32)
    dr = (myrt_drawable * raw.shape[0]).from_buffer_copy(raw.tobytes())
    return dict(indices=g["indices"], vertices=g["vertices"], drawables=dr)


def _check_against_reference(hits, ref, what):
    same = hits["prim"] == ref["prim"]
    n_diff = int((~same).sum())
    print(f"{what}: prim id agreement with the reference {same.mean():.6f} ({n_diff} of {same.size} differ)")
    # every disagreement is an exact tie in t that went to the smaller prim id
    assert np.array_equal(hits["t"], ref["t"])
    assert np.all(hits["prim"][~same] < ref["prim"][~same])
    assert np.all((hits["prim"][~same] >= 0) & (ref["prim"][~same] >= 0))
    hit = same & (ref["prim"] >= 0)
    assert np.array_equal(hits["u"][hit], ref["u"][hit])
    assert np.array_equal(hits["v"][hit], ref["v"][hit])
    return same.mean()


def test_oracle_instanced_matches_reference_golden(golden):
    g = golden("instanced_field.npz")
    sc = _scene_from_golden(g)
    got = po.instanced_closest(sc, g["rays"])
    _check_against_reference(got, g["hits"], "oracle")
    occ = po.instanced_closest(sc, g["shadow_rays"], any_hit=True)
    assert np.array_equal(occ, g["shadow_hit"])


def test_golden_scene_is_the_generator_output(golden):
    """The fixture's scene is instanced_field() (seeded), so the GPU tests can
    rebuild the same scene at other sizes."""
    g = golden("instanced_field.npz")
    sc = instanced_field()
    assert np.array_equal(sc["indices"], g["indices"])
    assert np.array_equal(sc["vertices"], g["vertices"])
    raw = np.frombuffer(C.string_at(C.addressof(sc["drawables"]), 160 * len(sc["drawables"])), np.uint32)
    assert np.array_equal(raw.reshape(-1, 40), g["drawables"])


def test_baked_world_triangles_differ_from_object_space_hits(golden):
    """Why the two-level walk exists: the same rays against the drawables baked
    into world space (one tree, what instancing = 0 does) round differently, so
    t and the barycentrics leave the reference's bits."""
    g = golden("instanced_field.npz")
    sc = _scene_from_golden(g)
    tris9 = po.bake_world_triangles(sc["indices"], sc["vertices"], sc["drawables"])
    baked = po.brute_closest(tris9, g["rays"])
    hit = (baked["prim"] >= 0) & (baked["prim"] == g["hits"]["prim"])
    assert (baked["t"][hit] != g["hits"]["t"][hit]).mean() > 0.05


@pytest.mark.gpu
@pytest.mark.parametrize("order", [1, 2])
def test_instanced_device_matches_reference_golden(ctx, golden, order):
    g = golden("instanced_field.npz")
    sc = _scene_from_golden(g)
    try:
        ctx.set_tuning(instancing=1, trace_order=order)
        ctx.upload_scene(**sc)
        hits = ctx.trace_closest(g["rays"])
        _check_against_reference(hits, g["hits"], f"device, trace_order {order}")
        occ = ctx.trace_any(g["shadow_rays"])
        assert np.array_equal(occ.astype(bool), g["shadow_hit"])
    finally:
        ctx.set_tuning()


@pytest.mark.gpu
@pytest.mark.parametrize("isect", [mb.ISECT_REFERENCE, mb.ISECT_WATERTIGHT])
def test_instanced_full_scene_bit_exact_vs_oracle(ctx, isect):
    """The 655,872-triangle icosphere scene (512 instances + floor): camera rays
    of a 512 x 384 view plus random rays, against the oracle's object-space
    walks (canonical ties: everything bit-exact)."""
    sc = icosphere_field()
    cam = pinhole_rays(512, 384, eye=(0.0, 1.0, -4.5), target=(0.0, -0.3, 0.0), vfov_deg=50)
    rng = np.random.default_rng(7)
    n = 65536
    o = rng.uniform(-2, 2, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rnd = np.zeros((n, 8), np.float32)
    rnd[:, 0:3], rnd[:, 4:7], rnd[:, 7] = o, d, np.inf
    rnd[::7, 3] = 0.05  # tmin
    rnd[::5, 7] = 0.7  # finite tmax
    rays = np.concatenate([cam, rnd], 0)
    ref = po.instanced_closest(sc, rays, isect=isect)
    try:
        ctx.set_tuning(instancing=1)
        ctx.upload_scene(**sc)
        hits = ctx.trace_closest(rays, intersector=isect)
        assert np.array_equal(hits, ref)
        occ = ctx.trace_any(rays, intersector=isect)
        assert np.array_equal(occ.astype(bool), ref["prim"] >= 0)
    finally:
        ctx.set_tuning()


@pytest.mark.gpu
def test_instanced_sorted_device_batch_and_stats(ctx):
    """A device-memory batch above the sorting threshold (1 Mi rays) on the
    two-level path equals the input-order answers; the per-ray counters count
    nodes of both levels and object-space triangle tests."""
    import torch

    sc = instanced_field(n_spheres=96, n_boxes=48)
    cam = pinhole_rays(1024, 1024, eye=(0.3, 1.5, -3.5), target=(0.0, -0.2, 0.0), vfov_deg=55)
    try:
        ctx.set_tuning(instancing=1, trace_order=1)
        ctx.upload_scene(**sc)
        rays = torch.from_numpy(cam).cuda()
        h1 = torch.empty((cam.shape[0], 4), dtype=torch.float32, device="cuda")
        h2 = torch.empty_like(h1)
        ctx.trace_closest_device(rays, h1)
        ctx.sync()
        ctx.set_tuning(instancing=1, trace_order=0)
        ctx.trace_closest_device(rays, h2)
        ctx.sync()
        # compare bits: a miss stores prim -1, whose bit pattern reads as a NaN float
        assert torch.equal(h1.view(torch.int32), h2.view(torch.int32))
        cn = torch.empty(cam.shape[0], dtype=torch.int32, device="cuda")
        ct = torch.empty_like(cn)
        h3 = torch.empty_like(h1)
        ctx.trace_closest_stats_device(rays, h3, cn, ct)
        ctx.sync()
        assert torch.equal(h1.view(torch.int32), h3.view(torch.int32))
        assert int(cn.min()) >= 1 and float(ct.float().mean()) > 0
        ref = po.instanced_closest(sc, cam[::37])
        assert np.array_equal(h1.cpu().numpy()[::37].copy().view(mb.HIT_DTYPE).reshape(-1), ref)
    finally:
        ctx.set_tuning()


@pytest.mark.gpu
def test_instanced_follows_transform_updates(ctx):
    """myrt_scene_set_transforms rebuilds the instance level: hits after moves
    equal the oracle on the moved scene, and a move back restores the first
    answers bit for bit."""
    sc = instanced_field(seed=5)
    rays = pinhole_rays(160, 120, eye=(0.3, 1.5, -3.5), target=(0.0, -0.2, 0.0), vfov_deg=55)
    try:
        ctx.set_tuning(instancing=1)
        ctx.upload_scene(**sc)
        first = ctx.trace_closest(rays)
        moved = (myrt_drawable * len(sc["drawables"])).from_buffer_copy(bytes(sc["drawables"]))
        rng = np.random.default_rng(3)
        for k in range(len(moved) - 1):
            m = np.array(moved[k].transformation[:], np.float32).reshape(4, 4).T
            m[:3, 3] += rng.uniform(-0.3, 0.3, 3).astype(np.float32)
            inv = np.linalg.inv(m.astype(np.float64)).astype(np.float32)
            moved[k].transformation[:] = m.T.ravel().tolist()
            moved[k].inverse_transformation[:] = inv.T.ravel().tolist()
        ctx.set_transforms(moved)
        got = ctx.trace_closest(rays)
        ref = po.instanced_closest(dict(sc, drawables=moved), rays)
        assert np.array_equal(got, ref)
        assert not np.array_equal(got, first)
        ctx.set_transforms(sc["drawables"])
        assert np.array_equal(ctx.trace_closest(rays), first)
    finally:
        ctx.set_tuning()


@pytest.mark.gpu
def test_instancing_needs_an_instanced_upload(ctx):
    sc = instanced_field()
    ctx.set_tuning()
    ctx.upload_scene(**sc)
    try:
        ctx.set_tuning(instancing=1)
        with pytest.raises(mb.MyrtError, match="instancing = 1"):
            ctx.trace_closest(pinhole_rays(8, 8))
    finally:
        ctx.set_tuning()
