"""GPU closest-hit / any-hit parity against the CPU oracle, through the C ABI.

Bar: bit-exact prim ids, t, u and v (integer/index work and the same IEEE
operations on both sides), for both intersectors, at the full sizes of the
closest-hit configuration (1024^2 rays, 32,768 triangles) and of the
path-tracing scene (655,872 triangles).
"""
import numpy as np
import pytest

import myrt_b200 as mb
import pyoracle as po
from myrt_b200.scenes import heightfield, icosphere_camera_rays, icosphere_field, pinhole_rays

pytestmark = pytest.mark.gpu


def _rand_rays(n, seed, lo=-1.3, hi=1.3):
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    r[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    r[:, 7] = np.inf
    r[::11, 7] = rng.uniform(0.05, 1.0, r[::11].shape[0])
    r[::13, 3] = rng.uniform(0.0, 0.2, r[::13].shape[0])
    r[::17, 4:7] = np.array([0.0, -1.0, 0.0])  # axis-aligned: zero direction components
    r[::19, 4:7] *= 3.5  # unnormalised direction
    return r


@pytest.fixture(scope="module")
def hf128(ctx):
    idx, pts = heightfield(128, seed=1)
    info = ctx.upload_scene(idx, pts)
    tris9 = pts[idx.reshape(-1, 3)].reshape(-1, 9)
    nodes, tris, _ = mb.build_bvh8(tris9)
    return dict(idx=idx, pts=pts, tris9=tris9, nodes=nodes, tris=tris, info=info)


def test_golden_closest_hits_on_gpu(ctx, golden):
    g = golden("closest_hf128.npz")
    idx, pts, rays, glsl = g["indices"], g["points"], g["rays"], g["glsl"]
    ctx.upload_scene(idx, pts)
    hits = ctx.trace_closest(rays)
    same = hits["prim"] == glsl["prim"]
    print(f"prim id agreement with the reference's GLSL traversal: {same.mean():.6f} "
          f"({int((~same).sum())} of {same.size} differ)")
    # no ray of the golden set ties exactly in t, so the tie rules (first visited in the reference,
    # smaller prim id here) never come into play: every id agrees
    assert same.all()
    assert np.array_equal(hits["t"], glsl["t"])
    hit = glsl["prim"] >= 0
    assert np.array_equal(hits["u"][hit], glsl["u"][hit])
    assert np.array_equal(hits["v"][hit], glsl["v"][hit])
    occ = ctx.trace_any(g["shadow_rays"])
    assert np.array_equal(occ.astype(bool), g["any_short_prim"] >= 0)


@pytest.mark.parametrize("isect", [mb.ISECT_REFERENCE, mb.ISECT_WATERTIGHT])
def test_closest_full_camera_bit_exact(ctx, hf128, isect):
    ctx.upload_scene(hf128["idx"], hf128["pts"])
    rays = pinhole_rays(1024, 1024)
    hits = ctx.trace_closest(rays, intersector=isect)
    ora, _, _ = po.bvh8_traverse(hf128["nodes"], hf128["tris"], rays, isect=isect)
    assert np.array_equal(hits, ora)
    sub = slice(None, None, 97)
    bf = po.brute_closest(hf128["tris9"], rays[sub], isect=isect)
    assert np.array_equal(hits[sub], bf)


@pytest.mark.parametrize("isect", [mb.ISECT_REFERENCE, mb.ISECT_WATERTIGHT])
def test_random_rays_closest_and_any(ctx, hf128, isect):
    ctx.upload_scene(hf128["idx"], hf128["pts"])
    rays = _rand_rays(300_000, seed=isect + 10)
    hits = ctx.trace_closest(rays, intersector=isect)
    ora, _, _ = po.bvh8_traverse(hf128["nodes"], hf128["tris"], rays, isect=isect)
    assert np.array_equal(hits, ora)
    occ = ctx.trace_any(rays, intersector=isect)
    occ_o, _, _ = po.bvh8_traverse(hf128["nodes"], hf128["tris"], rays, isect=isect, any_hit=True)
    assert np.array_equal(occ, occ_o)
    assert np.array_equal(occ.astype(bool), ora["prim"] >= 0)


def test_device_entry_points_and_counters(ctx, hf128):
    import torch

    ctx.upload_scene(hf128["idx"], hf128["pts"])
    rays = _rand_rays(100_000, seed=5)
    d_rays = torch.from_numpy(rays).cuda()
    d_hits = torch.empty((rays.shape[0], 4), dtype=torch.float32, device="cuda")
    d_n = torch.empty(rays.shape[0], dtype=torch.int32, device="cuda")
    d_t = torch.empty(rays.shape[0], dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    ctx.trace_closest_stats_device(d_rays, d_hits, d_n, d_t)
    ctx.sync()
    ora, cn, ct = po.bvh8_traverse(hf128["nodes"], hf128["tris"], rays)
    got = d_hits.cpu().numpy().view(mb.HIT_DTYPE).ravel()
    assert np.array_equal(got, ora)
    # the counters behind the roofline's bytes per ray are exact
    assert np.array_equal(d_n.cpu().numpy().astype(np.uint32), cn)
    assert np.array_equal(d_t.cpu().numpy().astype(np.uint32), ct)
    ctx.trace_closest_device(d_rays, d_hits)
    ctx.sync()
    assert np.array_equal(d_hits.cpu().numpy().view(mb.HIT_DTYPE).ravel(), ora)
    d_occ = torch.empty(rays.shape[0], dtype=torch.uint8, device="cuda")
    ctx.trace_any_device(d_rays, d_occ)
    ctx.sync()
    assert np.array_equal(d_occ.cpu().numpy().astype(bool), ora["prim"] >= 0)


def test_instanced_sphere_scene_bit_exact(ctx):
    s = icosphere_field()
    info = ctx.upload_scene(**s)
    assert info["triangles"] == 655_872
    tris9 = po.bake_world_triangles(s["indices"], s["vertices"], s["drawables"])
    rays = np.concatenate([icosphere_camera_rays(512, 512, spp=2), _rand_rays(200_000, seed=9, lo=-1.1, hi=1.1)])
    hits = ctx.trace_closest(rays)
    nodes, tris, _ = mb.build_bvh8(tris9)
    ora, _, _ = po.bvh8_traverse(nodes, tris, rays)
    assert np.array_equal(hits, ora)
    sub = slice(None, None, 331)
    assert np.array_equal(hits[sub], po.brute_closest(tris9, rays[sub]))
    occ = ctx.trace_any(rays)
    assert np.array_equal(occ.astype(bool), ora["prim"] >= 0)


def test_edge_cases(ctx):
    tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0]], np.float32)
    idx = np.array([0, 1, 2, 1, 3, 2], np.uint32)  # two triangles sharing an edge
    ctx.upload_scene(idx, tri)
    rays = np.zeros((6, 8), np.float32)
    rays[:, 6] = 1.0
    rays[:, 2] = -1.0
    rays[:, 7] = np.inf
    rays[0, 0:2] = (0.25, 0.25)  # inside the first triangle
    rays[1, 0:2] = (0.5, 0.5)    # on the shared edge: tie in t, smaller prim wins
    rays[2, 0:2] = (2.0, 2.0)    # miss
    rays[3, 0:2] = (0.25, 0.25)
    rays[3, 7] = 0.5             # tmax before the surface
    rays[4, 0:2] = (0.75, 0.75)
    rays[5, 0:2] = (0.25, 0.25)
    rays[5, 3] = 2.0             # tmin beyond the surface
    hits = ctx.trace_closest(rays)
    assert list(hits["prim"]) == [0, 0, -1, -1, 1, -1]
    assert hits["t"][0] == 1.0 and hits["t"][3] == 0.5
    assert np.array_equal(ctx.trace_any(rays), np.array([1, 1, 0, 0, 1, 0], np.uint8))
    # an empty batch is a no-op
    assert ctx.trace_closest(np.zeros((0, 8), np.float32)).size == 0


def test_errors_are_reported(ctx):
    with pytest.raises(mb.MyrtError):
        ctx.upload_scene(np.array([0, 1], np.uint32), np.zeros((3, 3), np.float32))  # not a multiple of 3
    with pytest.raises(mb.MyrtError):
        ctx.upload_scene(np.array([0, 1, 7], np.uint32), np.zeros((3, 3), np.float32))  # index out of range
    with pytest.raises(mb.MyrtError):
        ctx.trace_closest(np.zeros((4, 8), np.float32), intersector=7)


@pytest.mark.parametrize("refill", [1, 8, 32])
def test_persistent_traversal_bit_exact(ctx, hf128, refill):
    """The persistent kernel (lanes refilled with new rays) visits the same nodes
    per ray as the one-thread-per-ray kernel: same hits, same counters."""
    import torch

    ctx.upload_scene(hf128["idx"], hf128["pts"])
    rays = np.concatenate([pinhole_rays(256, 256), _rand_rays(100_000, seed=21)])
    ora, cn, ct = po.bvh8_traverse(hf128["nodes"], hf128["tris"], rays)
    try:
        ctx.set_tuning(trace_persistent=1, refill=refill, blocks_per_sm=0)
        assert np.array_equal(ctx.trace_closest(rays), ora)
        occ = ctx.trace_any(rays)
        assert np.array_equal(occ.astype(bool), ora["prim"] >= 0)
        d_rays = torch.from_numpy(rays).cuda()
        d_hits = torch.empty((rays.shape[0], 4), dtype=torch.float32, device="cuda")
        d_n = torch.empty(rays.shape[0], dtype=torch.int32, device="cuda")
        d_t = torch.empty(rays.shape[0], dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        ctx.trace_closest_stats_device(d_rays, d_hits, d_n, d_t)
        ctx.sync()
        assert np.array_equal(d_hits.cpu().numpy().view(mb.HIT_DTYPE).ravel(), ora)
        assert np.array_equal(d_n.cpu().numpy().astype(np.uint32), cn)
        assert np.array_equal(d_t.cpu().numpy().astype(np.uint32), ct)
    finally:
        ctx.set_tuning(trace_persistent=0)


def test_unit_step_traversal_bit_exact(ctx, hf128):
    """One node / triangle / pop per iteration walks the same order: same hits and counters."""
    import torch

    ctx.upload_scene(hf128["idx"], hf128["pts"])
    rays = np.concatenate([pinhole_rays(256, 256), _rand_rays(100_000, seed=22)])
    ora, cn, ct = po.bvh8_traverse(hf128["nodes"], hf128["tris"], rays)
    try:
        ctx.set_tuning(trace_unit_steps=1)
        assert np.array_equal(ctx.trace_closest(rays), ora)
        assert np.array_equal(ctx.trace_any(rays).astype(bool), ora["prim"] >= 0)
        d_rays = torch.from_numpy(rays).cuda()
        d_hits = torch.empty((rays.shape[0], 4), dtype=torch.float32, device="cuda")
        d_n = torch.empty(rays.shape[0], dtype=torch.int32, device="cuda")
        d_t = torch.empty(rays.shape[0], dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        ctx.trace_closest_stats_device(d_rays, d_hits, d_n, d_t)
        ctx.sync()
        assert np.array_equal(d_n.cpu().numpy().astype(np.uint32), cn)
        assert np.array_equal(d_t.cpu().numpy().astype(np.uint32), ct)
    finally:
        ctx.set_tuning()


@pytest.mark.parametrize("isect", [0, 1])
def test_shared_stack_traversal_bit_exact(ctx, hf128, isect):
    """The traversal stack in shared memory (tree depth + 1 entries per ray)
    walks the same order as the per-thread stack: same hits and counters, for
    closest and any hit, both intersectors."""
    import torch

    ctx.upload_scene(hf128["idx"], hf128["pts"])
    rays = np.concatenate([pinhole_rays(256, 256), _rand_rays(100_000, seed=23)])
    ora, cn, ct = po.bvh8_traverse(hf128["nodes"], hf128["tris"], rays, isect=isect)
    try:
        ctx.set_tuning(trace_smem_stack=1)
        assert np.array_equal(ctx.trace_closest(rays, intersector=isect), ora)
        assert np.array_equal(ctx.trace_any(rays, intersector=isect).astype(bool), ora["prim"] >= 0)
        d_rays = torch.from_numpy(rays).cuda()
        d_hits = torch.empty((rays.shape[0], 4), dtype=torch.float32, device="cuda")
        d_n = torch.empty(rays.shape[0], dtype=torch.int32, device="cuda")
        d_t = torch.empty(rays.shape[0], dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        ctx.trace_closest_stats_device(d_rays, d_hits, d_n, d_t, intersector=isect)
        ctx.sync()
        assert np.array_equal(d_n.cpu().numpy().astype(np.uint32), cn)
        assert np.array_equal(d_t.cpu().numpy().astype(np.uint32), ct)
    finally:
        ctx.set_tuning()


@pytest.mark.parametrize("isect", [0, 1])
@pytest.mark.parametrize("variant", [dict(trace_min_blocks=8), dict(trace_min_blocks=10), dict(trace_min_blocks=12),
                                     dict(trace_order=2, trace_min_blocks=10)])
def test_launch_variants_bit_exact(ctx, hf128, isect, variant):
    """The register caps (8, 10 and 12 blocks per SM) and the sorted order change
    how the walk runs, not what it finds: closest and any hit equal the
    oracle's, for both intersectors, on the height field and on the instanced
    icosphere scene."""
    ctx.upload_scene(hf128["idx"], hf128["pts"])
    rays = np.concatenate([pinhole_rays(256, 256), _rand_rays(100_000, seed=29)])
    ora, _, _ = po.bvh8_traverse(hf128["nodes"], hf128["tris"], rays, isect=isect)
    try:
        ctx.set_tuning(**variant)
        assert np.array_equal(ctx.trace_closest(rays, intersector=isect), ora)
        assert np.array_equal(ctx.trace_any(rays, intersector=isect).astype(bool), ora["prim"] >= 0)
        s = icosphere_field(n_spheres=64, subdiv=3, floor_cells=8, seed=9)
        ctx.upload_scene(**s)
        cam = pinhole_rays(192, 160, eye=(0.0, 1.0, -4.5), target=(0.0, -0.3, 0.0), vfov_deg=50)
        tris9 = po.bake_world_triangles(s["indices"], s["vertices"], s["drawables"])
        nodes, tris, _ = mb.build_bvh8(tris9)
        ref, _, _ = po.bvh8_traverse(nodes, tris, cam, isect=isect)
        assert np.array_equal(ctx.trace_closest(cam, intersector=isect), ref)
    finally:
        ctx.set_tuning()


@pytest.mark.parametrize("order", [1, 2])
def test_ray_order_does_not_change_results(ctx, hf128, order):
    """Sorted visiting order (trace_order 2) and input order (1) give the same
    hits, occlusion and per-ray counters as the oracle, through the host and
    the device entry points; rays are a shuffled mix of camera and random rays."""
    import torch

    ctx.upload_scene(hf128["idx"], hf128["pts"])
    rays = np.concatenate([pinhole_rays(256, 256), _rand_rays(150_000, seed=24)])
    rays = rays[np.random.default_rng(3).permutation(rays.shape[0])]
    ora, cn, ct = po.bvh8_traverse(hf128["nodes"], hf128["tris"], rays)
    try:
        ctx.set_tuning(trace_order=order)
        assert np.array_equal(ctx.trace_closest(rays), ora)
        assert np.array_equal(ctx.trace_any(rays).astype(bool), ora["prim"] >= 0)
        d_rays = torch.from_numpy(rays).cuda()
        d_hits = torch.empty((rays.shape[0], 4), dtype=torch.float32, device="cuda")
        d_n = torch.empty(rays.shape[0], dtype=torch.int32, device="cuda")
        d_t = torch.empty(rays.shape[0], dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        ctx.trace_closest_stats_device(d_rays, d_hits, d_n, d_t)
        ctx.sync()
        assert np.array_equal(d_hits.cpu().numpy().view(mb.HIT_DTYPE).ravel(), ora)
        assert np.array_equal(d_n.cpu().numpy().astype(np.uint32), cn)
        assert np.array_equal(d_t.cpu().numpy().astype(np.uint32), ct)
    finally:
        ctx.set_tuning()


def test_phase_timing(ctx, hf128):
    """Per-query device times of the ordering phase and the traversal kernel."""
    ctx.upload_scene(hf128["idx"], hf128["pts"])
    rays = pinhole_rays(1024, 1024)  # 1 Mi rays: sorted by default
    ctx.set_phase_timing(True)
    try:
        ctx.phase_times()
        ctx.trace_closest(rays)  # host path: input order
        import torch

        d_rays = torch.from_numpy(rays).cuda()
        d_hits = torch.empty((rays.shape[0], 4), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        ctx.trace_closest_device(d_rays, d_hits)
        t = ctx.phase_times()
        # the host query runs as 8 chunks of 128 Ki rays (an eighth of the query each), the device query as one
        assert t["queries"] == 8 + 1 and t["traverse_ms"] > 0 and t["order_ms"] > 0
        assert ctx.phase_times()["queries"] == 0
    finally:
        ctx.set_phase_timing(False)


def test_large_sorted_query_matches_input_order(ctx, hf128):
    """A device query of more than 2 Mi rays (an odd count) in sorted visiting
    order: hits, occlusion and per-ray counters equal input order and the
    oracle."""
    import torch

    ctx.upload_scene(hf128["idx"], hf128["pts"])
    rays = np.concatenate([pinhole_rays(1024, 1024), _rand_rays(1_200_001, seed=31)])
    rays = rays[np.random.default_rng(5).permutation(rays.shape[0])]
    n = rays.shape[0]
    assert n >= 2 << 20
    d_rays = torch.from_numpy(rays).cuda()
    out = {}
    try:
        for order in (1, 0):
            ctx.set_tuning(trace_order=order)
            d_hits = torch.empty((n, 4), dtype=torch.float32, device="cuda")
            d_occ = torch.empty(n, dtype=torch.uint8, device="cuda")
            d_n = torch.empty(n, dtype=torch.int32, device="cuda")
            d_t = torch.empty(n, dtype=torch.int32, device="cuda")
            torch.cuda.synchronize()
            ctx.trace_closest_device(d_rays, d_hits)
            ctx.trace_any_device(d_rays, d_occ)
            ctx.sync()
            hits = d_hits.cpu().numpy().copy()
            ctx.trace_closest_stats_device(d_rays, d_hits, d_n, d_t)
            ctx.sync()
            out[order] = (hits, d_occ.cpu().numpy(), d_hits.cpu().numpy(), d_n.cpu().numpy(), d_t.cpu().numpy())
    finally:
        ctx.set_tuning()
    for a, b in zip(out[0], out[1]):  # raw bits: a miss's prim -1 reads as NaN in float32
        assert np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8))
    sel = np.random.default_rng(6).choice(n, 200_000, replace=False)
    ora, cn, ct = po.bvh8_traverse(hf128["nodes"], hf128["tris"], rays[sel])
    assert np.array_equal(out[0][0][sel].view(mb.HIT_DTYPE).ravel(), ora)
    assert np.array_equal(out[0][3][sel].astype(np.uint32), cn)


def test_upload_of_a_tree_deeper_than_the_stack_is_refused(ctx, hf128):
    """myrt_scene_upload refuses a tree deeper than the traversal stack (32
    wide levels) with MYRT_ERR_UNSUPPORTED instead of letting kernels overflow
    it; the context then takes a normal scene and answers queries."""
    from myrt_b200.scenes import exponential_chain

    t9 = exponential_chain()
    with pytest.raises(mb.MyrtError, match="deeper than the traversal stack") as e:
        ctx.upload_scene(np.arange(t9.shape[0] * 3, dtype=np.uint32), t9.reshape(-1, 3))
    assert e.value.code == mb.MYRT_ERR_UNSUPPORTED
    ctx.upload_scene(hf128["idx"], hf128["pts"])
    rays = pinhole_rays(64, 64)
    hits = ctx.trace_closest(rays)
    assert (hits["prim"] >= 0).any()
