"""Device BVH build (linear BVH + 8-wide collapse on the GPU, tuning
bvh_builder = 1): every triangle exactly once and inside every quantised slot
box on its path from the root (the condition for conservative culling; a
child's own quantised boxes, rounded outwards on its own grid, may reach past
its parent's), and ray answers bit-identical to the host-built
tree's (closest-hit ties go to the smaller prim id, so answers do not depend on
the tree); per-ray node / triangle counters equal the oracle's walk of the same
device-built tree."""
import numpy as np
import pytest

import myrt_b200 as mb
import pyoracle as po
from myrt_b200.scenes import heightfield, icosphere_camera_rays, icosphere_field, pinhole_rays

pytestmark = pytest.mark.gpu


def _slot_boxes(node):
    """float64 [8, 2, 3] slot boxes (lo, hi) of one node (uint32 [20])."""
    p = node[0:3].view(np.float32).astype(np.float64)
    e = node[3].tobytes()
    scale = np.array([2.0 ** (int(e[a]) - 127) for a in range(3)])
    q = node[8:20].tobytes()
    qlo = np.frombuffer(q[0:24], np.uint8).reshape(3, 8).astype(np.float64)
    qhi = np.frombuffer(q[24:48], np.uint8).reshape(3, 8).astype(np.float64)
    lo = p[:, None] + qlo * scale[:, None]
    hi = p[:, None] + qhi * scale[:, None]
    return np.stack([lo.T, hi.T], 1)


def _check_tree(nodes, tris, n_prims):
    prims = tris[:, 3].view(np.uint32)
    assert np.array_equal(np.sort(prims), np.arange(n_prims, dtype=np.uint32))
    seen = np.zeros(len(nodes), bool)
    stack = [(0, (np.full(3, -np.inf), np.full(3, np.inf)))]
    while stack:
        ni, outer = stack.pop()
        assert not seen[ni]
        seen[ni] = True
        nd = nodes[ni]
        imask = int(nd[3] >> 24)
        child_base, tri_base = int(nd[4]), int(nd[5])
        meta = nd[6:8].tobytes()
        boxes = _slot_boxes(nd)
        rank = 0
        for s in range(8):
            m = meta[s]
            if m == 0:
                continue
            lo, hi = np.maximum(boxes[s][0], outer[0]), np.minimum(boxes[s][1], outer[1])
            if imask & (1 << s):
                stack.append((child_base + rank, (lo, hi)))
                rank += 1
            else:
                off, cnt = m & 31, m >> 5
                assert 1 <= cnt <= 4
                v = tris[tri_base + off: tri_base + off + cnt][:, [0, 1, 2, 4, 5, 6, 8, 9, 10]].reshape(-1, 3)
                assert np.all(v.astype(np.float64) >= lo) and np.all(v.astype(np.float64) <= hi)
    assert seen.all()


def _rand_rays(n, seed, lo=-1.3, hi=1.3):
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    r[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    r[:, 7] = np.inf
    r[::11, 7] = rng.uniform(0.05, 1.0, r[::11].shape[0])
    return r


@pytest.mark.parametrize("n", [1, 3, 5, 40, 128])
def test_device_build_heightfield(ctx, n):
    idx, pts = heightfield(n, seed=3) if n > 3 else (np.arange(3 * n, dtype=np.uint32),
                                                     np.random.default_rng(n).uniform(-1, 1, (3 * n, 3)).astype(
                                                         np.float32))
    tris9 = pts[idx.reshape(-1, 3)].reshape(-1, 9)
    hn, ht, _ = mb.build_bvh8(tris9)
    rays = np.concatenate([pinhole_rays(96, 96), _rand_rays(20_000, seed=n)])
    host, _, _ = po.bvh8_traverse(hn, ht, rays)
    try:
        ctx.set_tuning(bvh_builder=1)
        info = ctx.upload_scene(idx, pts)
        nodes, tris = ctx.scene_bvh()
        assert info["triangles"] == tris9.shape[0] and info["wide_depth"] >= 1
        _check_tree(nodes, tris, tris9.shape[0])
        dev_walk, cn, ct = po.bvh8_traverse(nodes, tris, rays)
        assert np.array_equal(dev_walk, host)
        got = ctx.trace_closest(rays)
        assert np.array_equal(got, host)
        assert np.array_equal(ctx.trace_any(rays).astype(bool), host["prim"] >= 0)
        import torch

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


def test_device_build_instanced_spheres(ctx):
    """The 655,872-triangle instanced scene: device-built tree, same answers as
    the host-built tree on camera and random rays."""
    s = icosphere_field()
    try:
        ctx.set_tuning(bvh_builder=1)
        info = ctx.upload_scene(**s)
        assert info["triangles"] == 655_872
        nodes, tris = ctx.scene_bvh()
        prims = np.sort(tris[:, 3].view(np.uint32))
        assert np.array_equal(prims, np.arange(655_872, dtype=np.uint32))
        tris9 = po.bake_world_triangles(s["indices"], s["vertices"], s["drawables"])
        rays = np.concatenate([icosphere_camera_rays(256, 256), _rand_rays(60_000, seed=5, lo=-1.1, hi=1.1)])
        hn, ht, _ = mb.build_bvh8(tris9)
        host, _, _ = po.bvh8_traverse(hn, ht, rays)
        assert np.array_equal(ctx.trace_closest(rays), host)
        assert np.array_equal(ctx.trace_any(rays).astype(bool), host["prim"] >= 0)
    finally:
        ctx.set_tuning()


def _moved(drawables, seed):
    """New transforms (rotation about y, scale, translation) and material
    indices for every drawable of an instanced scene."""
    from myrt_b200._abi import myrt_drawable

    rng = np.random.default_rng(seed)
    out = (myrt_drawable * len(drawables))()
    for k, d in enumerate(drawables):
        m = np.array(d.transformation[:], np.float64).reshape(4, 4).T
        a = rng.uniform(0, 2 * np.pi)
        rot = np.array([[np.cos(a), 0, np.sin(a), 0], [0, 1, 0, 0], [-np.sin(a), 0, np.cos(a), 0], [0, 0, 0, 1]])
        mv = np.eye(4)
        mv[:3, 3] = rng.uniform(-0.3, 0.3, 3)
        m2 = mv @ m @ rot if k % 3 else m  # every third drawable keeps its transform
        out[k] = d
        out[k].transformation[:] = m2.T.astype(np.float32).ravel().tolist()
        out[k].inverse_transformation[:] = np.linalg.inv(m2).T.astype(np.float32).ravel().tolist()
        out[k].material_index = (d.material_index + k) % 7
    return out


def test_set_transforms_equals_reupload(ctx):
    """Moving the instances on the device (re-bake + device rebuild) answers
    rays and renders images exactly like uploading the moved scene again."""
    from myrt_b200.camera import look_at
    from myrt_b200.scenes import icosphere_field_lit

    s, lights = icosphere_field_lit(n_spheres=48, subdiv=2, floor_cells=4, seed=8)
    moved = _moved(s["drawables"], seed=3)
    rays = np.concatenate([icosphere_camera_rays(160, 120), _rand_rays(30_000, seed=6, lo=-1.2, hi=1.2)])
    iv, ip = look_at((0, 1, -4.5), (0, -0.3, 0), vfov_deg=50, aspect=4 / 3)
    ctx.upload_scene(**s)
    ctx.set_area_lights(lights)
    info = ctx.set_transforms(moved)
    assert info["triangles"] == sum(d.index_count for d in moved) // 3
    got = ctx.trace_closest(rays)
    got_any = ctx.trace_any(rays)
    ctx.render_physical(iv, ip, 64, 48, spp=4, max_depth=5, seed=2)
    img, _ = ctx.read_accumulation(64, 48)
    ctx.upload_scene(**dict(s, drawables=moved))
    ref = ctx.trace_closest(rays)
    assert np.array_equal(got, ref)
    assert np.array_equal(got_any, ctx.trace_any(rays))
    ctx.render_physical(iv, ip, 64, 48, spp=4, max_depth=5, seed=2)
    ref_img, _ = ctx.read_accumulation(64, 48)
    assert np.array_equal(img, ref_img)
    # geometry changes are refused
    bad = _moved(s["drawables"], seed=4)
    bad[0].index_count -= 3
    with pytest.raises(mb.MyrtError):
        ctx.set_transforms(bad)


@pytest.mark.parametrize("builder", [0, 1])
def test_repeated_moves_equal_reupload(ctx, builder):
    """Moves alternate between two sets of tree and corner buffers (the second
    move builds into the spare set, the third into the first tree again, ...).
    After every move in a sequence that returns to earlier poses, ray answers
    and forward-renderer visibility equal an upload of that pose, for a scene
    first built on the host (0) and on the device (1)."""
    from myrt_b200.camera import look_at
    from myrt_b200.scenes import icosphere_field_lit

    s, _ = icosphere_field_lit(n_spheres=40, subdiv=2, floor_cells=4, seed=9)
    poses = [_moved(s["drawables"], seed=3), _moved(s["drawables"], seed=5), _moved(s["drawables"], seed=3),
             s["drawables"], _moved(s["drawables"], seed=7)]
    rays = np.concatenate([icosphere_camera_rays(96, 72), _rand_rays(20_000, seed=11, lo=-1.2, hi=1.2)])
    view, proj = look_at((0, 1, -4.5), (0, -0.3, 0), vfov_deg=50, aspect=4 / 3)
    W, H = 96, 72

    def answers():
        ctx.forward_render(view, proj, W, H, 1, 256)
        return ctx.trace_closest(rays), ctx.trace_any(rays), ctx.forward_read(W, H, 256)["visibility"]

    refs = {}
    try:
        for i, p in enumerate(poses):
            key = id(p) if i != 2 else id(poses[0])
            if key not in refs:
                ctx.set_tuning(bvh_builder=builder)
                ctx.upload_scene(**dict(s, drawables=p))
                refs[key] = answers()
        ctx.set_tuning(bvh_builder=builder)
        ctx.upload_scene(**s)
        for i, p in enumerate(poses):
            ctx.set_transforms(p)
            got = answers()
            ref = refs[id(p) if i != 2 else id(poses[0])]
            assert np.array_equal(got[0], ref[0]), i
            assert np.array_equal(got[1], ref[1]), i
            assert np.array_equal(got[2], ref[2]), i
    finally:
        ctx.set_tuning()
