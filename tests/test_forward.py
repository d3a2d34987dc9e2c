"""Forward (raster preview) renderer: the oracle's rasteriser against known
answers and against ray casting, and the library's light camera against the
restatement of forward_renderer.cpp:306-310. CPU only."""
import numpy as np
import pytest

import pyoracle as po
from myrt_b200 import forward_default_shadow
from myrt_b200.camera import view_projection
from myrt_b200.scenes import icosphere, icosphere_field, pbr_material

EMPTY = np.uint64(0xFFFFFFFFFFFFFFFF)


def _ortho(l, r, b, t, n, f):
    m = np.zeros((4, 4), np.float64)
    m[0, 0], m[1, 1], m[2, 2] = 2 / (r - l), 2 / (t - b), -2 / (f - n)
    m[0, 3], m[1, 3], m[2, 3], m[3, 3] = -(r + l) / (r - l), -(t + b) / (t - b), -(f + n) / (f - n), 1
    return m


def _quad(x0, y0, x1, y1, z):
    v = np.array([[x0, y0, z], [x1, y0, z], [x1, y1, z], [x0, y1, z]], np.float32)
    return v, np.array([0, 1, 2, 0, 2, 3], np.uint32)


def _scene(parts):
    verts, idx, base = [], [], 0
    for v, i in parts:
        verts.append(v)
        idx.append(i + base)
        base += len(v)
    v = np.concatenate(verts)
    n = np.tile(np.array([[0, 0, 1]], np.float32), (len(v), 1))
    return dict(indices=np.concatenate(idx), vertices=v, normals=n, materials=np.array([[0, 0]], np.int32),
                material_data=pbr_material([0.5, 0.5, 0.5]))


def test_default_shadow_camera_matches_restatement():
    a = np.radians(-45.0)
    c, s = np.cos(a), np.sin(a)
    rot = np.array([[1, 0, 0, 0], [0, c, -s, 0], [0, s, c, 0], [0, 0, 0, 1]])
    tr = np.eye(4)
    tr[2, 3] = 15.0
    view = np.linalg.inv(rot @ tr)
    proj = _ortho(-20, 20, 20, -20, 0.01, 1000.0)
    v, p = forward_default_shadow()
    assert np.allclose(v, view, atol=1e-6) and np.allclose(p, proj, atol=1e-9)
    # the light looks down at 45 degrees from +y +z, towards the origin
    light = np.linalg.inv(v) @ np.array([0, 0, 1, 0])
    assert np.allclose(light[:3] / np.linalg.norm(light[:3]), [0, np.sqrt(0.5), np.sqrt(0.5)], atol=1e-6)


def test_oracle_raster_quads_depth_order_and_ties():
    # orthographic 16x16 view of [0,16]^2: pixel (x, y) has its centre at (x + 0.5, y + 0.5)
    view, proj = np.eye(4, dtype=np.float32), _ortho(0, 16, 0, 16, -10, 10).astype(np.float32)
    far_q = _quad(2, 2, 10, 10, -1.0)    # triangles 0, 1 (z = -1: depth 0.55)
    near_q = _quad(6, 6, 14, 14, 1.0)    # 2, 3 (nearer)
    tie_q = _quad(0, 0, 4, 4, -1.0)      # 4, 5: overlaps far_q at equal depth, drawn later
    s = _scene([far_q, near_q, tie_q])
    out = po.forward_render(s, 16, 16, view, proj, 1, 4, view, proj, result=False)
    vis = out["visibility"]
    prim = np.where(vis == EMPTY, -1, (vis & np.uint64(0xFFFFFFFF)).astype(np.int64))
    depth = (vis >> np.uint64(32)).astype(np.int64)
    # coverage: centres strictly inside each quad's square
    for y in range(16):
        for x in range(16):
            cx, cy = x + 0.5, y + 0.5
            if 6 < cx < 14 and 6 < cy < 14:
                want = {2, 3}
            elif 2 < cx < 10 and 2 < cy < 10:
                want = {0, 1}
            elif 0 < cx < 4 and 0 < cy < 4:
                want = {4, 5}
            else:
                want = {-1}
            assert prim[y, x] in want, (x, y, prim[y, x])
    # equal depth: the first-drawn quad keeps the overlap (GL_LESS)
    assert prim[3, 3] in (0, 1)
    # 24-bit depth: z = -1 gives z_ndc = -0.1 * z = 0.1 (ortho near -10, far 10), depth 0.55
    assert depth[4, 4] == int(np.rint(0.55 * 16777215))
    # the shared diagonal of a quad: each centre belongs to exactly one triangle
    s1 = _scene([far_q])
    v1 = po.forward_render(s1, 16, 16, view, proj, 1, 4, view, proj, result=False)["visibility"]
    assert ((v1 != EMPTY).sum()) == 8 * 8


def test_oracle_raster_matches_ray_casting():
    """The rasteriser's triangle at each pixel centre is the closest hit of the
    ray through that centre, up to edges and 24-bit depth ties."""
    si, sp = icosphere(2)
    parts = [(sp * 0.8 + np.array([-0.5, 0.0, 0.0], np.float32), si),
             (sp * 0.6 + np.array([0.6, 0.2, 0.5], np.float32), si)]
    s = _scene(parts)
    W = H = 64
    eye, target = (0.3, 0.8, -3.0), (0.0, 0.0, 0.0)
    view, proj = view_projection(eye, target, vfov_deg=45, aspect=1.0, near=0.1, far=20.0)
    out = po.forward_render(s, W, H, view, proj, 1, 4, view, proj, result=False)
    vis = out["visibility"]
    prim = np.where(vis == EMPTY, -1, (vis & np.uint64(0xFFFFFFFF)).astype(np.int64))
    inv = np.linalg.inv(proj.astype(np.float64) @ view.astype(np.float64))
    ys, xs = np.mgrid[0:H, 0:W]
    nx, ny = (xs + 0.5) / W * 2 - 1, (ys + 0.5) / H * 2 - 1
    a = np.stack([nx, ny, -np.ones_like(nx), np.ones_like(nx)], -1) @ inv.T
    b = np.stack([nx, ny, np.ones_like(nx), np.ones_like(nx)], -1) @ inv.T
    a, b = a[..., :3] / a[..., 3:], b[..., :3] / b[..., 3:]
    rays = np.zeros((H * W, 8), np.float32)
    rays[:, :3] = a.reshape(-1, 3)
    rays[:, 4:7] = (b - a).reshape(-1, 3)
    rays[:, 7] = 1.0
    tris9 = po.bake_world_triangles(s["indices"], s["vertices"])
    hits = po.brute_closest(tris9, rays)
    agree = (hits["prim"].reshape(H, W) == prim).mean()
    assert (prim >= 0).mean() > 0.3
    assert agree > 0.985, agree


def test_oracle_raster_near_plane_crossing():
    """A floor that reaches behind the eye (corners with w <= 0) covers the
    lower half of the image without holes; nothing above the horizon."""
    v = np.array([[-50, 0, -50], [50, 0, -50], [50, 0, 50], [-50, 0, 50]], np.float32)
    s = _scene([(v, np.array([0, 1, 2, 0, 2, 3], np.uint32))])
    W, H = 48, 32
    view, proj = view_projection((0, 1, 0), (0, 1, 5), vfov_deg=60, aspect=W / H, near=0.05, far=200.0)
    vis = po.forward_render(s, W, H, view, proj, 1, 4, view, proj, result=False)["visibility"]
    covered = vis != EMPTY
    assert covered[: H // 2 - 1].all()   # rows below the horizon (row 0 = bottom)
    assert not covered[H // 2 + 1:].any()


def test_oracle_forward_resolve_is_finite_and_lit():
    s = icosphere_field(n_spheres=6, subdiv=1, floor_cells=2, seed=3)
    W, H = 40, 32
    view, proj = view_projection((0, 1.0, -4.0), (0, -0.3, 0), vfov_deg=50, aspect=W / H)
    sv, sp = forward_default_shadow()
    out = po.forward_render(s, W, H, view, proj, 7, 64, sv, sp)
    res = out["result"]
    assert np.isfinite(res).all()
    fg = out["visibility"] != EMPTY
    assert fg.any() and (~fg).any()
    assert (res[..., 3][fg] == 0).all() and (res[..., 3][~fg] == 1).all()
    assert res[fg][:, :3].mean() > 0.01


@pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("seed,eye", [(7, (0, 1.0, -4.0)), (123456789, (1.5, 0.4, -2.5))])
def test_resolve_pinned_to_the_reference_shader(seed, eye):
    """The oracle's resolve pass equals the reference's own resolve.frag
    (compiled as C++ by oracle/build_ref.py) run on the same G-buffer and
    shadow map, bit for bit after the RGBA16F store."""
    s = icosphere_field(n_spheres=8, subdiv=1, floor_cells=2, seed=3)
    W, H = 48, 36
    view, proj = view_projection(eye, (0, -0.3, 0), vfov_deg=55, aspect=W / H)
    sv, sp = forward_default_shadow()
    out = po.forward_render(s, W, H, view, proj, seed, 256, sv, sp)
    ref = po.ref_forward_resolve(out["gbuffer"], out["shadow_map"], view, proj, sv, sp, seed, s["materials"],
                                 s["material_data"])
    ref16 = ref.astype(np.float16).astype(np.float32)
    fg = out["visibility"] != EMPTY
    assert fg.mean() > 0.2
    assert np.array_equal(out["result"], ref16, equal_nan=True)
