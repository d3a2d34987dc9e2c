"""Seeded synthetic scenes and ray sets for the benchmark configurations.

All inputs are synthetic: no dataset or asset is read. Geometry is float32,
built in float64 and rounded once, so every machine produces identical bits.

* ``heightfield``  -- N x N cell grid on [-1,1]^2 in xz, vertex y ~ U[0, amp),
  two triangles per cell (the 128 x 128 / 32,768-triangle closest-hit case).
* ``icosphere_field`` -- random icospheres plus a tessellated floor quad (the
  655,872-triangle path-tracing case).
* ``pinhole_rays`` -- one ray per pixel centre of a pinhole camera.
"""
from __future__ import annotations

import numpy as np


def heightfield(n: int = 128, amp: float = 0.1, seed: int = 1):
    """Return (indices uint32[3T], points float32[V,3]) for an n x n cell grid."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(-1.0, 1.0, n + 1)
    gx, gz = np.meshgrid(xs, xs, indexing="xy")
    gy = rng.uniform(0.0, amp, size=gx.shape)
    pts = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1).astype(np.float32)
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="xy")
    v00 = (j * (n + 1) + i).ravel()
    v10 = v00 + 1
    v01 = v00 + (n + 1)
    v11 = v01 + 1
    tris = np.stack([np.stack([v00, v01, v10], 1), np.stack([v10, v01, v11], 1)], axis=1).reshape(-1, 3)
    return tris.astype(np.uint32).ravel(), pts


def pinhole_rays(width: int, height: int, eye=(0.0, 2.0, -3.0), target=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0),
                 vfov_deg: float = 60.0, jitter: np.ndarray | None = None) -> np.ndarray:
    """Rays through pixel centres (row-major, y down), as float32[n, 8]:
    origin xyz, tmin (0), direction xyz (unit), tmax (+inf)."""
    eye = np.asarray(eye, np.float64)
    fwd = np.asarray(target, np.float64) - eye
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, np.asarray(up, np.float64))
    right /= np.linalg.norm(right)
    upv = np.cross(right, fwd)
    tan_half = np.tan(np.radians(vfov_deg) * 0.5)
    aspect = width / height
    px, py = np.meshgrid(np.arange(width, dtype=np.float64), np.arange(height, dtype=np.float64), indexing="xy")
    px = px.ravel() + 0.5
    py = py.ravel() + 0.5
    if jitter is not None:
        px = px + jitter[:, 0]
        py = py + jitter[:, 1]
    sx = (2.0 * px / width - 1.0) * tan_half * aspect
    sy = (1.0 - 2.0 * py / height) * tan_half
    d = fwd[None, :] + sx[:, None] * right[None, :] + sy[:, None] * upv[None, :]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.empty((d.shape[0], 8), np.float32)
    rays[:, 0:3] = eye
    rays[:, 3] = 0.0
    rays[:, 4:7] = d
    rays[:, 7] = np.inf
    return rays


def icosphere(subdiv: int = 3):
    """Unit icosphere: (indices uint32[3T], points float32[V,3]); 20 * 4**subdiv triangles."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.asarray(faces, np.uint32).ravel(), np.asarray(verts, np.float64).astype(np.float32)


def pack_unorm4x8(rgba) -> np.uint32:
    c = np.clip(np.asarray(rgba, np.float64), 0.0, 1.0)
    b = np.rint(c * 255.0).astype(np.uint32)
    return np.uint32(b[0] | (b[1] << 8) | (b[2] << 16) | (b[3] << 24))


def pbr_material(albedo, ior=1.5, roughness=0.5, metallic=0.0, transmission=0.0) -> np.ndarray:
    """The reference app's 7-float PBR record (src/main.cpp:447-464): albedo as
    vec4unorm8 bits, ior, roughness, metallic, transmission, albedo texture (0, 0)."""
    rec = np.zeros(7, np.float32)
    rec[0] = pack_unorm4x8([*albedo, 1.0]).view(np.float32)
    rec[1:5] = ior, roughness, metallic, transmission
    return rec


def _affine(scale: float, t) -> tuple[np.ndarray, np.ndarray]:
    m = np.zeros(16, np.float32)
    m[0] = m[5] = m[10] = scale
    m[12:15] = t
    m[15] = 1.0
    inv = np.zeros(16, np.float32)
    inv[0] = inv[5] = inv[10] = 1.0 / scale
    inv[12:15] = -np.asarray(t, np.float64) / scale
    inv[15] = 1.0
    return m, inv


def icosphere_field(n_spheres: int = 512, subdiv: int = 3, floor_cells: int = 16, seed: int = 2):
    """Random icospheres (radius log-uniform [0.02, 0.2], centres U[-1,1]^3) plus
    a floor quad at y = -1.2 tessellated into 2 * floor_cells^2 triangles, as
    instanced drawables with one material each (GGX roughness U[0.05, 1],
    albedo U[0.2, 0.9]^3, metallic Bernoulli(0.3)). Default: 512 * 1280 + 512
    = 655,872 triangles. Returns a dict of Context.upload_scene arguments."""
    from ._abi import myrt_drawable

    rng = np.random.default_rng(seed)
    si, sp = icosphere(subdiv)
    # floor: unit grid on [-3,3]^2 at y = -1.2
    g = np.linspace(-3.0, 3.0, floor_cells + 1)
    gx, gz = np.meshgrid(g, g, indexing="xy")
    fp = np.stack([gx.ravel(), np.full(gx.size, -1.2), gz.ravel()], 1).astype(np.float32)
    i, j = np.meshgrid(np.arange(floor_cells), np.arange(floor_cells), indexing="xy")
    v00 = (j * (floor_cells + 1) + i).ravel()
    fi = np.stack([np.stack([v00, v00 + floor_cells + 1, v00 + 1], 1),
                   np.stack([v00 + 1, v00 + floor_cells + 1, v00 + floor_cells + 2], 1)], 1).reshape(-1)
    indices = np.concatenate([si, fi.astype(np.uint32)])
    vertices = np.concatenate([sp, fp]).astype(np.float32)
    normals = np.concatenate([sp, np.tile(np.array([[0.0, 1.0, 0.0]], np.float32), (fp.shape[0], 1))])
    radius = np.exp(rng.uniform(np.log(0.02), np.log(0.2), n_spheres))
    centre = rng.uniform(-1.0, 1.0, (n_spheres, 3))
    rough = rng.uniform(0.05, 1.0, n_spheres)
    albedo = rng.uniform(0.2, 0.9, (n_spheres, 3))
    metal = (rng.uniform(0.0, 1.0, n_spheres) < 0.3).astype(np.float32)
    drawables = (myrt_drawable * (n_spheres + 1))()
    mat_data = [pbr_material([0.6, 0.6, 0.6], roughness=0.8)]
    for k in range(n_spheres):
        m, inv = _affine(float(radius[k]), centre[k])
        d = drawables[k]
        d.transformation[:] = m.tolist()
        d.inverse_transformation[:] = inv.tolist()
        d.indices_base_index, d.points_base_index, d.index_count = 0, 0, si.size
        d.material_index = k + 1
        mat_data.append(pbr_material(albedo[k], roughness=float(rough[k]), metallic=float(metal[k])))
    fl = drawables[n_spheres]
    fl.transformation[:] = _affine(1.0, (0, 0, 0))[0].tolist()
    fl.inverse_transformation[:] = _affine(1.0, (0, 0, 0))[1].tolist()
    fl.indices_base_index, fl.points_base_index, fl.index_count = si.size, sp.shape[0], fi.size
    fl.material_index = 0
    mat_data = np.stack(mat_data)
    materials = np.stack([np.zeros(len(mat_data), np.int32), np.arange(len(mat_data), dtype=np.int32) * 7], 1)
    return dict(indices=indices, vertices=vertices, normals=normals, drawables=drawables, materials=materials,
                material_data=mat_data.ravel())


_GOLDEN64 = np.uint64(0x9E3779B97F4A7C15)


def counter_uniform(index: np.ndarray, stream: int, seed: int = 0) -> np.ndarray:
    """Uniform float64 numbers in [0, 1), one per entry of `index`, as a pure
    function of (seed, index, stream): the SplitMix64 output function (Steele,
    Lea and Flood, OOPSLA 2014) over the counter 8 * index + stream. Any
    subset of a ray batch can be regenerated exactly from its indices."""
    with np.errstate(over="ignore"):
        z = (np.asarray(index, np.uint64) * np.uint64(8) + np.uint64(stream & 7) + np.uint64(seed) * np.uint64(1 << 40)
             + np.uint64(1)) * _GOLDEN64
        z ^= z >> np.uint64(30)
        z *= np.uint64(0xBF58476D1CE4E5B9)
        z ^= z >> np.uint64(27)
        z *= np.uint64(0x94D049BB133111EB)
        z ^= z >> np.uint64(31)
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))


def _unit(v: np.ndarray) -> np.ndarray:
    return v / np.sqrt(v[..., 0] * v[..., 0] + v[..., 1] * v[..., 1] + v[..., 2] * v[..., 2])[..., None]


ICOSPHERE_EYE, ICOSPHERE_TARGET, ICOSPHERE_VFOV = (0.0, 1.0, -4.5), (0.0, -0.3, 0.0), 50.0


def jittered_camera_rays(index: np.ndarray, res: int, seed: int = 1000) -> np.ndarray:
    """Camera rays of a res x res view of the icosphere scene, ray `i` through
    pixel i mod res^2 (row-major, y down) at a uniformly jittered position
    inside it (sample i div res^2), float32 [len(index), 8]. Rays depend only on
    (index, res, seed), so a sample of indices gives exactly the same rays as
    the full batch."""
    index = np.asarray(index, np.int64)
    eye = np.asarray(ICOSPHERE_EYE, np.float64)
    fwd = _unit(np.asarray(ICOSPHERE_TARGET, np.float64) - eye)
    right = _unit(np.cross(fwd, np.array([0.0, 1.0, 0.0])))
    up = np.cross(right, fwd)
    tan_half = np.tan(np.radians(ICOSPHERE_VFOV) / 2)
    pix = index % (res * res)
    px = (pix % res) + counter_uniform(index, 0, seed)
    py = (pix // res) + counter_uniform(index, 1, seed)
    sx = (2.0 * px / res - 1.0) * tan_half
    sy = (1.0 - 2.0 * py / res) * tan_half
    d = _unit(fwd[None] + sx[:, None] * right[None] + sy[:, None] * up[None])
    rays = np.empty((index.size, 8), np.float32)
    rays[:, 0:3] = eye
    rays[:, 3] = 0.0
    rays[:, 4:7] = d
    rays[:, 7] = np.inf
    return rays


def diffuse_bounce_rays(rays: np.ndarray, prim: np.ndarray, t: np.ndarray, tris9: np.ndarray, index: np.ndarray,
                        seed: int = 1000) -> np.ndarray:
    """The first diffuse bounce of each hit ray: origin at the hit point moved
    1e-4 along the face normal turned toward the ray, cosine-distributed
    direction about that normal (random numbers from the parent ray's index).
    rays float32 [n, 8], prim int32 [n] (hits only, >= 0), t float32 [n],
    tris9 float32 [T, 9] world triangles by prim id. Returns float32 [n, 8]."""
    tri = tris9[prim].astype(np.float64).reshape(-1, 3, 3)
    n = _unit(np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]))
    d = rays[:, 4:7].astype(np.float64)
    n = np.where(((n * d).sum(1) > 0)[:, None], -n, n)
    p = rays[:, 0:3].astype(np.float64) + t.astype(np.float64)[:, None] * d
    u1 = counter_uniform(index, 2, seed)
    u2 = counter_uniform(index, 3, seed)
    a = np.where((np.abs(n[:, 0]) > 0.9)[:, None], np.array([0.0, 1.0, 0.0]), np.array([1.0, 0.0, 0.0]))
    tt = _unit(np.cross(n, a))
    b = np.cross(n, tt)
    r = np.sqrt(u1)
    phi = 2.0 * np.pi * u2
    wd = _unit((r * np.cos(phi))[:, None] * tt + (r * np.sin(phi))[:, None] * b
               + np.sqrt(np.maximum(1.0 - u1, 0.0))[:, None] * n)
    out = np.empty((prim.size, 8), np.float32)
    out[:, 0:3] = p + 1e-4 * n
    out[:, 3] = 0.0
    out[:, 4:7] = wd
    out[:, 7] = np.inf
    return out


def world_triangles(scene: dict) -> np.ndarray:
    """World-space triangles float32 [T, 9] of an upload_scene argument dict,
    in the library's prim numbering (drawables in order, triangles in index
    order), each corner transformed in float64 and rounded once."""
    idx = scene["indices"].astype(np.int64)
    v = scene["vertices"].astype(np.float64).reshape(-1, 3)
    out = []
    for d in scene["drawables"]:
        m = np.array(d.transformation[:], np.float64).reshape(4, 4).T
        sel = idx[d.indices_base_index: d.indices_base_index + d.index_count] + d.points_base_index
        p = v[sel] @ m[:3, :3].T + m[:3, 3]
        out.append(p.reshape(-1, 9))
    return np.concatenate(out).astype(np.float32)


def _rotation(axis, angle) -> np.ndarray:
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    c, s = np.cos(angle), np.sin(angle)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + s * K + (1 - c) * (K @ K)


def exponential_chain(ratio: float = 1.2, k0: int = -450, k1: int = 480) -> np.ndarray:
    """A degenerate scene: triangles k = k0 .. k1-1 at x = ratio^k along the x
    axis, each 0.3 x its distance from the origin in size (those that overflow
    float32 are dropped). Every SAH split cuts off only a few triangles, so the
    tree grows about one level per few triangles: with the defaults, deeper
    than the traversal stack allows (32 wide levels). float32 [T, 9]."""
    k = np.arange(k0, k1, dtype=np.float64)
    x = ratio ** k
    s = 0.3 * x
    z = np.zeros_like(x)
    t = np.stack([x, z, z, x + s, z, z, x, s, z], 1)
    keep = np.isfinite(t).all(1) & (np.abs(t).max(1) < 1e37)
    return t[keep].astype(np.float32)


def unit_box():
    """Axis-aligned cube [-1, 1]^3 as 12 triangles: (indices uint32, points float32)."""
    p = np.array([[x, y, z] for z in (-1, 1) for y in (-1, 1) for x in (-1, 1)], np.float32)
    quads = [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]
    tri = []
    for a, b, c, d in quads:
        tri += [a, b, c, a, c, d]
    return np.array(tri, np.uint32), p


def instanced_field(n_spheres: int = 48, n_boxes: int = 24, subdiv: int = 2, floor_cells: int = 8, seed: int = 21):
    """Instances with general affine transforms: icospheres and boxes under
    random rotations, non-uniform scales (0.05-0.3 per axis) and translations in
    [-1, 1]^3, plus a floor grid at y = -1.2 drawn with an identity transform.
    Each drawable's inverse_transformation is its transformation inverted in
    float64 and rounded to float32. Returns upload_scene arguments."""
    from ._abi import myrt_drawable

    rng = np.random.default_rng(seed)
    si, sp = icosphere(subdiv)
    bi, bp = unit_box()
    g = np.linspace(-3.0, 3.0, floor_cells + 1)
    gx, gz = np.meshgrid(g, g, indexing="xy")
    fp = np.stack([gx.ravel(), np.full(gx.size, -1.2), gz.ravel()], 1).astype(np.float32)
    i, j = np.meshgrid(np.arange(floor_cells), np.arange(floor_cells), indexing="xy")
    v00 = (j * (floor_cells + 1) + i).ravel()
    fi = np.stack([np.stack([v00, v00 + floor_cells + 1, v00 + 1], 1),
                   np.stack([v00 + 1, v00 + floor_cells + 1, v00 + floor_cells + 2], 1)], 1).reshape(-1)
    indices = np.concatenate([si, bi, fi.astype(np.uint32)])
    vertices = np.concatenate([sp, bp, fp]).astype(np.float32)
    normals = np.concatenate([sp, bp / np.linalg.norm(bp, axis=1, keepdims=True),
                              np.tile(np.array([[0.0, 1.0, 0.0]], np.float32), (fp.shape[0], 1))]).astype(np.float32)
    geo = [(0, 0, si.size), (si.size, sp.shape[0], bi.size), (si.size + bi.size, sp.shape[0] + bp.shape[0], fi.size)]
    kinds = [0] * n_spheres + [1] * n_boxes
    drawables = (myrt_drawable * (len(kinds) + 1))()
    for k, kind in enumerate(kinds):
        R = _rotation(rng.normal(size=3), rng.uniform(0, 2 * np.pi))
        S = np.diag(rng.uniform(0.05, 0.3, 3))
        M = np.eye(4)
        M[:3, :3] = R @ S
        M[:3, 3] = rng.uniform(-1.0, 1.0, 3)
        m32 = M.astype(np.float32)
        inv = np.linalg.inv(m32.astype(np.float64)).astype(np.float32)
        d = drawables[k]
        d.transformation[:] = m32.T.ravel().tolist()  # column-major
        d.inverse_transformation[:] = inv.T.ravel().tolist()
        d.indices_base_index, d.points_base_index, d.index_count = geo[kind]
        d.material_index = 0
    fl = drawables[len(kinds)]
    eye = np.eye(4, dtype=np.float32).ravel().tolist()
    fl.transformation[:] = eye
    fl.inverse_transformation[:] = eye
    fl.indices_base_index, fl.points_base_index, fl.index_count = geo[2]
    mat = np.array([[0, 0]], np.int32)
    return dict(indices=indices, vertices=vertices, normals=normals, drawables=drawables, materials=mat,
                material_data=pbr_material([0.6, 0.6, 0.6], roughness=0.8))


def icosphere_camera_rays(width: int = 512, height: int = 512, spp: int = 1, seed: int = 5) -> np.ndarray:
    """Camera rays of the icosphere scene; spp > 1 adds sub-pixel jitter."""
    rng = np.random.default_rng(seed)
    out = []
    for s in range(spp):
        jit = None if spp == 1 else rng.uniform(-0.5, 0.5, (width * height, 2))
        out.append(pinhole_rays(width, height, eye=(0.0, 1.0, -4.5), target=(0.0, -0.3, 0.0), vfov_deg=50.0,
                                jitter=jit))
    return np.concatenate(out, 0)


def area_light(center, size, emission) -> np.ndarray:
    """Square light of side `size` centred at `center`, facing -y (down):
    one [12] row (corner, edge_u, edge_v, emission) for set_area_lights."""
    c = np.asarray(center, np.float32)
    h = np.float32(size) / 2
    row = np.zeros(12, np.float32)
    row[0:3] = c - np.array([h, 0, h], np.float32)
    row[3:6] = [size, 0, 0]
    row[6:9] = [0, 0, size]
    row[9:12] = np.broadcast_to(np.asarray(emission, np.float32), 3)
    return row


def icosphere_field_lit(n_spheres: int = 512, subdiv: int = 3, floor_cells: int = 16, seed: int = 2):
    """The icosphere field plus its one 0.2 x 0.2 ceiling light of emission 20
    at y = 1.6 (above every sphere), facing down: (scene, lights[1, 12])."""
    s = icosphere_field(n_spheres=n_spheres, subdiv=subdiv, floor_cells=floor_cells, seed=seed)
    return s, area_light((0.0, 1.6, 0.0), 0.2, 20.0)[None, :]


def _grid(nu: int, nv: int, origin, eu, ev, height=None, up=None):
    """nu x nv quads spanning origin + [0,1] eu + [0,1] ev (2 triangles each,
    wound so that cross(eu, ev) is the front side), optionally displaced by
    height[(nv+1), (nu+1)] along `up`. Returns (indices, vertices)."""
    u = np.linspace(0.0, 1.0, nu + 1)
    v = np.linspace(0.0, 1.0, nv + 1)
    uu, vv = np.meshgrid(u, v)
    pts = (np.asarray(origin, np.float64)[None, None] + uu[..., None] * np.asarray(eu, np.float64) +
           vv[..., None] * np.asarray(ev, np.float64))
    if height is not None:
        pts = pts + height[..., None] * np.asarray(up, np.float64)
    pts = pts.reshape(-1, 3).astype(np.float32)
    i = np.arange(nv)[:, None] * (nu + 1) + np.arange(nu)[None, :]
    a, b, c, d = i, i + 1, i + nu + 2, i + nu + 1
    idx = np.stack([a, b, c, a, c, d], -1).reshape(-1).astype(np.uint32)
    return idx, pts


def guiding_box(slab_cells: int = 708, wall_cells: int = 8, seed: int = 7, plate: float = 0.5,
                plate_y: float = 0.75, gap: float = 0.2, light_x: float = 0.0):
    """Indirect-dominated scene: the closed box [-1,1]^3 (walls facing
    inwards), two displaced occluder slabs of 2 * slab_cells^2 triangles each
    (height U[0, 0.05]; default 1,002,528 each) and a 0.05 x 0.05 ceiling light
    (emission 400) at (light_x, 0.995, 0) hidden behind a plate x plate
    occluder at y = plate_y (default 0.5 x 0.5 at y = 0.75): the light lands on
    the plate and the upper walls, the plate throws it onto the ceiling, and
    the room is lit mostly by that bright ceiling. Slab 1 (y = 0.3) leaves a
    slot of width `gap` at x = +1, slab 2 (y = -0.3) one at x = -1, so light
    reaches the middle and bottom levels only through those slots. Returns
    (scene, lights[1, 12])."""
    rng = np.random.default_rng(seed)
    parts = []  # (indices, vertices, material)
    n = wall_cells
    walls = [  # origin, eu, ev with cross(eu, ev) pointing into the box
        ((-1, -1, -1), (2, 0, 0), (0, 0, 2)),   # floor, +y
        ((-1, 1, -1), (0, 0, 2), (2, 0, 0)),    # ceiling, -y
        ((-1, -1, -1), (0, 2, 0), (2, 0, 0)),   # back z = -1, +z
        ((-1, -1, 1), (2, 0, 0), (0, 2, 0)),    # front z = +1, -z
        ((-1, -1, -1), (0, 0, 2), (0, 2, 0)),   # x = -1, +x
        ((1, -1, -1), (0, 2, 0), (0, 0, 2)),    # x = +1, -x
    ]
    for k, (o, eu, ev) in enumerate(walls):
        idx, pts = _grid(n, n, o, eu, ev)
        parts.append((idx, pts, 0 if k != 4 else 1))
    for (x0, x1, y) in ((-1.0, 1.0 - gap, 0.3), (-1.0 + gap, 1.0, -0.3)):
        h = rng.uniform(0.0, 0.05, (slab_cells + 1, slab_cells + 1))
        idx, pts = _grid(slab_cells, slab_cells, (x0, y, -1.0), (0, 0, 2.0), (x1 - x0, 0, 0), h, (0, 1, 0))
        parts.append((idx, pts, 2))
    # the occluder plate under the light (a thin double-sided sheet)
    idx, pts = _grid(1, 1, (light_x - plate / 2, plate_y, -plate / 2), (0, 0, plate), (plate, 0, 0))
    parts.append((idx, pts, 0))
    from ._abi import myrt_drawable

    indices, vertices = [], []
    drawables = (myrt_drawable * len(parts))()
    eye = np.eye(4, dtype=np.float32).ravel().tolist()
    ioff = voff = 0
    for k, (idx, pts, mat) in enumerate(parts):
        indices.append(idx)
        vertices.append(pts)
        d = drawables[k]
        d.transformation[:] = eye
        d.inverse_transformation[:] = eye
        d.indices_base_index, d.points_base_index, d.index_count = ioff, voff, idx.size
        d.material_index = mat
        ioff += idx.size
        voff += pts.shape[0]
    mat_data = np.concatenate([pbr_material([0.75, 0.75, 0.75], ior=1.5, roughness=0.9),
                               pbr_material([0.75, 0.3, 0.25], ior=1.5, roughness=0.7),
                               pbr_material([0.6, 0.65, 0.7], ior=1.5, roughness=0.4)])
    materials = np.array([[0, 0], [0, 7], [0, 14]], np.int32)
    scene = dict(indices=np.concatenate(indices), vertices=np.concatenate(vertices), drawables=drawables,
                 materials=materials, material_data=mat_data)
    light = area_light((light_x, 0.995, 0.0), 0.05, 400.0)[None, :]
    return scene, light


def heightfield_scene(n: int, seed: int = 1, albedo=(0.7, 0.6, 0.5), roughness: float = 0.4):
    """The n x n height field (2 n^2 triangles) with one PBR material and a
    0.5 x 0.5 area light (emission 12) at y = 1.5: (scene, lights[1, 12])."""
    idx, pts = heightfield(n, seed=seed)
    s = dict(indices=idx, vertices=pts, materials=np.array([[0, 0]], np.int32),
             material_data=pbr_material(list(albedo), ior=1.5, roughness=roughness))
    return s, area_light((0.0, 1.5, 0.0), 0.5, 12.0)[None, :]


def uneven_batch(n_scenes: int = 16, seed: int = 11, tri_range=(1e4, 2e6)):
    """Batched uneven scenes: n_scenes height-field / icosphere scenes with
    triangle counts log-uniform in tri_range, one view each at a resolution
    from {128, 256, 512, 1024}^2 and 4-64 spp. Returns (scenes, jobs):
    scenes = [(scene, lights, triangles)], jobs = Batch job dicts (without the
    camera matrices' numpy conversion; keys as myrt_b200.Batch expects)."""
    from .camera import look_at

    rng = np.random.default_rng(seed)
    scenes, jobs = [], []
    for k in range(n_scenes):
        tris = float(np.exp(rng.uniform(np.log(tri_range[0]), np.log(tri_range[1]))))
        res = int(rng.choice([128, 256, 512, 1024]))
        spp = int(rng.integers(4, 65))
        if k % 2 == 0:
            n = max(2, int(round(np.sqrt(tris / 2))))
            s, lights = heightfield_scene(n, seed=100 + k)
            count = 2 * n * n
            eye, tgt, vfov = (0.0, 1.5, -2.5), (0.0, 0.0, 0.0), 60.0
        else:
            spheres = max(1, int(round((tris - 512) / 1280)))
            s, lights = icosphere_field_lit(n_spheres=spheres, seed=200 + k)
            count = 1280 * spheres + 512
            eye, tgt, vfov = (0.0, 1.0, -4.5), (0.0, -0.3, 0.0), 50.0
        iv, ip = look_at(eye, tgt, vfov_deg=vfov, aspect=1.0)
        scenes.append((s, lights, count))
        jobs.append(dict(scene=k, width=res, height=res, spp=spp, seed=1000 + k, max_depth=8, rr_start=3,
                         inverse_view=iv, inverse_projection=ip))
    return scenes, jobs
