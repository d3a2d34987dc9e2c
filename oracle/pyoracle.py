"""ctypes front end of the CPU oracle (liboracle.so) and, when built, of the
reference's own code compiled here (_ref/libmyrt_ref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and bench.py's
CPU-baseline leg, as the checker. The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libmyrt_ref.so"

P = C.c_void_p
SZ = C.c_size_t
I = C.c_int

_orc = None
_ref = None


def oracle() -> C.CDLL:
    global _orc
    if _orc is None:
        if not ORACLE_LIB.exists():
            raise RuntimeError(f"{ORACLE_LIB} is missing: run `python oracle/build.py`")
        h = C.CDLL(str(ORACLE_LIB))
        sig = {
            "orc_isect_reference": (I, [P, P, P, P, P]),
            "oracle_post_pass": (I, [I, P, P, P, I, I, P, I, I, P, I, I]),
            "oracle_half_rn": (C.c_float, [C.c_float]),
            "orc_refbvh_build": (P, [P, SZ, P]),
            "orc_refbvh_free": (None, [P]),
            "orc_refbvh_node_count": (SZ, [P]),
            "orc_refbvh_nodes": (None, [P, P]),
            "orc_refbvh_indices": (None, [P, P]),
            "orc_refbvh_traverse": (None, [P, P, P, P, P, SZ, I, I, P, P, P, P, I]),
            "orc_bvh8_traverse": (None, [P, P, P, SZ, I, I, P, P, P, P, P, P, P, I]),
            "orc_brute_closest": (None, [P, SZ, P, SZ, I, P, P, P, P, I]),
            "orc_instanced_query": (None, [P, P, P, P, P, SZ, P, SZ, I, I, P, P, P, P, I]),
            "orc_set_glsl_math": (None, [I]),
            "orc_glsl_eval": (None, [I, P, P, SZ, P]),
            "orc_host_rng": (None, [C.c_uint32, I, I, P, P]),
            "orc_render_reference": (None, [SZ, P, P, P, P, P, SZ, P, P, P, I, I, I, I, C.c_uint32, P, P, P, P, P,
                                            P, P, P, P, P, I, I, C.c_float, I, I, P, P, P, I, I, C.c_float,
                                            C.c_float, C.c_float, I]),
            "orc_random_stream": (None, [P, I, I, I, I, I, P, P]),
            "orc_wang_hash": (C.c_uint32, [C.c_uint32]),
            "orc_transform_local_to_world": (None, [P, P, P]),
            "orc_pack_unorm4x8": (C.c_uint32, [P]),
            "orc_intersect_sphere": (C.c_float, [P, P, P, C.c_float]),
            "orc_material_bounce_eval": (None, [P, P, P, P, P, P, P, P, P]),
            "orc_material_eval": (None, [P, I, C.c_float, P, P, P, P, P]),
            "orc_sdf_map": (None, [P, P, P, I, P, SZ, I, P, P, P]),
            "orc_sdf_trace": (None, [P, P, P, P, I, P, SZ, I, C.c_float, I, P, P, P, P, P, P, I]),
            "orc_render_physical": (None, [SZ, P, P, P, P, SZ, P, P, P, P, I, P, I, I, I, C.c_uint32, I, I,
                                           C.c_uint32, P, P, P, P, P, P, I, I, C.c_float, I, P, I]),
            "orc_refbvh_query": (None, [P, P, P, P, P, SZ, I, I, I, P, P, P, P, I]),
            "orc_pass_color": (None, [I, P, P, P, P, I, I, C.c_uint32, I, I, P, I, P, I, P]),
            "orc_pass_generate": (None, [I, I, P, P, I, P, I, I, C.c_float, C.c_float, C.c_float, P, I, I, I, P]),
            "orc_forward_render": (None, [I, P, P, P, P, P, I, P, I, I, P, P, C.c_uint32, I, P, P, I, P, P, P, P, P,
                                          P, P]),
        }
        for k, (r, a) in sig.items():
            f = getattr(h, k)
            f.restype, f.argtypes = r, a
        _orc = h
    return _orc


def ref_available() -> bool:
    return REF_LIB.exists()


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        h = C.CDLL(str(REF_LIB))
        sig = {
            "ref_bvh_build": (P, [P, SZ, P, SZ, I]),
            "ref_bvh_free": (None, [P]),
            "ref_bvh_aabb": (None, [P, P]),
            "ref_bvh_build_instances": (P, [P, P, SZ]),
            "ref_glsl_traverse_instanced": (None, [P, P, P, P, P, P, P, P, SZ, I, P, P, P, P, P, I]),
            "ref_bvh_node_count": (SZ, [P]),
            "ref_bvh_index_count": (SZ, [P]),
            "ref_bvh_nodes": (None, [P, P]),
            "ref_bvh_indices": (None, [P, P]),
            "ref_pick_closest": (None, [P, P, SZ, P, P, P, P, I]),
            "ref_glsl_traverse": (None, [P, P, P, P, P, SZ, I, P, P, P, P, I]),
            "ref_glsl_wang_hash": (C.c_uint32, [C.c_uint32]),
            "ref_glsl_random_stream": (None, [P, I, I, I, I, I, P, P]),
            "ref_glsl_random_values": (None, [C.c_uint32, P, I, P, P]),
            "ref_glsl_intersect_triangle": (I, [P, P, P, P, P]),
            "ref_glsl_intersect_sphere": (C.c_float, [P, P, P, C.c_float]),
            "ref_glsl_transform_local_to_world": (None, [P, P, P]),
            "ref_glsl_pack_unorm4x8": (C.c_uint32, [P]),
            "ref_glsl_material_bounce_eval": (None, [P, P, P, P, P, P, P, P, P]),
            "ref_glsl_material_eval": (None, [P, I, C.c_float, P, P, P, P, P]),
            "ref_sdf_map": (None, [P, P, P, I, P, SZ, I, P, P, P]),
            "ref_sdf_trace": (None, [P, P, P, P, I, P, SZ, I, C.c_float, I, P, P, P, P, P, P]),
            "ref_post_pass": (I, [I, P, P, P, I, I, P, I, I, P]),
            "ref_forward_resolve": (None, [I, I, P, P, I, P, P, P, P, C.c_uint32, P, P, P]),
            "ref_pass_color": (None, [I, P, P, P, P, I, I, C.c_uint32, I, I, P, I, P, P]),
            "ref_pass_generate": (None, [I, I, P, P, I, P, I, I, C.c_float, C.c_float, C.c_float, P, I, I, I, P]),
        }
        for k, (r, a) in sig.items():
            f = getattr(h, k)
            f.restype, f.argtypes = r, a
        _ref = h
    return _ref


def nthreads() -> int:
    return os.cpu_count() or 1


def _hits(n):
    return np.empty(n, np.int32), np.empty(n, np.float32), np.empty(n, np.float32), np.empty(n, np.float32)


def _pack(prim, t, u, v):
    out = np.empty(prim.size, [("prim", np.int32), ("t", np.float32), ("u", np.float32), ("v", np.float32)])
    out["prim"], out["t"], out["u"], out["v"] = prim, t, u, v
    return out


# ---- oracle restatement -----------------------------------------------------
def refbvh_build(indices: np.ndarray, points: np.ndarray):
    """Restated reference build (dont_split). Returns (nodes uint32[N,12], bvh_indices)."""
    L = oracle()
    idx = np.ascontiguousarray(indices, np.uint32)
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    h = L.orc_refbvh_build(idx.ctypes.data, idx.size, pts.ctypes.data)
    try:
        n = L.orc_refbvh_node_count(h)
        nodes = np.zeros((n, 12), np.uint32)
        L.orc_refbvh_nodes(h, nodes.ctypes.data)
        bi = np.zeros(idx.size // 3, np.uint32)
        L.orc_refbvh_indices(h, bi.ctypes.data)
        return nodes, bi
    finally:
        L.orc_refbvh_free(h)


def refbvh_traverse(nodes, bvh_indices, indices, points, rays, any_hit=False, canonical=True):
    L = oracle()
    p4 = np.zeros((points.shape[0], 4), np.float32)
    p4[:, :3] = points
    r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    out = _hits(r.shape[0])
    nodes = np.ascontiguousarray(nodes)
    bvh_indices = np.ascontiguousarray(bvh_indices, np.uint32)
    indices = np.ascontiguousarray(indices, np.uint32)
    L.orc_refbvh_traverse(nodes.ctypes.data, bvh_indices.ctypes.data, indices.ctypes.data, p4.ctypes.data,
                          r.ctypes.data, r.shape[0], int(any_hit), int(canonical), *[o.ctypes.data for o in out],
                          nthreads())
    return _pack(*out)


def bvh8_traverse(nodes, tris, rays, isect=0, any_hit=False):
    """The device algorithm on the CPU. Returns (hits, n_nodes, n_tris[, occluded])."""
    L = oracle()
    r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    n = r.shape[0]
    out = _hits(n)
    cn = np.zeros(n, np.uint32)
    ct = np.zeros(n, np.uint32)
    occ = np.zeros(n, np.uint8)
    nodes = np.ascontiguousarray(nodes, np.uint32)
    tris = np.ascontiguousarray(tris, np.float32)
    L.orc_bvh8_traverse(nodes.ctypes.data, tris.ctypes.data, r.ctypes.data, n, int(any_hit), int(isect),
                        *[o.ctypes.data for o in out], cn.ctypes.data, ct.ctypes.data, occ.ctypes.data, nthreads())
    if any_hit:
        return occ, cn, ct
    return _pack(*out), cn, ct


def brute_closest(tris9: np.ndarray, rays: np.ndarray, isect=0):
    L = oracle()
    t9 = np.ascontiguousarray(tris9, np.float32).reshape(-1, 9)
    r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    out = _hits(r.shape[0])
    L.orc_brute_closest(t9.ctypes.data, t9.shape[0], r.ctypes.data, r.shape[0], int(isect),
                        *[o.ctypes.data for o in out], nthreads())
    return _pack(*out)


# ---- the reference's own code (oracle/_ref) -----------------------------------
def ref_bvh(indices, points, split: bool):
    L = ref()
    idx = np.ascontiguousarray(indices, np.uint32)
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    h = L.ref_bvh_build(idx.ctypes.data, idx.size, pts.ctypes.data, pts.shape[0], int(split))
    return h


def ref_bvh_arrays(h):
    L = ref()
    nodes = np.zeros((L.ref_bvh_node_count(h), 12), np.uint32)
    L.ref_bvh_nodes(h, nodes.ctypes.data)
    bi = np.zeros(L.ref_bvh_index_count(h), np.uint32)
    L.ref_bvh_indices(h, bi.ctypes.data)
    return nodes, bi


def ref_pick_closest(h, rays, threads=None):
    L = ref()
    r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    out = _hits(r.shape[0])
    L.ref_pick_closest(h, r.ctypes.data, r.shape[0], *[o.ctypes.data for o in out], threads or nthreads())
    return _pack(*out)


def ref_glsl_traverse(nodes, bvh_indices, indices, points, rays, any_hit=False, threads=None):
    L = ref()
    p4 = np.zeros((points.shape[0], 4), np.float32)
    p4[:, :3] = points
    r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    out = _hits(r.shape[0])
    nodes = np.ascontiguousarray(nodes)
    bvh_indices = np.ascontiguousarray(bvh_indices, np.uint32)
    indices = np.ascontiguousarray(indices, np.uint32)
    L.ref_glsl_traverse(nodes.ctypes.data, bvh_indices.ctypes.data, indices.ctypes.data, p4.ctypes.data,
                        r.ctypes.data, r.shape[0], int(any_hit), *[o.ctypes.data for o in out], threads or nthreads())
    return _pack(*out)


# ---- GLSL built-ins of the restated shader passes ------------------------------
GLSL_FNS = {"sin": 0, "cos": 1, "atan": 2, "exp": 3, "pow": 4}


class glsl_math:
    """Context manager: the oracle's restated passes use the host libm (0, the
    default, as the reference compiled in oracle/_ref does) or the library's
    built-ins (1, myrt_b200/csrc/glmath.hpp, as the device does)."""

    def __init__(self, mode: int):
        self.mode = mode

    def __enter__(self):
        oracle().orc_set_glsl_math(self.mode)
        return self

    def __exit__(self, *exc):
        oracle().orc_set_glsl_math(0)


def glsl_eval(name: str, x, y=None) -> np.ndarray:
    """The library's built-in `name` evaluated on the host (glmath.hpp)."""
    xs = np.ascontiguousarray(x, np.float32).ravel()
    ys = None if y is None else np.ascontiguousarray(np.broadcast_to(np.float32(y) if np.isscalar(y) else y,
                                                                      xs.shape), np.float32).ravel()
    out = np.empty_like(xs)
    oracle().orc_glsl_eval(GLSL_FNS[name], xs.ctypes.data, None if ys is None else ys.ctypes.data, xs.size,
                           out.ctypes.data)
    return out


# ---- instanced scenes: two-level walks (pt_trace.comp:284-309) ---------------
def _geometries(scene):
    """Distinct geometries of a scene's drawables, keyed like the reference's
    push_geometry results: (indices_base, points_base, index_count) -> slot;
    and per drawable its slot and first global prim id."""
    keys, slot, base, acc = {}, [], [], 0
    for d in scene["drawables"]:
        k = (int(d.indices_base_index), int(d.points_base_index), int(d.index_count))
        slot.append(keys.setdefault(k, len(keys)))
        base.append(acc)
        acc += k[2] // 3
    return list(keys), np.array(slot, np.int64), np.array(base, np.int64)


def _points4(scene):
    v = np.asarray(scene["vertices"], np.float32)
    p4 = np.zeros((v.shape[0], 4), np.float32)
    p4[:, :3] = v[:, :3]
    return p4


def instanced_closest(scene: dict, rays, any_hit=False, isect=0):
    """The oracle's restatement of the instanced query (orc_instanced_query):
    per drawable, the ray in object space through the restated reference tree
    of its geometry; canonical ties on global prim ids. Returns hits (closest)
    or a bool array (any hit)."""
    L = oracle()
    idx = np.ascontiguousarray(scene["indices"], np.uint32)
    p4 = _points4(scene)
    geoms, _, _ = _geometries(scene)
    node_blocks, idx_blocks, bases = [], [], {}
    nn = ni = 0
    for (ib, pb, cnt) in geoms:
        local = np.ascontiguousarray(idx[ib:ib + cnt])
        pts = np.ascontiguousarray(p4[pb:, :3])
        nodes, bi = refbvh_build(local, pts)
        bases[(ib, pb, cnt)] = (nn, ni)
        node_blocks.append(nodes)
        idx_blocks.append(bi)
        nn += nodes.shape[0]
        ni += bi.size
    nodes = np.ascontiguousarray(np.concatenate(node_blocks), np.uint32)
    bi = np.ascontiguousarray(np.concatenate(idx_blocks), np.uint32)
    dr = _drawables_with_bases(scene, bases)
    r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    out = _hits(r.shape[0])
    L.orc_instanced_query(nodes.ctypes.data, bi.ctypes.data, idx.ctypes.data, p4.ctypes.data, dr.ctypes.data,
                          len(scene["drawables"]), r.ctypes.data, r.shape[0], int(any_hit), int(isect),
                          *[o.ctypes.data for o in out], nthreads())
    h = _pack(*out)
    return h["prim"] >= 0 if any_hit else h


def _drawables_with_bases(scene, bases) -> np.ndarray:
    """The drawables as 40-word records with bvh_node_base_index and
    bvh_index_base_index pointing at their geometry's tree."""
    import ctypes as _C
    n = len(scene["drawables"])
    raw = np.frombuffer(_C.string_at(_C.addressof(scene["drawables"]), 160 * n), np.uint32).reshape(n, 40).copy()
    for i, d in enumerate(scene["drawables"]):
        nb, ib = bases[(int(d.indices_base_index), int(d.points_base_index), int(d.index_count))]
        raw[i, 32], raw[i, 33] = nb, ib
    return raw


def ref_instanced(scene: dict, rays, any_hit=False, threads=None):
    """The reference's own instanced query (oracle/_ref): geometry trees built
    by bvh.cpp with split_aabbs (scene::push_geometry), the tree over the
    drawables' world boxes with dont_split (scene::enqueue / prepare), walked
    by the compiled bvh.impl.glsl + visit_object_aabb. Returns (drawable,
    local prim, hits with global prim ids)."""
    L = ref()
    idx = np.ascontiguousarray(scene["indices"], np.uint32)
    p4 = _points4(scene)
    geoms, slot, base = _geometries(scene)
    node_blocks, idx_blocks, bases, boxes = [], [], {}, []
    nn = ni = 0
    for (ib, pb, cnt) in geoms:
        local = np.ascontiguousarray(idx[ib:ib + cnt])
        pts = np.ascontiguousarray(p4[pb:, :3])
        h = ref_bvh(local, pts, split=True)
        nodes, bi = ref_bvh_arrays(h)
        box = np.zeros(6, np.float32)
        L.ref_bvh_aabb(h, box.ctypes.data)
        L.ref_bvh_free(h)
        bases[(ib, pb, cnt)] = (nn, ni)
        node_blocks.append(nodes)
        idx_blocks.append(bi)
        boxes.append(box)
        nn += nodes.shape[0]
        ni += bi.size
    onodes = np.ascontiguousarray(np.concatenate(node_blocks), np.uint32)
    obi = np.ascontiguousarray(np.concatenate(idx_blocks), np.uint32)
    dr = _drawables_with_bases(scene, bases)
    dboxes = np.ascontiguousarray(np.stack([boxes[k] for k in slot]), np.float32)
    xf = np.ascontiguousarray(dr[:, 0:16].view(np.float32))
    th = L.ref_bvh_build_instances(dboxes.ctypes.data, xf.ctypes.data, dr.shape[0])
    gnodes, gbi = ref_bvh_arrays(th)
    L.ref_bvh_free(th)
    r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    n = r.shape[0]
    geom = np.empty(n, np.int32)
    out = _hits(n)
    L.ref_glsl_traverse_instanced(gnodes.ctypes.data, gbi.ctypes.data, onodes.ctypes.data, obi.ctypes.data,
                                  idx.ctypes.data, p4.ctypes.data, dr.ctypes.data, r.ctypes.data, n, int(any_hit),
                                  geom.ctypes.data, *[o.ctypes.data for o in out], threads or nthreads())
    h = _pack(*out)
    local = h["prim"].copy()
    hit = geom >= 0
    h["prim"][hit] = (base[geom[hit]] + local[hit]).astype(np.int32)
    return geom, local, h


# ---- scene baking (numpy, independent of the product's C++ bake) -----------
def bake_world_triangles(indices, vertices, drawables=None) -> np.ndarray:
    """World-space triangles float32[T, 9] in the product's prim numbering
    (drawable by drawable, then index order); float32 arithmetic with the same
    left-to-right sums as a column-major mat4 * vec4."""
    idx = np.asarray(indices, np.uint32)
    v = np.asarray(vertices, np.float32)[:, :3]
    if drawables is None or len(drawables) == 0:
        return v[idx.reshape(-1, 3)].reshape(-1, 9)
    out = []
    for d in drawables:
        m = np.array(d.transformation[:], np.float32)
        sel = idx[d.indices_base_index: d.indices_base_index + d.index_count].astype(np.int64) + d.points_base_index
        p = v[sel]
        ident = np.array_equal(m, np.eye(4, dtype=np.float32).ravel())
        if not ident:
            x, y, z = p[:, 0], p[:, 1], p[:, 2]
            one = np.float32(1.0)
            p = np.stack([((m[r] * x + m[4 + r] * y) + m[8 + r] * z) + m[12 + r] * one for r in range(3)], 1)
        out.append(p.reshape(-1, 9).astype(np.float32))
    return np.concatenate(out, 0)


def bake_world_attributes(indices, normals, uvs, drawables, n_vertices):
    """Per-triangle corner normals [T, 9] (normal matrix = transpose of the
    inverse's 3x3, left-to-right sums; not normalised) and uvs [T, 6], and the
    per-triangle material index, in prim order."""
    idx = np.asarray(indices, np.uint32)
    if drawables is None or len(drawables) == 0:
        class _D:  # one identity drawable over the whole buffer
            transformation = np.eye(4, dtype=np.float32).ravel()
            inverse_transformation = np.eye(4, dtype=np.float32).ravel()
            indices_base_index, points_base_index, index_count, material_index = 0, 0, idx.size, 0
        drawables = [_D()]
    nrm, uv, mat = [], [], []
    for d in drawables:
        sel = idx[d.indices_base_index: d.indices_base_index + d.index_count].astype(np.int64) + d.points_base_index
        m = np.array(d.transformation[:], np.float32)
        inv = np.array(d.inverse_transformation[:], np.float32)
        ident = np.array_equal(m, np.eye(4, dtype=np.float32).ravel())
        if normals is not None:
            n = np.asarray(normals, np.float32)[:, :3][sel]
            if not ident:
                nm = np.array([[inv[r * 4 + c] for r in range(3)] for c in range(3)], np.float32).ravel()  # nm[c*3+r]
                x, y, z = n[:, 0], n[:, 1], n[:, 2]
                n = np.stack([(nm[r] * x + nm[3 + r] * y) + nm[6 + r] * z for r in range(3)], 1)
            nrm.append(n.reshape(-1, 9).astype(np.float32))
        if uvs is not None:
            uv.append(np.asarray(uvs, np.float32)[sel].reshape(-1, 6))
        mat.append(np.full(d.index_count // 3, d.material_index, np.int32))
    return (np.concatenate(nrm) if nrm else None, np.concatenate(uv) if uv else None, np.concatenate(mat))


def host_rng(seed: int, frames: int, bounces: int):
    """Per-pass (seed, 1024-float texture) in sequential_pathtracer's draw order."""
    passes = 2 * bounces + 3
    seeds = np.zeros(frames * passes, np.int32)
    tex = np.zeros((frames * passes, 1024), np.float32)
    oracle().orc_host_rng(seed, frames, bounces, seeds.ctypes.data, tex.ctypes.data)
    return seeds, tex


def prepare_reference(scene: dict):
    """World-space triangles and attributes of a scene and the reference's
    tree over them (bvh.cpp's build restated), as render_reference uses them."""
    tris9 = bake_world_triangles(scene["indices"], scene["vertices"], scene.get("drawables"))
    nrm, uvs, mat = bake_world_attributes(scene["indices"], scene.get("normals"), scene.get("uvs"),
                                          scene.get("drawables"), len(scene["vertices"]))
    idx = np.arange(tris9.shape[0] * 3, dtype=np.uint32)
    nodes, bi = refbvh_build(idx, tris9.reshape(-1, 3))
    return tris9, nrm, uvs, mat, nodes, bi


def render_reference(scene: dict, width: int, height: int, bounces: int, frames: int, inv_view, inv_proj,
                     seed: int = 5489, accum=None, display=None, sample_index0: int = 0, textures=None,
                     cubemap=None, dof: bool = False, lens_size=(0.2, 0.2), focus: float = 1.0,
                     bokeh_slot: int = -1, prepared=None):
    """Reference-shading render on the CPU (restated passes). scene: dict with
    indices, vertices, normals, uvs, drawables, materials, material_data.
    textures: list of (rgba [H, W, 4], wrap) or None per slot; cubemap:
    [6, S, S, 4] (stored at half precision, as the device stores it).
    prepared: the result of prepare_reference(scene), to skip the world-space
    bake and the tree build (scene::prepare's work) on repeated renders."""
    L = oracle()
    tris9, nrm, uvs, mat, nodes, bi = prepared if prepared is not None else prepare_reference(scene)
    refs = np.ascontiguousarray(scene.get("materials", np.zeros((1, 2), np.int32)), np.int32).reshape(-1, 2)
    mdata = np.ascontiguousarray(scene.get("material_data", np.zeros(7, np.float32)), np.float32).ravel()
    seeds, tex = host_rng(seed, frames, bounces)
    if accum is None:
        accum = np.zeros((height, width, 4), np.float32)
    if display is None:
        display = np.zeros((height, width, 4), np.float32)
    iv = np.ascontiguousarray(inv_view, np.float32).ravel()
    ip = np.ascontiguousarray(inv_proj, np.float32).ravel()
    nrm_p = nrm.ctypes.data if nrm is not None else None
    uv_p = uvs.ctypes.data if uvs is not None else None
    sdf = scene.get("sdf")  # optional: dict(lib=SdfLibrary, drawables=[N,36], steps=, eps=)
    if sdf is not None:
        s_ins, s_prs, s_par = _sdf_arrays(sdf["lib"])
        s_dr = np.ascontiguousarray(sdf["drawables"], np.float32).reshape(-1, 36)
        sdf_args = [s_ins.ctypes.data, s_prs.ctypes.data, s_par.ctypes.data, s_dr.ctypes.data, s_dr.shape[0],
                    int(sdf["steps"]), float(sdf["eps"])]
    else:
        sdf_args = [None, None, None, None, 0, 0, 0.0]
    texs = [None if t is None else (np.ascontiguousarray(t[0], np.float32), int(t[1])) for t in (textures or [])]
    tex_ptrs = (C.c_void_p * max(1, len(texs)))(*[t[0].ctypes.data if t else None for t in texs])
    tex_dims = np.array([[t[0].shape[1], t[0].shape[0], t[1]] if t else [0, 0, 0] for t in texs] or [[0, 0, 0]],
                        np.int32)
    cube = None
    if cubemap is not None:
        cube = np.ascontiguousarray(np.asarray(cubemap, np.float32).astype(np.float16).astype(np.float32))
    L.orc_render_reference(tris9.shape[0], tris9.ctypes.data, nrm_p, uv_p, mat.ctypes.data, refs.ctypes.data,
                           refs.shape[0], mdata.ctypes.data, nodes.ctypes.data, bi.ctypes.data, width, height, bounces,
                           frames, sample_index0, iv.ctypes.data, ip.ctypes.data, seeds.ctypes.data, tex.ctypes.data,
                           accum.ctypes.data, display.ctypes.data, *sdf_args, nthreads(), len(texs),
                           C.cast(tex_ptrs, C.c_void_p), tex_dims.ctypes.data,
                           cube.ctypes.data if cube is not None else None, cube.shape[1] if cube is not None else 0,
                           int(dof), float(lens_size[0]), float(lens_size[1]), float(focus),
                           bokeh_slot + 1 if bokeh_slot >= 0 else 0)
    return accum, display


# ---- forward (raster preview) renderer -------------------------------------------
def forward_render(scene: dict, width: int, height: int, view, proj, random_seed: int, shadow_size: int,
                   shadow_view, shadow_proj, textures=None, result: bool = True) -> dict:
    """forward_renderer::run on the CPU (restated passes). Matrices are numpy
    [4, 4] in math layout. Returns visibility / shadow visibility keys (uint64),
    gbuffer [3, H, W, 4] and result [H, W, 4] (half-rounded float32),
    shadow_map [S, S, 4]."""
    L = oracle()
    tris9 = np.ascontiguousarray(bake_world_triangles(scene["indices"], scene["vertices"], scene.get("drawables")))
    nrm, uvs, mat = bake_world_attributes(scene["indices"], scene.get("normals"), scene.get("uvs"),
                                          scene.get("drawables"), len(scene["vertices"]))
    refs = np.ascontiguousarray(scene.get("materials", np.zeros((1, 2), np.int32)), np.int32).reshape(-1, 2)
    mdata = np.ascontiguousarray(scene.get("material_data", np.zeros(7, np.float32)), np.float32).ravel()

    def cm(m):
        return np.ascontiguousarray(np.asarray(m, np.float32).T).ravel()

    v, p, sv, sp = cm(view), cm(proj), cm(shadow_view), cm(shadow_proj)
    S = shadow_size
    out = {"visibility": np.empty((height, width), np.uint64), "shadow_visibility": np.empty((S, S), np.uint64),
           "gbuffer": np.empty((3, height, width, 4), np.float32), "shadow_map": np.empty((S, S, 4), np.float32),
           "result": np.empty((height, width, 4), np.float32) if result else None}
    texs = [None if t is None else (np.ascontiguousarray(t[0], np.float32), int(t[1])) for t in (textures or [])]
    tex_ptrs = (C.c_void_p * max(1, len(texs)))(*[t[0].ctypes.data if t else None for t in texs])
    tex_dims = np.array([[t[0].shape[1], t[0].shape[0], t[1]] if t else [0, 0, 0] for t in texs] or [[0, 0, 0]],
                        np.int32)
    nrm_c = np.ascontiguousarray(nrm, np.float32) if nrm is not None else None
    uv_c = np.ascontiguousarray(uvs, np.float32) if uvs is not None else None
    L.orc_forward_render(tris9.shape[0], tris9.ctypes.data, nrm_c.ctypes.data if nrm_c is not None else None,
                         uv_c.ctypes.data if uv_c is not None else None, mat.ctypes.data, refs.ctypes.data,
                         refs.shape[0], mdata.ctypes.data, width, height, v.ctypes.data, p.ctypes.data,
                         int(random_seed) & 0xFFFFFFFF, S, sv.ctypes.data, sp.ctypes.data, len(texs),
                         C.cast(tex_ptrs, C.c_void_p), tex_dims.ctypes.data, out["visibility"].ctypes.data,
                         out["gbuffer"].ctypes.data, out["shadow_visibility"].ctypes.data,
                         out["shadow_map"].ctypes.data, out["result"].ctypes.data if result else None)
    return out


def ref_forward_resolve(gbuffer, shadow_map, view, proj, shadow_view, shadow_proj, random_seed: int, materials,
                        material_data) -> np.ndarray:
    """The reference's own forward/resolve.frag (compiled by oracle/build_ref.py)
    over a G-buffer [3, H, W, 4] and a shadow map [S, S, 4]; returns the colour
    [H, W, 4] before the RGBA16F store."""
    L = ref()
    g = np.ascontiguousarray(gbuffer, np.float32)
    sm = np.ascontiguousarray(shadow_map, np.float32)
    H, W = g.shape[1], g.shape[2]

    def cm(m):
        return np.ascontiguousarray(np.asarray(m, np.float32).T).ravel()

    v, p, sv, sp = cm(view), cm(proj), cm(shadow_view), cm(shadow_proj)
    refs = np.ascontiguousarray(materials, np.int32).reshape(-1, 2)
    md = np.ascontiguousarray(material_data, np.float32).ravel()
    out = np.empty((H, W, 4), np.float32)
    L.ref_forward_resolve(W, H, g.ctypes.data, sm.ctypes.data, sm.shape[0], v.ctypes.data, p.ctypes.data,
                          sv.ctypes.data, sp.ctypes.data, int(random_seed) & 0xFFFFFFFF, refs.ctypes.data,
                          md.ctypes.data, out.ctypes.data)
    return out


# ---- single passes of the reference shading mode (pinning) ----------------------
def pass_generate(width, height, inv_view, inv_proj, seed, random_tex, dof=False, lens=(0.0, 0.0), focus=1.0,
                  bokeh=None, bokeh_wrap=0, use_ref=False) -> np.ndarray:
    """pt_generate.comp over the image: the oracle's restatement, or (use_ref)
    the reference's shader compiled by oracle/build_ref.py. Returns the
    generate_output_t records as float32 [H * W, 20] (int fields as bits)."""
    L = ref() if use_ref else oracle()
    fn = L.ref_pass_generate if use_ref else L.orc_pass_generate
    iv = np.ascontiguousarray(inv_view, np.float32).ravel()
    ip = np.ascontiguousarray(inv_proj, np.float32).ravel()
    tex = np.ascontiguousarray(random_tex, np.float32)
    bk = np.ascontiguousarray(bokeh, np.float32) if bokeh is not None else None
    out = np.zeros((width * height, 20), np.float32)
    fn(width, height, iv.ctypes.data, ip.ctypes.data, int(seed), tex.ctypes.data, tex.size, int(dof),
       float(lens[0]), float(lens[1]), float(focus), bk.ctypes.data if bk is not None else None,
       bk.shape[1] if bk is not None else 0, bk.shape[0] if bk is not None else 0, int(bokeh_wrap),
       out.ctypes.data)
    return out


def pass_color(gen, trace, accum, display, sample_index, force, seed, random_tex, materials, material_data,
               use_ref=False):
    """pt_color.comp over the rays of gen / trace (float32 [n, 20] / [n, 16],
    updated copies are returned with the images)."""
    L = ref() if use_ref else oracle()
    g = np.array(gen, np.float32, copy=True, order="C")
    t = np.array(trace, np.float32, copy=True, order="C")
    a = np.array(accum, np.float32, copy=True, order="C")
    d = np.array(display, np.float32, copy=True, order="C")
    tex = np.ascontiguousarray(random_tex, np.float32)
    refs = np.ascontiguousarray(materials, np.int32).reshape(-1, 2)
    md = np.ascontiguousarray(material_data, np.float32).ravel()
    H, W = a.shape[0], a.shape[1]
    args = [g.shape[0], g.ctypes.data, t.ctypes.data, a.ctypes.data, d.ctypes.data, W, H, int(sample_index),
            int(force), int(seed), tex.ctypes.data, tex.size, refs.ctypes.data]
    if use_ref:
        L.ref_pass_color(*args, md.ctypes.data)
    else:
        L.orc_pass_color(*args, refs.shape[0], md.ctypes.data)
    return g, t, a, d


# ---- SDF ----------------------------------------------------------------------
def _sdf_arrays(lib):
    return (np.ascontiguousarray(lib.instrs, np.int32), np.ascontiguousarray(lib.programs, np.int32),
            np.ascontiguousarray(lib.params, np.float32))


def sdf_map(lib, prog: int, pts, load_materials=False, rng_states=None, use_ref=False):
    ins, prs, par = _sdf_arrays(lib)
    p = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
    n = p.shape[0]
    d = np.zeros(n, np.float32)
    m = np.zeros(n, np.int32)
    rs = None if rng_states is None else np.ascontiguousarray(rng_states, np.uint32)
    fn = ref().ref_sdf_map if use_ref else oracle().orc_sdf_map
    fn(ins.ctypes.data, prs.ctypes.data, par.ctypes.data, prog, p.ctypes.data, n, int(load_materials),
       None if rs is None else rs.ctypes.data, d.ctypes.data, m.ctypes.data)
    return d, m


def sdf_trace(lib, drawables, rays, steps, eps, any_hit=False, rng_states=None, use_ref=False):
    ins, prs, par = _sdf_arrays(lib)
    dr = np.ascontiguousarray(drawables, np.float32).reshape(-1, 36)
    r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    n = r.shape[0]
    hit = np.zeros(n, np.int32)
    t = np.zeros(n, np.float32)
    nn = np.zeros((n, 3), np.float32)
    uv = np.zeros((n, 2), np.float32)
    mat = np.zeros(n, np.int32)
    rs = None if rng_states is None else np.ascontiguousarray(rng_states, np.uint32)
    args = [ins.ctypes.data, prs.ctypes.data, par.ctypes.data, dr.ctypes.data, dr.shape[0], r.ctypes.data, n, steps,
            float(eps), int(any_hit), None if rs is None else rs.ctypes.data, hit.ctypes.data, t.ctypes.data,
            nn.ctypes.data, uv.ctypes.data, mat.ctypes.data]
    if use_ref:
        ref().ref_sdf_trace(*args)
    else:
        oracle().orc_sdf_trace(*args, nthreads())
    return dict(hit=hit, t=t, normal=nn, uv=uv, material=mat)


# ---- physical mode --------------------------------------------------------------
def physical_lights(lights) -> np.ndarray:
    """24 floats per light (corner, edge_u, edge_v, emission, normal, area, du,
    prob, dv, cdf), computed in double and rounded like the device upload.
    lights: [n, 12] float32 (corner, edge_u, edge_v, emission)."""
    L = np.asarray(lights, np.float32).reshape(-1, 12).astype(np.float64)
    out = np.zeros((L.shape[0], 24), np.float32)
    power = []
    for i, q in enumerate(L):
        u, w = q[3:6], q[6:9]

        def cross(x, y):
            return np.array([x[1] * y[2] - x[2] * y[1], x[2] * y[0] - x[0] * y[2], x[0] * y[1] - x[1] * y[0]])

        c = cross(u, w)
        area = np.sqrt((c[0] * c[0] + c[1] * c[1]) + c[2] * c[2])
        nn = c / area
        a1, b1 = cross(w, nn), cross(nn, u)
        sa = (a1[0] * u[0] + a1[1] * u[1]) + a1[2] * u[2]
        sb = (b1[0] * w[0] + b1[1] * w[1]) + b1[2] * w[2]
        out[i, 0:12] = q[0:12]
        out[i, 12:15] = nn
        out[i, 15] = area
        out[i, 16:19] = a1 / sa
        out[i, 20:23] = b1 / sb
        e = q[9:12]
        power.append(((0.2126 * e[0] + 0.7152 * e[1]) + 0.0722 * e[2]) * area)
    total = 0.0
    for pw in power:
        total = total + pw
    run = 0.0
    for i, pw in enumerate(power):
        p = pw / total if total > 0 else 1.0 / len(power)
        run = run + p
        out[i, 19] = p
        out[i, 23] = 1.0 if i + 1 == len(power) else run
    return out


def mat_mul4(a, b) -> np.ndarray:
    """Column-major 4x4 product in float32 with the device's summation order."""
    a = np.asarray(a, np.float32).ravel()
    b = np.asarray(b, np.float32).ravel()
    out = np.zeros(16, np.float32)
    for c in range(4):
        for r in range(4):
            out[c * 4 + r] = ((a[0 * 4 + r] * b[c * 4 + 0] + a[1 * 4 + r] * b[c * 4 + 1]) + a[2 * 4 + r] * b[c * 4 + 2]) \
                + a[3 * 4 + r] * b[c * 4 + 3]
    return out


def render_physical(scene: dict, width: int, height: int, spp: int, inv_view, inv_proj, lights, env=(0, 0, 0),
                    max_depth: int = 8, rr_start: int = 3, seed: int = 0, sample0: int = 0, fp64: bool = False,
                    accum=None):
    """Physical-mode render on the CPU, path at a time (the device's method,
    restated). Returns the accumulation (rgb sum, count), float32 or float64."""
    L = oracle()
    tris9 = bake_world_triangles(scene["indices"], scene["vertices"], scene.get("drawables"))
    nrm, _, mat = bake_world_attributes(scene["indices"], scene.get("normals"), None, scene.get("drawables"),
                                        len(scene["vertices"]))
    idx = np.arange(tris9.shape[0] * 3, dtype=np.uint32)
    nodes, bi = refbvh_build(idx, tris9.reshape(-1, 3))
    refs = np.ascontiguousarray(scene.get("materials", np.zeros((1, 2), np.int32)), np.int32).reshape(-1, 2)
    mdata = np.ascontiguousarray(scene.get("material_data", np.zeros(7, np.float32)), np.float32).ravel()
    lt = physical_lights(lights) if lights is not None and len(lights) else np.zeros((0, 24), np.float32)
    env = np.ascontiguousarray(env, np.float32)
    vp = mat_mul4(inv_view, inv_proj)
    eye = np.ascontiguousarray(np.asarray(inv_view, np.float32).ravel()[12:15])
    dt = np.float64 if fp64 else np.float32
    if accum is None:
        accum = np.zeros((height, width, 4), dt)
    sdf = scene.get("sdf")
    if sdf is not None:
        s_ins, s_prs, s_par = _sdf_arrays(sdf["lib"])
        s_dr = np.ascontiguousarray(sdf["drawables"], np.float32).reshape(-1, 36)
        sdf_args = [s_ins.ctypes.data, s_prs.ctypes.data, s_par.ctypes.data, s_dr.ctypes.data, s_dr.shape[0],
                    int(sdf["steps"]), float(sdf["eps"])]
    else:
        sdf_args = [None, None, None, None, 0, 0, 0.0]
    nrm_p = nrm.ctypes.data if nrm is not None else None
    L.orc_render_physical(tris9.shape[0], tris9.ctypes.data, nrm_p, mat.ctypes.data, refs.ctypes.data, refs.shape[0],
                          mdata.ctypes.data, nodes.ctypes.data, bi.ctypes.data, lt.ctypes.data, lt.shape[0],
                          env.ctypes.data, width, height, spp, sample0, max_depth, rr_start, seed, vp.ctypes.data,
                          eye.ctypes.data, *sdf_args, int(fp64), accum.ctypes.data, nthreads())
    return accum


def post_pass(op: int, img: np.ndarray, i=(0, 0, 0), p=(0.0, 0.0, 0.0, 0.0), overlay: np.ndarray | None = None,
              out_size: tuple[int, int] | None = None) -> np.ndarray:
    """One post-processing pass on a float32 [H, W, 4] image (oracle_post.cpp)."""
    L = oracle()
    a = np.ascontiguousarray(img, np.float32)
    h, w = a.shape[:2]
    oh, ow = out_size if out_size else (h, w)
    ov = np.ascontiguousarray(overlay if overlay is not None else a, np.float32)
    out = np.empty((oh, ow, 4), np.float32)
    ip = np.asarray(i, np.int32)
    fp = np.asarray(p, np.float32)
    rc = L.oracle_post_pass(int(op), ip.ctypes.data, fp.ctypes.data, a.ctypes.data, w, h, ov.ctypes.data,
                            ov.shape[1], ov.shape[0], out.ctypes.data, ow, oh)
    if rc:
        raise ValueError(f"unknown post pass {op}")
    return out


def ref_post_pass(op: int, img: np.ndarray, i=(0, 0, 0), p=(0.0, 0.0, 0.0, 0.0),
                  overlay: np.ndarray | None = None) -> np.ndarray:
    """The reference's own pp_*.comp shader (compiled in oracle/_ref) on a
    float32 [H, W, 4] image."""
    a = np.ascontiguousarray(img, np.float32)
    h, w = a.shape[:2]
    ov = np.ascontiguousarray(overlay if overlay is not None else a, np.float32)
    out = np.zeros((h, w, 4), np.float32)
    ip = np.asarray(i, np.int32)
    fp = np.asarray(p, np.float32)
    rc = ref().ref_post_pass(int(op), ip.ctypes.data, fp.ctypes.data, a.ctypes.data, w, h, ov.ctypes.data,
                             ov.shape[1], ov.shape[0], out.ctypes.data)
    if rc:
        raise ValueError(f"no reference shader for post pass {op}")
    return out
