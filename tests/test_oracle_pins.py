"""The oracle restatement against golden vectors from the reference's own code.

tests/golden/*.npz were produced by tests/golden/make_golden.py from the
reference sources compiled in oracle/_ref (bvh.cpp, the GLSL traversal and
intersector). These tests need no reference tree and no GPU.
"""
import numpy as np

import pyoracle as po


def test_restated_build_matches_reference_bvh(golden):
    g = golden("refbvh_hf16.npz")
    nodes, bi = po.refbvh_build(g["indices"], g["points"])
    # 36 meaningful bytes per 48-byte node (min, type|parent, max, first, second)
    assert np.array_equal(nodes[:, :9], g["nodes_nosplit"][:, :9])
    assert np.array_equal(bi, g["bvh_indices_nosplit"])


def test_restated_traversal_matches_reference_glsl(golden):
    g = golden("closest_hf128.npz")
    idx, pts, rays = g["indices"], g["points"], g["rays"]
    # the oracle's restated traversal over the restated (dont_split) tree, first-visited ties
    nodes, bi = po.refbvh_build(idx, pts)
    o = po.refbvh_traverse(nodes, bi, idx, pts, rays, canonical=False)
    glsl = g["glsl"]
    assert np.array_equal(o["prim"], glsl["prim"])
    hit = glsl["prim"] >= 0
    # same triangle + same Moller-Trumbore -> bit-identical t and barycentrics
    assert np.array_equal(o["t"][hit], glsl["t"][hit])
    assert np.array_equal(o["u"][hit], glsl["u"][hit])
    assert np.array_equal(o["v"][hit], glsl["v"][hit])


def test_reference_cpu_pick_agrees_with_glsl(golden):
    g = golden("closest_hf128.npz")
    assert np.array_equal(g["pick"]["prim"], g["glsl"]["prim"])
    assert np.array_equal(g["pick"]["t"], g["glsl"]["t"])


def test_canonical_oracle_matches_reference_hits(golden):
    """Canonical tie-break (min t, then min prim) vs the reference's first-visited rule."""
    g = golden("closest_hf128.npz")
    idx, pts, rays = g["indices"], g["points"], g["rays"]
    tris9 = pts[idx.reshape(-1, 3)].reshape(-1, 9)
    bf = po.brute_closest(tris9, rays, isect=0)
    glsl = g["glsl"]
    same = bf["prim"] == glsl["prim"]
    # any disagreement must be an exact tie in t
    assert np.array_equal(bf["t"], glsl["t"])
    assert same.mean() >= 0.999


def test_any_hit_matches_reference(golden):
    g = golden("closest_hf128.npz")
    idx, pts = g["indices"], g["points"]
    nodes, bi = po.refbvh_build(idx, pts)
    for rays, ref_prim in ((g["rays"], g["any_prim"]), (g["shadow_rays"], g["any_short_prim"])):
        o = po.refbvh_traverse(nodes, bi, idx, pts, rays, any_hit=True, canonical=False)
        assert np.array_equal(o["prim"] >= 0, ref_prim >= 0)


def test_intersect_triangle_kat(golden):
    k = golden("glsl_kat.npz")
    o, d, v = k["tri_o"], k["tri_d"], k["tri_v"]  # bind once: NpzFile returns a new array per access
    ref_hit, ref_t, ref_uv = k["tri_hit"], k["tri_t"], k["tri_uv"]
    assert ref_hit.sum() > 100 and (ref_hit == 0).sum() > 10
    for i in range(o.shape[0]):
        t = np.zeros(1, np.float32)
        uv = np.zeros(2, np.float32)
        oi, di, vi = (np.ascontiguousarray(a[i]) for a in (o, d, v))
        h = po.oracle().orc_isect_reference(oi.ctypes.data, di.ctypes.data, vi.ctypes.data, t.ctypes.data,
                                            uv.ctypes.data)
        assert h == ref_hit[i]
        if h:
            assert t[0] == ref_t[i]
            assert np.array_equal(uv, ref_uv[i])
