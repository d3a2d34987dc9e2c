"""Host BVH builder: structure invariants and CPU traversal parity (no GPU)."""
import numpy as np
import pytest

import myrt_b200 as mb
import pyoracle as po
from myrt_b200.scenes import heightfield, icosphere_field, pinhole_rays


def _decode(nodes):
    """Per node: p (3 floats), scale (3), imask, child_base, tri_base, meta[8], qlo[3,8], qhi[3,8]."""
    raw = nodes.view(np.uint8).reshape(-1, 80)
    p = nodes[:, 0:3].view(np.float32)
    e = raw[:, 12:15].astype(np.int32) - 127
    imask = raw[:, 15]
    child_base = nodes[:, 4]
    tri_base = nodes[:, 5]
    meta = raw[:, 24:32]
    qlo = raw[:, 32:56].reshape(-1, 3, 8)
    qhi = raw[:, 56:80].reshape(-1, 3, 8)
    return p, np.ldexp(1.0, e), imask, child_base, tri_base, meta, qlo, qhi


def _check_tree(nodes, tris, tris9):
    p, scale, imask, cbase, tbase, meta, qlo, qhi = _decode(nodes)
    n_nodes = nodes.shape[0]
    seen_nodes = np.zeros(n_nodes, np.int32)
    seen_tris = np.zeros(tris.shape[0], np.int32)
    seen_nodes[0] = 1
    sub_lo = np.full((n_nodes, 3), np.inf)
    sub_hi = np.full((n_nodes, 3), -np.inf)
    internal_slots = []
    # children always have larger indices than their parent: walk in reverse
    # for subtree bounds, forward for the per-slot checks
    for n in range(n_nodes):
        k_internal = 0
        for s in range(8):
            lo = p[n] + qlo[n, :, s] * scale[n]
            hi = p[n] + qhi[n, :, s] * scale[n]
            if meta[n, s] == 0:
                assert not (imask[n] >> s) & 1
                continue
            if (imask[n] >> s) & 1:
                c = cbase[n] + k_internal
                assert c > n
                k_internal += 1
                seen_nodes[c] += 1
                internal_slots.append((n, c, lo, hi))
            else:
                cnt, off = int(meta[n, s]) >> 5, int(meta[n, s]) & 31
                assert 1 <= cnt <= 4
                for k in range(cnt):
                    ti = tbase[n] + off + k
                    seen_tris[ti] += 1
                    tri = tris[ti]
                    pid = tri[3:4].view(np.int32)[0]
                    v = tri[[0, 1, 2, 4, 5, 6, 8, 9, 10]].reshape(3, 3)
                    assert np.array_equal(v.ravel(), tris9[pid])
                    # conservative quantisation: the triangle lies inside its slot box
                    assert np.all(v.min(0) >= lo) and np.all(v.max(0) <= hi)
                    sub_lo[n] = np.minimum(sub_lo[n], v.min(0))
                    sub_hi[n] = np.maximum(sub_hi[n], v.max(0))
    for n, c, lo, hi in reversed(internal_slots):
        sub_lo[n] = np.minimum(sub_lo[n], sub_lo[c])
        sub_hi[n] = np.maximum(sub_hi[n], sub_hi[c])
    for n, c, lo, hi in internal_slots:
        # every triangle below an internal slot lies inside that slot's box
        assert np.all(sub_lo[c] >= lo) and np.all(sub_hi[c] <= hi)
    assert np.all(seen_nodes == 1), "every wide node is referenced exactly once"
    assert np.all(seen_tris == 1), "every triangle reference is reached exactly once"
    pids = tris[:, 3].view(np.int32)
    assert np.array_equal(np.sort(pids), np.arange(tris9.shape[0])), "each prim appears exactly once"


@pytest.mark.parametrize("n", [1, 2, 5, 16, 64])
def test_tree_invariants_heightfield(n):
    idx, pts = heightfield(n, seed=n)
    tris9 = pts[idx.reshape(-1, 3)].reshape(-1, 9)
    nodes, tris, info = mb.build_bvh8(tris9)
    assert info["triangles"] == tris9.shape[0]
    assert info["max_leaf_size"] <= 4
    _check_tree(nodes, tris, tris9)


def test_tree_invariants_instanced_spheres():
    s = icosphere_field(n_spheres=24, subdiv=2, floor_cells=4)
    tris9 = po.bake_world_triangles(s["indices"], s["vertices"], s["drawables"])
    nodes, tris, info = mb.build_bvh8(tris9)
    _check_tree(nodes, tris, tris9)


def test_single_and_degenerate_triangles():
    one = np.array([[0, 0, 0, 1, 0, 0, 0, 1, 0]], np.float32)
    nodes, tris, info = mb.build_bvh8(one)
    assert info["wide_nodes"] == 1 and info["triangles"] == 1
    # all-identical centroids (stacked copies) must still build with leaves <= 4
    many = np.repeat(one, 37, axis=0)
    nodes, tris, info = mb.build_bvh8(many)
    assert info["max_leaf_size"] <= 4
    _check_tree(nodes, tris, many)
    # zero-area triangles
    deg = np.zeros((9, 9), np.float32)
    deg[:, 0::3] = np.arange(9)[:, None]
    nodes, tris, info = mb.build_bvh8(deg)
    _check_tree(nodes, tris, deg)


def test_empty_build():
    nodes, tris, info = mb.build_bvh8(np.zeros((0, 9), np.float32))
    assert info["wide_nodes"] == 0 and info["triangles"] == 0


@pytest.mark.parametrize("isect", [0, 1])
def test_cpu_bvh8_traversal_equals_brute_force(isect):
    idx, pts = heightfield(48, seed=3)
    tris9 = pts[idx.reshape(-1, 3)].reshape(-1, 9)
    nodes, tris, _ = mb.build_bvh8(tris9)
    rays = pinhole_rays(96, 96)
    rng = np.random.default_rng(0)
    rnd = rays.copy()
    rnd[:, 0:3] = rng.uniform(-1.2, 1.2, (rays.shape[0], 3)).astype(np.float32)
    d = rng.normal(size=(rays.shape[0], 3))
    rnd[:, 4:7] = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    rnd[::5, 7] = 0.7  # finite tmax
    rnd[::7, 3] = 0.3  # non-zero tmin
    for r in (rays, rnd):
        b8, cn, ct = po.bvh8_traverse(nodes, tris, r, isect=isect)
        bf = po.brute_closest(tris9, r, isect=isect)
        assert np.array_equal(b8, bf)
        occ, _, _ = po.bvh8_traverse(nodes, tris, r, isect=isect, any_hit=True)
        assert np.array_equal(occ.astype(bool), bf["prim"] >= 0)


def test_exponential_chain_is_deeper_than_the_traversal_stack():
    """The degenerate chain the GPU tests use to check that an upload of a tree
    deeper than 32 wide levels is refused really builds one."""
    from myrt_b200.scenes import exponential_chain

    nodes, tris, info = mb.build_bvh8(exponential_chain())
    assert info["wide_depth"] > 32
    assert info["triangles"] == exponential_chain().shape[0]
