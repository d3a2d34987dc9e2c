"""SDF drawables: the oracle restatement against the reference's own
raymarch.glsl + sdf.hpp snippets (golden vectors from oracle/_ref), and the
device implementation against the oracle.

Device bar: hit flags, t, normals and materials bit-exact (the evaluator is
compiled without FMA contraction and uses only +, *, /, sqrt, min/max, abs);
uv within 1e-5 (triplanar weights use pow, CUDA's powf vs the host libm).
"""
import numpy as np
import pytest

import pyoracle as po
from myrt_b200 import sdf as S


class _Lib:  # the fixture's arrays in SdfLibrary's shape
    def __init__(self, k):
        self.instrs, self.programs, self.params = k["instrs"], k["programs"], k["params"]


def test_sdf_map_matches_reference(golden):
    k = golden("sdf_kat.npz")
    lib = _Lib(k)
    pts, states = k["pts"], k["states"]
    for prog in range(3):
        for load in (0, 1):
            d, m = po.sdf_map(lib, prog, pts, bool(load), states)
            assert np.array_equal(d, k[f"map{prog}_{load}_d"])
            if load:
                assert np.array_equal(m, k[f"map{prog}_{load}_m"])


@pytest.mark.parametrize("anyh", [0, 1])
def test_sdf_trace_matches_reference(golden, anyh):
    k = golden("sdf_kat.npz")
    lib = _Lib(k)
    res = po.sdf_trace(lib, k["drawables"], k["rays"], 256, 1e-4, bool(anyh), k["states"][:1536])
    for key, v in res.items():
        assert np.array_equal(v, k[f"trace{anyh}_{key}"]), key
    assert res["hit"].sum() > 100


def test_builder_program_shape():
    lib = S.SdfLibrary()
    i = lib.add(S.smooth_union(S.translate(S.sphere(0.5, 3), (1, 2, 3)), S.box((1, 1, 1), 2), 0.25))
    assert i == 0
    assert lib.instrs.tolist() == [[S.TRANSLATE, 0], [S.SPHERE, 3], [S.BOX, 5], [S.SMOOTH_UNION, 9]]
    assert lib.params.tolist() == [1, 2, 3, 0.5, 3, 1, 1, 1, 2, 0.25]
    assert lib.programs.tolist() == [[0, 4]]


@pytest.mark.gpu
def test_sdf_trace_gpu_matches_oracle(ctx, golden):
    k = golden("sdf_kat.npz")
    lib = _Lib(k)
    dr, rays, states = k["drawables"], k["rays"], k["states"][:1536]
    ctx.upload_sdf(lib.instrs, lib.programs, lib.params, dr)
    for anyh in (False, True):
        got = ctx.trace_sdf(rays, 256, 1e-4, any_hit=anyh, rng_states=states)
        ora = po.sdf_trace(lib, dr, rays, 256, 1e-4, anyh, states)
        assert np.array_equal(got["hit"], ora["hit"])
        assert np.array_equal(got["t"], ora["t"])
        if not anyh:
            assert np.array_equal(got["normal"], ora["normal"])
            assert np.array_equal(got["material"], ora["material"])
            np.testing.assert_allclose(got["uv"], ora["uv"], rtol=1e-5, atol=1e-6)
    ctx.upload_sdf(np.zeros((0, 2)), np.zeros((0, 2)), np.zeros(0), np.zeros((0, 36)))


@pytest.mark.gpu
def test_sdf_field_256_prims_gpu(ctx):
    """The hybrid configuration's SDF: 256 spheres/boxes/tori under smooth union k = 0.1."""
    lib = S.SdfLibrary()
    lib.add(S.random_sdf_field(256, k=0.1, seed=9))
    dr = S.sdf_drawables([np.eye(4)], [0])
    rng = np.random.default_rng(4)
    rays = np.zeros((8192, 8), np.float32)
    rays[:, 0:3] = np.array([0.0, 0.3, -3.5])
    aim = rng.uniform(-0.35, 0.35, (8192, 3)) + np.array([0.0, 0.0, 1.0])
    rays[:, 4:7] = aim / np.linalg.norm(aim, axis=1, keepdims=True)
    rays[:, 7] = np.inf
    states = rng.integers(1, 2**32, 8192, dtype=np.uint64).astype(np.uint32)
    ctx.upload_sdf(lib.instrs, lib.programs, lib.params, dr)
    got = ctx.trace_sdf(rays, 256, 1e-4, rng_states=states)
    ora = po.sdf_trace(lib, dr, rays, 256, 1e-4, False, states)
    assert got["hit"].sum() > 1000
    assert np.array_equal(got["hit"], ora["hit"])
    assert np.array_equal(got["t"], ora["t"])
    assert np.array_equal(got["material"], ora["material"])
    ctx.upload_sdf(np.zeros((0, 2)), np.zeros((0, 2)), np.zeros(0), np.zeros((0, 36)))


@pytest.mark.gpu
def test_sdf_upload_rejects_bad_programs(ctx):
    import myrt_b200 as mb

    dr = S.sdf_drawables([np.eye(4)], [0])
    bad = [
        (np.array([[S.UNION, 0]]), np.array([[0, 1]]), np.zeros(1)),           # operator without operands
        (np.array([[S.SPHERE, 0]]), np.array([[0, 1]]), np.zeros(1)),          # parameter outside the buffer
        (np.array([[99, 0]]), np.array([[0, 1]]), np.zeros(4)),                # unknown opcode
        (np.array([[S.SPHERE, 0], [S.SPHERE, 0]]), np.array([[0, 2]]), np.zeros(2)),  # two results
        (np.array([[S.TRANSLATE, 0]]), np.array([[0, 1]]), np.zeros(3)),       # modifier without primitive
    ]
    for ins, prs, par in bad:
        with pytest.raises(mb.MyrtError):
            ctx.upload_sdf(ins, prs, par, dr)
    with pytest.raises(mb.MyrtError):  # drawable references a missing program
        ctx.upload_sdf(np.array([[S.SPHERE, 0]]), np.array([[0, 1]]), np.zeros(2), S.sdf_drawables([np.eye(4)], [3]))


@pytest.mark.gpu
def test_sdf_exact_skipping_matches_oracle(ctx):
    """Left-to-right unions and smooth unions of translated spheres, boxes, tori
    and capsules: the device skips groups far from the point (bounding-sphere
    test); hits, t, normals and materials stay bit-identical to the oracle,
    which evaluates every primitive."""
    rng = np.random.default_rng(12)
    prims = []
    for i in range(96):
        kind = i % 4
        mat = int(rng.integers(0, 4))
        if kind == 0:
            p = S.sphere(float(rng.uniform(0.03, 0.12)), mat)
        elif kind == 1:
            p = S.box(tuple(rng.uniform(0.02, 0.1, 3)), mat)
        elif kind == 2:
            p = S.torus(float(rng.uniform(0.05, 0.12)), float(rng.uniform(0.01, 0.04)), mat)
        else:
            p = S.vertical_capsule(float(rng.uniform(0.0, 0.2)), float(rng.uniform(0.02, 0.05)), mat)
        prims.append(S.translate(p, rng.uniform(-0.8, 0.8, 3)))
    acc = prims[0]
    for i, nd in enumerate(prims[1:]):
        acc = S.union(acc, nd) if i % 3 == 0 else S.smooth_union(acc, nd, 0.1)
    lib = S.SdfLibrary()
    lib.add(acc)
    lib.add(S.random_sdf_field(128, k=0.1, seed=4, chain=True))
    dr = S.sdf_drawables([np.eye(4), np.array([[1, 0, 0, 0.3], [0, 1, 0, 0], [0, 0, 1, 0.2], [0, 0, 0, 1]])], [0, 1])
    n = 6144
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = np.array([0.0, 0.2, -3.0])
    aim = rng.uniform(-0.3, 0.3, (n, 3)) + np.array([0.0, 0.0, 1.0])
    rays[:, 4:7] = aim / np.linalg.norm(aim, axis=1, keepdims=True)
    rays[:, 7] = np.inf
    states = rng.integers(1, 2**32, n, dtype=np.uint64).astype(np.uint32)
    ctx.upload_sdf(lib.instrs, lib.programs, lib.params, dr)
    try:
        for anyh in (False, True):
            got = ctx.trace_sdf(rays, 256, 1e-4, any_hit=anyh, rng_states=states)
            ora = po.sdf_trace(lib, dr, rays, 256, 1e-4, anyh, states)
            assert got["hit"].sum() > 500
            assert np.array_equal(got["hit"], ora["hit"])
            assert np.array_equal(got["t"], ora["t"])
            if not anyh:
                assert np.array_equal(got["normal"], ora["normal"])
                assert np.array_equal(got["material"], ora["material"])
    finally:
        ctx.upload_sdf(np.zeros((0, 2)), np.zeros((0, 2)), np.zeros(0), np.zeros((0, 36)))


@pytest.mark.gpu
@pytest.mark.parametrize("shape", ["chain", "tree", "right_fold"])
def test_sdf_cell_lists_and_early_exit_exact(ctx, shape):
    """Union / smooth-union trees (left folds, balanced trees, right folds with
    unions mixed in) get per-cell instruction segments and an escape sphere at
    upload (tuning sdf_cells). Hits, t, normals and materials are identical
    with the grid off (1), at the default (0 = 32 cells) and at 8 and 96 cells,
    for rays that start outside the field, inside its grid, pass it by or
    leave it, with finite and infinite tmax; the default also equals the
    oracle on a subset."""
    rng = np.random.default_rng(21)
    lib = S.SdfLibrary()
    if shape == "right_fold":
        r2 = np.random.default_rng(4)
        for n_prims, k in ((22, 0.08), (16, 0.05)):
            nodes = [S.translate(S.sphere(float(r2.uniform(0.03, 0.15)), int(r2.integers(0, 4))),
                                 r2.uniform(-0.7, 0.7, 3)) for _ in range(n_prims)]
            acc = nodes[-1]
            for i, nd in enumerate(reversed(nodes[:-1])):
                acc = S.smooth_union(nd, acc, k) if i % 4 else S.union(nd, acc)
            lib.add(acc)
    else:
        chain = shape == "chain"
        lib.add(S.random_sdf_field(256, k=0.1, seed=9, extent=0.8, chain=chain))
        lib.add(S.random_sdf_field(48, k=0.05, seed=3, extent=0.5, chain=chain))
    dr = S.sdf_drawables([np.array([[1, 0, 0, 0.0], [0, 1, 0, -0.2], [0, 0, 1, 0.3], [0, 0, 0, 1]]),
                          np.array([[0.8, 0, 0, 1.2], [0, 0.8, 0, 0.1], [0, 0, 0.8, -0.4], [0, 0, 0, 1]])], [0, 1])
    n = 1 << 16
    rays = np.zeros((n, 8), np.float32)
    o = rng.uniform(-2.5, 2.5, (n, 3))
    o[: n // 4] = rng.uniform(-0.8, 0.8, (n // 4, 3))          # inside the grid
    d = rng.normal(size=(n, 3))
    aim = -o + rng.uniform(-0.4, 0.4, (n, 3))
    d[n // 2:] = aim[n // 2:]                                  # aimed at the field
    rays[:, 0:3] = o
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 7] = np.where(np.arange(n) % 3 == 0, 2.0, np.inf)
    states = rng.integers(1, 2**32, n, dtype=np.uint64).astype(np.uint32)
    res = {}
    try:
        for cells in (1, 0, 8, 96):
            ctx.set_tuning(sdf_cells=cells)
            ctx.upload_sdf(lib.instrs, lib.programs, lib.params, dr)
            res[cells] = [ctx.trace_sdf(rays, 256, 1e-4, any_hit=a, rng_states=states) for a in (False, True)]
    finally:
        ctx.set_tuning()
        ctx.upload_sdf(np.zeros((0, 2)), np.zeros((0, 2)), np.zeros(0), np.zeros((0, 36)))
    full = res[1]
    assert full[0]["hit"].sum() > 2000 and full[1]["hit"].sum() > 2000
    for cells in (0, 8, 96):
        for a in (0, 1):
            for key, v in full[a].items():
                assert np.array_equal(res[cells][a][key], v), (cells, a, key)
    sub = slice(0, n, 16)
    ora = po.sdf_trace(lib, dr, rays[sub], 256, 1e-4, False, states[sub])
    for key in ("hit", "t", "normal", "material"):
        assert np.array_equal(res[0][0][key][sub], ora[key]), key


def test_sdf_library_emits_deep_folds():
    """The flat-program emitter walks the tree without recursion: a left fold of
    3,000 translated spheres serialises in post order (translate, sphere, then
    translate, sphere, smooth union per further primitive)."""
    n = 3000
    acc = S.translate(S.sphere(0.1, 1), (0.0, 0.0, 0.0))
    for i in range(1, n):
        acc = S.smooth_union(acc, S.translate(S.sphere(0.1, 1), (0.01 * i, 0.0, 0.0)), 0.05)
    lib = S.SdfLibrary()
    assert lib.add(acc) == 0
    ops = lib.instrs[:, 0]
    assert lib.programs.tolist() == [[0, 3 * n - 1]]
    assert ops[:2].tolist() == [S.TRANSLATE, S.SPHERE]
    assert (ops[2:].reshape(-1, 3) == [S.TRANSLATE, S.SPHERE, S.SMOOTH_UNION]).all()
    # parameter offsets point at each translation's own x offset
    offs = lib.instrs[2::3, 1]
    assert np.allclose(lib.params[offs], 0.01 * np.arange(1, n))
