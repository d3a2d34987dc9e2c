"""Generates the golden fixtures in tests/golden/ from the reference's own code.

Run in a container that has the reference tree (it builds oracle/_ref first):
    python tests/golden/make_golden.py            (all fixtures)
    python tests/golden/make_golden.py instanced  (instanced_field.npz only)

Every output comes from code compiled from the reference's sources
(oracle/_ref/libmyrt_ref.so; see oracle/build_ref.py), never from the oracle
restatement, so the restatement can be checked against them on machines that
do not have the reference tree.

Fixtures:
  refbvh_hf16.npz   16x16-cell height field (512 triangles): the reference BVH
                    (bvh.cpp) with dont_split and with split_aabbs.
  closest_hf128.npz the 128x128-cell height field (32,768 triangles) of the
                    closest-hit configuration; 4,096 camera rays (every 16th
                    pixel in x and y of the 1024^2 pinhole camera) and 2,048
                    random rays; hits from the reference's CPU pick path
                    (scene::pick over bvh::traverse + ray_t::intersect) and from
                    its GLSL traversal (bvh.impl.glsl + pt_trace.comp visitor),
                    closest and any-hit.
  instanced_field.npz  an instanced scene (48 icospheres and 24 boxes under
                    random rotations, non-uniform scales and translations, plus
                    a floor): 6,912 camera rays and 2,048 random rays through the
                    reference's two-level walk -- geometry trees by bvh.cpp with
                    split_aabbs (scene::push_geometry), the tree over the
                    drawables' world boxes with dont_split (scene::prepare),
                    bvh.impl.glsl with visit_object_aabb (pt_trace.comp:284-309)
                    -- closest and any-hit (shadow rays with finite tmax).
  glsl_kat.npz      known answers of random.glsl, intersect.glsl,
                    transform.glsl, color.glsl and the PBR material
                    (pbr.glsl / ggx.glsl / material_new.glsl) on seeded inputs.
"""
from __future__ import annotations

import ctypes as C
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from myrt_b200.scenes import heightfield, pinhole_rays  # noqa: E402

OUT = Path(__file__).resolve().parent


def random_rays(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    o = np.stack([rng.uniform(-1.5, 1.5, n), rng.uniform(0.2, 2.0, n), rng.uniform(-1.5, 1.5, n)], 1)
    target = np.stack([rng.uniform(-1, 1, n), rng.uniform(0, 0.1, n), rng.uniform(-1, 1, n)], 1)
    d = target - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    # a share of axis-aligned and grazing directions
    d[: n // 16] = np.array([0.0, -1.0, 0.0])
    d[n // 16: n // 8, 1] = -1e-3
    d[n // 16: n // 8] /= np.linalg.norm(d[n // 16: n // 8], axis=1, keepdims=True)
    rays = np.empty((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3] = 0.0
    rays[:, 4:7] = d
    rays[:, 7] = np.inf
    return rays


def main() -> int:
    subprocess.run([sys.executable, str(ROOT / "oracle" / "build.py")], check=True)
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle as po  # noqa: E402

    if not po.ref_available():
        print("oracle/_ref not built (reference tree missing); fixtures unchanged")
        return 1
    L = po.ref()

    # -- reference BVH on a small height field --
    idx16, pts16 = heightfield(16, seed=7)
    out = {"indices": idx16, "points": pts16}
    for split in (False, True):
        h = po.ref_bvh(idx16, pts16, split)
        nodes, bi = po.ref_bvh_arrays(h)
        L.ref_bvh_free(h)
        tag = "split" if split else "nosplit"
        out[f"nodes_{tag}"] = nodes
        out[f"bvh_indices_{tag}"] = bi
    np.savez_compressed(OUT / "refbvh_hf16.npz", **out)

    # -- closest / any hit on the 32,768-triangle height field --
    idx, pts = heightfield(128, seed=1)
    cam = pinhole_rays(1024, 1024).reshape(1024, 1024, 8)[::16, ::16].reshape(-1, 8)
    rays = np.concatenate([cam, random_rays(2048, seed=3)], 0)
    h = po.ref_bvh(idx, pts, True)
    nodes, bi = po.ref_bvh_arrays(h)
    pick = po.ref_pick_closest(h, rays)
    L.ref_bvh_free(h)
    glsl = po.ref_glsl_traverse(nodes, bi, idx, pts, rays)
    anyh = po.ref_glsl_traverse(nodes, bi, idx, pts, rays, any_hit=True)
    # shadow-style rays: towards a point above the surface with a finite tmax
    sh = rays.copy()
    sh[:, 7] = np.where(np.isfinite(glsl["t"]), glsl["t"] * 0.5, 3.0).astype(np.float32)
    any_short = po.ref_glsl_traverse(nodes, bi, idx, pts, sh, any_hit=True)
    np.savez_compressed(OUT / "closest_hf128.npz", indices=idx, points=pts, rays=rays, shadow_rays=sh,
                        pick=pick, glsl=glsl, any_prim=anyh["prim"], any_short_prim=any_short["prim"])

    # -- GLSL known answers --
    rng = np.random.default_rng(11)
    kat = {}
    a = rng.integers(0, 2**32, 256, dtype=np.uint64).astype(np.uint32)
    kat["wang_in"] = a
    kat["wang_out"] = np.array([L.ref_glsl_wang_hash(int(x)) for x in a], np.uint32)
    tex = rng.uniform(0, 1, 1024).astype(np.float32)
    kat["tex"] = tex
    px = rng.integers(0, 2048, (64, 2)).astype(np.int32)
    seeds = rng.integers(0, 2**31 - 1, 64).astype(np.int32)
    streams = np.zeros((64, 32), np.float32)
    states = np.zeros(64, np.uint32)
    for i in range(64):
        st = C.c_uint32()
        L.ref_glsl_random_stream(tex.ctypes.data, 1024, int(px[i, 0]), int(px[i, 1]), int(seeds[i]), 32,
                                 streams[i].ctypes.data, C.byref(st))
        states[i] = st.value
    kat.update(rs_px=px, rs_seed=seeds, rs_stream=streams, rs_state=states)
    # triangle tests incl. shared edges and near-degenerate triangles
    tri = rng.uniform(-1, 1, (512, 9)).astype(np.float32)
    tri[:32, 6:9] = tri[:32, 0:3] + 1e-7  # degenerate
    o = rng.uniform(-2, 2, (512, 3)).astype(np.float32)
    w = rng.dirichlet([1, 1, 1], 512)
    w[32:96] = np.array([0.5, 0.5, 0.0])  # on an edge
    target = (w[:, :1] * tri[:, 0:3] + w[:, 1:2] * tri[:, 3:6] + w[:, 2:3] * tri[:, 6:9])
    d = (target - o)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d = d.astype(np.float32)
    it = np.zeros(512, np.float32)
    ib = np.zeros((512, 2), np.float32)
    ih = np.zeros(512, np.int32)
    for i in range(512):
        t = C.c_float()
        ih[i] = L.ref_glsl_intersect_triangle(o[i].ctypes.data, d[i].ctypes.data, tri[i].ctypes.data, C.byref(t),
                                              ib[i].ctypes.data)
        it[i] = t.value
    kat.update(tri_o=o, tri_d=d, tri_v=tri, tri_hit=ih, tri_t=it, tri_uv=ib)
    s0 = rng.uniform(-1, 1, (128, 3)).astype(np.float32)
    sr = rng.uniform(0.1, 1.5, 128).astype(np.float32)
    kat["sph_o"], kat["sph_d"], kat["sph_c"], kat["sph_r"] = o[:128], d[:128], s0, sr
    kat["sph_t"] = np.array([L.ref_glsl_intersect_sphere(o[i].ctypes.data, d[i].ctypes.data, s0[i].ctypes.data,
                                                         float(sr[i])) for i in range(128)], np.float32)
    vv = rng.normal(size=(128, 3)).astype(np.float32)
    nn = rng.normal(size=(128, 3)).astype(np.float32)
    nn /= np.linalg.norm(nn, axis=1, keepdims=True)
    nn[:8] = np.array([1.0, 0.0, 0.0], np.float32)  # parallel to the first helper axis
    tl = np.zeros((128, 3), np.float32)
    for i in range(128):
        L.ref_glsl_transform_local_to_world(vv[i].ctypes.data, nn[i].ctypes.data, tl[i].ctypes.data)
    kat.update(tlw_v=vv, tlw_n=nn, tlw_out=tl)
    col = rng.uniform(-0.2, 1.2, (64, 4)).astype(np.float32)
    kat["pack_in"] = col
    kat["pack_out"] = np.array([L.ref_glsl_pack_unorm4x8(c.ctypes.data) for c in col], np.uint32)
    # PBR material: bounce + evaluate from a given RNG state, then NEE evaluate
    nm = 256
    mats = np.zeros((nm, 7), np.float32)
    alb = rng.uniform(0, 1, (nm, 4)).astype(np.float32)
    alb[:, 3] = 1.0
    packed = np.array([L.ref_glsl_pack_unorm4x8(c.ctypes.data) for c in alb], np.uint32)
    mats[:, 0] = packed.view(np.float32)
    mats[:, 1] = rng.uniform(1.0, 2.0, nm)
    mats[:, 2] = rng.uniform(0.02, 1.0, nm)
    mats[:, 3] = (rng.uniform(0, 1, nm) < 0.3).astype(np.float32)
    mats[:, 4] = np.where(rng.uniform(0, 1, nm) < 0.2, rng.uniform(0, 1, nm), 0.0)
    tv = rng.normal(size=(nm, 3)).astype(np.float32)
    tv /= np.linalg.norm(tv, axis=1, keepdims=True)
    nrm = rng.normal(size=(nm, 3)).astype(np.float32)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    rng_in = np.stack([rng.integers(1, 2**32, nm, dtype=np.uint64).astype(np.uint32),
                       rng.integers(0, 6, nm).astype(np.uint32)], 1)
    gen = np.zeros((nm, 3), np.float32)
    refl = np.zeros((nm, 3), np.float32)
    pdf = np.zeros(nm, np.float32)
    lobe = np.zeros(nm, np.int32)
    resample = np.zeros(nm, np.float32)
    rng_out = rng_in.copy()
    ltd = rng.normal(size=(nm, 3)).astype(np.float32)
    ltd /= np.linalg.norm(ltd, axis=1, keepdims=True)
    nee_refl = np.zeros((nm, 3), np.float32)
    nee_pdf = np.zeros(nm, np.float32)
    for i in range(nm):
        io = rng_out[i].copy()
        pd = C.c_float()
        lb = C.c_int()
        rs = C.c_float()
        L.ref_glsl_material_bounce_eval(mats[i].ctypes.data, io.ctypes.data, tv[i].ctypes.data, nrm[i].ctypes.data,
                                        gen[i].ctypes.data, refl[i].ctypes.data, C.byref(pd), C.byref(lb),
                                        C.byref(rs))
        rng_out[i] = io
        pdf[i], lobe[i], resample[i] = pd.value, lb.value, rs.value
        pd2 = C.c_float()
        L.ref_glsl_material_eval(mats[i].ctypes.data, int(lb.value), float(rs.value), ltd[i].ctypes.data,
                                 tv[i].ctypes.data, nrm[i].ctypes.data, nee_refl[i].ctypes.data, C.byref(pd2))
        nee_pdf[i] = pd2.value
    kat.update(mat=mats, mat_tv=tv, mat_n=nrm, mat_rng_in=rng_in, mat_rng_out=rng_out, mat_gen=gen, mat_refl=refl,
               mat_pdf=pdf, mat_lobe=lobe, mat_resample=resample, mat_ltd=ltd, mat_nee_refl=nee_refl,
               mat_nee_pdf=nee_pdf)
    np.savez_compressed(OUT / "glsl_kat.npz", **kat)

    # -- SDF: the reference's raymarch.glsl + sdf.hpp snippets (compiled in _ref) --
    from myrt_b200 import sdf as S

    lib = S.SdfLibrary()
    lib.add(S.random_sdf_field(48, seed=5))
    lib.add(S.smooth_union(S.mirror_axis(S.translate(S.sphere(0.3, 1), (0.4, 0.0, 0.0)), 0),
                           S.union(S.box((0.2, 0.3, 0.1), 2),
                                   S.subtraction(S.torus(0.5, 0.1, 3), S.vertical_capsule(0.5, 0.15, 4))), 0.2))
    lib.add(S.intersection(S.menger_fractal(5), S.box((0.9, 0.9, 0.9), 6)))
    pts = rng.uniform(-1.2, 1.2, (2048, 3)).astype(np.float32)
    states = rng.integers(1, 2**32, 2048, dtype=np.uint64).astype(np.uint32)
    sk = dict(instrs=lib.instrs, programs=lib.programs, params=lib.params, pts=pts, states=states)
    for prog in range(3):
        for load in (0, 1):
            d, m = po.sdf_map(lib, prog, pts, bool(load), states, use_ref=True)
            sk[f"map{prog}_{load}_d"], sk[f"map{prog}_{load}_m"] = d, m
    shift = np.array([[1, 0, 0, 0.3], [0, 1, 0, -0.1], [0, 0, 1, 0.2], [0, 0, 0, 1.0]])
    scale = np.diag([0.8, 1.2, 1.0, 1.0])
    dr = S.sdf_drawables([np.eye(4), shift @ scale, np.eye(4)], [1, 0, 2])
    rays = np.zeros((1536, 8), np.float32)
    rays[:, 0:3] = rng.uniform(-2, 2, (1536, 3))
    dd = rng.normal(size=(1536, 3))
    rays[:, 4:7] = dd / np.linalg.norm(dd, axis=1, keepdims=True)
    rays[:, 7] = np.inf
    aim = rng.uniform(-0.3, 0.3, (512, 3)) + np.array([0.0, 0.0, 1.0])
    rays[::3, 0:3] = np.array([0.0, 0.0, -3.0])
    rays[::3, 4:7] = aim / np.linalg.norm(aim, axis=1, keepdims=True)
    rays[1::7, 7] = 2.5
    sk.update(drawables=dr, rays=rays)
    for anyh in (0, 1):
        res = po.sdf_trace(lib, dr, rays, 256, 1e-4, bool(anyh), states[:1536], use_ref=True)
        for k, v in res.items():
            sk[f"trace{anyh}_{k}"] = v
    np.savez_compressed(OUT / "sdf_kat.npz", **sk)
    make_post_kat()
    make_instanced()
    for f in sorted(OUT.glob("*.npz")):
        print(f.name, f.stat().st_size)
    return 0


POST_CASES = [  # (name, op, i, p): the reference's post-processing shaders
    ("denoise", 0, (0, 0, 0), (10.0, 0.05, 0.0, 0.0)),
    ("denoise_wide", 0, (0, 0, 0), (2.0, 0.3, 0.0, 0.0)),
    ("blur_x", 1, (0, 0, 0), (1.25, 0.0, 0.0, 0.0)),
    ("blur_y", 1, (1, 0, 0), (2.5, 0.0, 0.0, 0.0)),
    ("cutoff_above", 2, (1, 0, 0), (1.0, 1.0, 1.0, 1.0)),
    ("cutoff_below", 2, (0, 0, 0), (0.5, 0.7, 0.9, 1.1)),
    ("add", 3, (0, 0, 0), (0.3, 0.0, 0.0, 0.0)),
    ("tonemap", 4, (0, 0, 0), (0.0, 0.0, 0.0, 0.0)),
    ("fxaa", 5, (0, 0, 0), (0.0, 0.0, 0.0, 0.0)),
]


def make_instanced() -> None:
    """instanced_field.npz (see the module docstring)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle as po

    from myrt_b200.scenes import instanced_field

    sc = instanced_field()
    cam = pinhole_rays(96, 72, eye=(0.3, 1.5, -3.5), target=(0.0, -0.2, 0.0), vfov_deg=55)
    rng = np.random.default_rng(41)
    n = 2048
    o = rng.uniform(-2.5, 2.5, (n, 3))
    tgt = rng.uniform(-1.0, 1.0, (n, 3))
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rnd = np.zeros((n, 8), np.float32)
    rnd[:, 0:3], rnd[:, 4:7], rnd[:, 7] = o, d, np.inf
    rays = np.concatenate([cam, rnd], 0)
    geom, local, hits = po.ref_instanced(sc, rays)
    sh = rays.copy()
    # just past the first hit (occluded) on even rays, halfway to it on odd rays, 2.0 on misses
    scale = np.where(np.arange(sh.shape[0]) % 2 == 0, 1.001, 0.5)
    sh[:, 7] = np.where(hits["prim"] >= 0, hits["t"] * scale, 2.0).astype(np.float32)
    sgeom, _, shadow = po.ref_instanced(sc, sh, any_hit=True)
    raw = po._drawables_with_bases(sc, {k: (0, 0) for k in po._geometries(sc)[0]})
    raw[:, 32:34] = 0
    np.savez_compressed(OUT / "instanced_field.npz", indices=sc["indices"], vertices=sc["vertices"],
                        drawables=raw, rays=rays, drawable=geom, local_prim=local, hits=hits, shadow_rays=sh,
                        shadow_hit=sgeom >= 0)


def make_post_kat() -> None:
    """post_kat.npz: the reference's pp_*.comp shaders (compiled in oracle/_ref
    with the GL-sampling shim of oracle/ref_harness_post.cpp) on seeded
    RGBA16F images of odd sizes."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle as po

    rng = np.random.default_rng(31)
    img = rng.uniform(0.0, 1.6, (37, 53, 4)).astype(np.float16).astype(np.float32)
    ldr = rng.uniform(0.0, 1.0, (37, 53, 4)).astype(np.float16).astype(np.float32)
    ov = rng.uniform(0.0, 2.0, (19, 27, 4)).astype(np.float16).astype(np.float32)
    kat = dict(img=img, ldr=ldr, overlay=ov)
    for name, op, i, p in POST_CASES:
        src = ldr if op == 0 else img
        kat[name] = po.ref_post_pass(op, src, i=i, p=p, overlay=ov if op == 3 else None)
    np.savez_compressed(OUT / "post_kat.npz", **kat)


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "post":
        make_post_kat()
        sys.exit(0)
    if len(sys.argv) > 1 and sys.argv[1] == "instanced":
        make_instanced()
        sys.exit(0)
    sys.exit(main())
