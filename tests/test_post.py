"""Post-processing passes (src/pt/pp_*.comp, post_process.cpp, main.cpp:840-875).

CPU: the oracle's half rounding against numpy's float16, and properties of the
oracle's passes. GPU: every pass against the oracle on odd-sized images,
bit-exact; denoise and tonemap call exp / pow, which are the library's GLSL
built-ins (glmath.hpp) on the device and in the oracle when it is switched to
them (its default, the host libm, pins it to the reference's compiled
pp_*.comp).
"""
import numpy as np
import pytest

import pyoracle as po

DENOISE, BLUR, CUTOFF, ADD, TONEMAP, FXAA, SCALE = range(7)


def _img(h, w, seed, hi=2.0, band=3.0):
    rng = np.random.default_rng(seed)
    a = rng.uniform(0.0, hi, (h, w, 4)).astype(np.float32)
    a[h // 3: h // 2, :, :3] *= band  # a bright band for cutoff / bloom
    return a.astype(np.float16).astype(np.float32)  # the reference's RGBA16F inputs


def test_half_rounding_matches_numpy():
    rng = np.random.default_rng(1)
    v = np.concatenate([rng.normal(0, 1, 20000), rng.normal(0, 1e-5, 5000), rng.normal(0, 3e4, 5000),
                        np.array([65504, 65519.99, 65520, 65536, 1e9, -65520, 2.0 ** -24, 2.0 ** -25,
                                  1.5 * 2.0 ** -25, 2.0 ** -14, 0.0, -0.0])]).astype(np.float32)
    L = po.oracle()
    got = np.array([L.oracle_half_rn(float(x)) for x in v], np.float32)
    with np.errstate(over="ignore"):
        ref = v.astype(np.float16).astype(np.float32)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


POST_CASES = [("denoise", DENOISE, (0, 0, 0), (10.0, 0.05, 0.0, 0.0)),
              ("denoise_wide", DENOISE, (0, 0, 0), (2.0, 0.3, 0.0, 0.0)),
              ("blur_x", BLUR, (0, 0, 0), (1.25, 0.0, 0.0, 0.0)), ("blur_y", BLUR, (1, 0, 0), (2.5, 0.0, 0.0, 0.0)),
              ("cutoff_above", CUTOFF, (1, 0, 0), (1.0, 1.0, 1.0, 1.0)),
              ("cutoff_below", CUTOFF, (0, 0, 0), (0.5, 0.7, 0.9, 1.1)), ("add", ADD, (0, 0, 0), (0.3, 0.0, 0.0, 0.0)),
              ("tonemap", TONEMAP, (0, 0, 0), (0.0, 0.0, 0.0, 0.0)), ("fxaa", FXAA, (0, 0, 0), (0.0, 0.0, 0.0, 0.0))]


@pytest.mark.parametrize("name,op,i,p", POST_CASES)
def test_oracle_matches_reference_shaders(golden, name, op, i, p):
    """The restatement against the reference's own pp_*.comp shaders, compiled
    as C++ (golden vectors from oracle/_ref; tests/golden/make_golden.py post):
    bit-exact, the host libm on both sides."""
    k = golden("post_kat.npz")
    src = k["ldr"] if op == DENOISE else k["img"]
    got = po.post_pass(op, src, i=i, p=p, overlay=k["overlay"] if op == ADD else None)
    assert np.array_equal(got.view(np.uint32), k[name].view(np.uint32))


def test_oracle_pass_properties():
    a = np.full((9, 13, 4), 0.5, np.float32)
    # the 31 blur weights sum to 1 within float rounding
    b = po.post_pass(BLUR, a, i=(1, 0, 0), p=(1.25, 0, 0, 0))
    assert np.allclose(b, 0.5, atol=2e-3)
    # FXAA keeps a constant image (alpha set to 1)
    f = po.post_pass(FXAA, a)
    assert np.allclose(f[..., :3], 0.5) and np.all(f[..., 3] == 1.0)
    # cutoff zeroes channels at or below the threshold
    img = _img(7, 5, 2)
    c = po.post_pass(CUTOFF, img, i=(1, 0, 0), p=(1, 1, 1, 1))
    assert np.array_equal(c, np.where(img <= 1.0, 0.0, img).astype(np.float32))
    # scale by 1 reproduces the image
    s = po.post_pass(SCALE, img, out_size=img.shape[:2])
    assert np.array_equal(s, img)
    # filmic curve: 0 below the toe, monotone above
    t = po.post_pass(TONEMAP, np.linspace(0, 4, 64, dtype=np.float32).repeat(4).reshape(1, 64, 4), i=(1, 0, 0))
    assert t[0, 0, 0] == 0.0 and np.all(np.diff(t[0, :, 0]) >= 0) and np.all(t[..., 3] == 1.0)


@pytest.mark.gpu
@pytest.mark.parametrize("op,i,p", [
    (BLUR, (0, 0, 0), (1.25, 0, 0, 0)), (BLUR, (1, 0, 0), (2.5, 0, 0, 0)),
    (CUTOFF, (1, 0, 0), (1, 1, 1, 1)), (CUTOFF, (0, 0, 0), (0.5, 0.7, 0.9, 1.1)),
    (ADD, (0, 0, 0), (0.3, 0, 0, 0)), (FXAA, (0, 0, 0), (0, 0, 0, 0)),
    (SCALE, (0, 0, 0), (0, 0, 0, 0)),
])
def test_pass_bit_exact(ctx, op, i, p):
    import torch

    from myrt_b200 import post

    img = _img(45, 67, 3)
    ov = _img(23, 33, 4)
    out_size = (17, 29) if op == SCALE else None
    got = post.run(ctx, op, torch.from_numpy(img).cuda(), i=i, p=p,
                   overlay=torch.from_numpy(ov).cuda() if op == ADD else None, out_size=out_size)
    ref = po.post_pass(op, img, i=i, p=p, overlay=ov if op == ADD else None, out_size=out_size)
    assert np.array_equal(got.cpu().numpy(), ref)


@pytest.mark.gpu
@pytest.mark.parametrize("op,i,p", [(DENOISE, (0, 0, 0), (10.0, 0.05, 0, 0)), (DENOISE, (0, 0, 0), (2.0, 0.3, 0, 0)),
                                    (TONEMAP, (1, 0, 0), (0, 0, 0, 0)), (TONEMAP, (0, 0, 0), (0, 0, 0, 0))])
def test_pass_transcendental(ctx, op, i, p):
    import torch

    from myrt_b200 import post

    # denoise on display-range input: where a centre is far above 1 every range
    # weight underflows and both sides divide (near) zero by (near) zero
    img = _img(45, 67, 5, hi=1.0, band=1.0) if op == DENOISE else _img(45, 67, 5, hi=1.2)
    got = post.run(ctx, op, torch.from_numpy(img).cuda(), i=i, p=p).cpu().numpy()
    with po.glsl_math(1):
        ref = po.post_pass(op, img, i=i, p=p)
    assert np.array_equal(got, ref, equal_nan=True)


@pytest.mark.gpu
def test_frame_chain_matches_oracle(ctx):
    """main.cpp's frame chain (down-scale 1/1.5, bloom, tonemap, FXAA) composed
    on the device and from the oracle's passes."""
    import torch

    from myrt_b200 import post

    img = _img(96, 128, 7, hi=3.0)
    got = post.frame(ctx, torch.from_numpy(img).cuda(), super_sampling=1.5).cpu().numpy()

    def oscale(a, f):
        return po.post_pass(SCALE, a, out_size=post.scaled_size(a.shape[0], a.shape[1], f))

    with po.glsl_math(1):
        ref = _oracle_frame(img, oscale)
    assert got.shape == ref.shape == (64, 85, 4)
    assert np.array_equal(got, ref, equal_nan=True)


def _oracle_frame(img, oscale):
    r = oscale(img, 1.0 / 1.5)
    b = po.post_pass(CUTOFF, r, i=(1, 0, 0), p=(1, 1, 1, 1))
    b = po.post_pass(CUTOFF, b, i=(1, 0, 0), p=(1, 1, 1, 1))
    b = oscale(b, 0.5)
    b = po.post_pass(BLUR, po.post_pass(BLUR, b, i=(0, 0, 0), p=(1.25, 0, 0, 0)), i=(1, 0, 0), p=(1.25, 0, 0, 0))
    b = oscale(b, 2.0)
    r = po.post_pass(ADD, r, p=(0.3, 0, 0, 0), overlay=b)
    r = po.post_pass(TONEMAP, r, i=(1, 0, 0))
    return po.post_pass(FXAA, r)
