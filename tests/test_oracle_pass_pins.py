"""The oracle's restated reference-shading passes against the reference's own
pt_generate.comp and pt_color.comp, compiled as C++ by oracle/build_ref.py:
bit for bit on the same buffers. The color pass runs on synthetic trace
records that reach every branch (light hits, misses to the sky, Russian
roulette, the degenerate-pdf exits, next-event light terms), over several
PBR materials, for a first and a later sample and with force_write_color."""
import numpy as np
import pytest

import pyoracle as po
from myrt_b200.camera import look_at
from myrt_b200.scenes import pack_unorm4x8, pbr_material

pytestmark = pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref not built")

W, H = 32, 24  # multiples of pt_generate's 8x8 work group


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _random_tex(seed):
    return np.random.default_rng(seed).random(1024, dtype=np.float32)


def _camera():
    return look_at((0.3, 1.0, -3.0), (0.0, 0.0, 0.0), vfov_deg=50, aspect=W / H)


@pytest.mark.parametrize("dof", [False, True])
def test_generate_pass_pinned(dof):
    iv, ip = _camera()
    tex = _random_tex(1)
    rng = np.random.default_rng(2)
    bokeh = None
    if dof:  # a mask with dark texels, so bokeh_get retries
        bokeh = np.zeros((16, 16, 4), np.float32)
        bokeh[..., :3] = (rng.random((16, 16, 1)) > 0.5) * rng.random((16, 16, 3))
        bokeh[..., 3] = 1.0
    kw = dict(dof=dof, lens=(0.3, 0.2), focus=2.5, bokeh=bokeh, bokeh_wrap=0)
    a = po.pass_generate(W, H, iv, ip, 12345, tex, **kw)
    b = po.pass_generate(W, H, iv, ip, 12345, tex, use_ref=True, **kw)
    assert np.array_equal(_bits(a), _bits(b))
    assert np.isfinite(a).all() and np.abs(a[:, 4:7]).max() > 0.1  # unit directions written


def _materials():
    mats = [pbr_material([0.8, 0.3, 0.2], ior=1.5, roughness=0.6),
            pbr_material([0.9, 0.9, 0.9], ior=1.3, roughness=0.05, metallic=1.0),
            pbr_material([0.2, 0.5, 0.9], ior=1.45, roughness=0.3, transmission=0.8),
            pbr_material([0.5, 0.5, 0.5], ior=1.1, roughness=1.0, metallic=0.3, transmission=0.2)]
    data = np.concatenate(mats).astype(np.float32)
    refs = np.stack([np.zeros(len(mats), np.int32), 7 * np.arange(len(mats), dtype=np.int32)], 1)
    return refs, data


def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)


def _rays(seed):
    rng = np.random.default_rng(seed)
    iv, ip = _camera()
    gen = po.pass_generate(W, H, iv, ip, 777, _random_tex(seed))
    n = gen.shape[0]
    pdf = rng.choice([1.0, 0.9, 0.5, 0.1, 1e-6], n).astype(np.float32)
    gen[:, 16] = pdf                                            # pdf
    gen[:, 8:11] = rng.random((n, 3), dtype=np.float32)       # reflectance
    gen[:, 12:16] = 0.1 * rng.random((n, 4), dtype=np.float32)  # colour so far
    tr = np.zeros((n, 16), np.float32)
    tr[:, 0:3] = rng.uniform(-1, 1, (n, 3))
    tr[:, 3] = rng.choice([0, 1, 1, 1, 2], n).astype(np.int32).view(np.float32)
    tr[:, 4:7] = _unit(rng, n)  # random orientation: some face the ray, some face away
    tr[:, 7] = np.arange(n, dtype=np.uint32).view(np.float32)
    tr[:, 8:10] = rng.random((n, 2), dtype=np.float32)
    tr[:, 10] = rng.integers(0, 4, n).astype(np.int32).view(np.float32)
    colors = [pack_unorm4x8(rng.random(4)) for _ in range(n)]
    tr[:, 11] = np.array(colors, np.uint32).view(np.float32)
    tr[:, 12:15] = _unit(rng, n)
    tr[:, 15] = np.where(rng.random(n) < 0.3, 0.0, rng.uniform(0.0, 5.0, n)).astype(np.float32)
    return gen, tr


@pytest.mark.parametrize("sample_index,force", [(0, 0), (3, 0), (5, 1)])
def test_color_pass_pinned(sample_index, force):
    gen, tr = _rays(10 + sample_index)
    refs, data = _materials()
    rng = np.random.default_rng(4)
    acc = np.zeros((H, W, 4), np.float32)
    if sample_index:
        acc[..., :3] = rng.random((H, W, 3), dtype=np.float32) * sample_index
        acc[..., 3] = sample_index
    disp = np.zeros((H, W, 4), np.float32)
    tex = _random_tex(20 + sample_index)
    a = po.pass_color(gen, tr, acc, disp, sample_index, force, 4242, tex, refs, data)
    b = po.pass_color(gen, tr, acc, disp, sample_index, force, 4242, tex, refs, data, use_ref=True)
    for x, y in zip(a, b):
        assert np.array_equal(_bits(x), _bits(y))
    alive = a[1][:, 3].view(np.int32)
    if force:  # force_write_color finishes every ray that hit something
        assert (alive == 0).all()
    else:  # the branches were taken: some rays continue (gen changed), some finished
        assert (alive == 0).any() and (alive == 1).any()
        assert not np.array_equal(_bits(a[0]), _bits(gen))
