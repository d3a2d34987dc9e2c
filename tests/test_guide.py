"""Learned path guiding: the vMF-mixture MLP (tcgen05 forward / backward
kernels) against the numpy oracle, its training, and what it gains in
rendering.

Tolerances: the device rounds layer inputs and output gradients to BF16 like
the oracle, but accumulates in FP32 in another order, which can flip a BF16
rounding; lobe parameters are compared within 2e-2 (99 % of entries) and the
gradient vector within 2e-2 relative L2 error.
"""
import numpy as np
import pytest

import pyguide as pg
import pyoracle as po
from myrt_b200.camera import look_at
from myrt_b200.scenes import guiding_box


def _rand_out(n, rng, scale=2.0):
    return rng.normal(0, scale, (n, 64))


def _unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def test_mixture_pdf_normalised():
    rng = np.random.default_rng(1)
    out = _rand_out(4, rng, 3.0)
    # Fibonacci sphere quadrature
    m = 200000
    i = np.arange(m) + 0.5
    z = 1 - 2 * i / m
    r = np.sqrt(1 - z * z)
    ph = np.pi * (1 + 5 ** 0.5) * i
    d = np.stack([r * np.cos(ph), r * np.sin(ph), z], 1)
    for k in range(4):
        q = pg.pdf(np.repeat(out[k:k + 1], m, 0), d)
        assert abs(q.mean() * 4 * np.pi - 1) < 2e-3


def test_loss_gradient_matches_finite_differences():
    rng = np.random.default_rng(2)
    n = 6
    out = _rand_out(n, rng, 1.5)
    d = _unit(rng.normal(size=(n, 3)))
    w = rng.uniform(0.5, 2, n)
    g, _ = pg.loss_grad_out(out, d, w)
    eps = 1e-6
    for j in list(range(40)):
        o1, o2 = out.copy(), out.copy()
        o1[:, j] += eps
        o2[:, j] -= eps
        fd = (-w * np.log(pg.pdf(o1, d)) + w * np.log(pg.pdf(o2, d))) / (2 * eps)
        np.testing.assert_allclose(g[:, j], fd, rtol=1e-4, atol=1e-6)


def test_backprop_matches_finite_differences():
    """Parameter gradient of the oracle's backward pass (rounding disabled by
    using BF16-exact parameters and inputs that stay away from ReLU kinks)."""
    rng = np.random.default_rng(3)
    params = pg.bf16(rng.normal(0, 0.2, pg.N_PARAMS).astype(np.float32))
    bounds = np.array([-1, -1, -1, 1, 1, 1], np.float32)
    s = np.zeros((3, 16), np.float32)
    s[:, 0:3] = rng.uniform(-0.9, 0.9, (3, 3))
    s[:, 3] = 1.0
    s[:, 4:7] = _unit(rng.normal(size=(3, 3)))
    s[:, 8:11] = _unit(rng.normal(size=(3, 3)))
    s[:, 12:15] = _unit(rng.normal(size=(3, 3)))

    def loss_fp64(p):
        X = pg.encode(s[:, 0:3], s[:, 4:7], s[:, 8:11], bounds).astype(np.float64)
        Wt, b = p[:4 * 4096].reshape(4, 64, 64), p[4 * 4096:].reshape(4, 64)  # float64: keep the FD step
        h = X
        for l in range(4):
            z = h @ Wt[l].T + b[l]
            h = np.maximum(z, 0) if l < 3 else z
        return (-s[:, 3] * np.log(pg.pdf(h, s[:, 12:15].astype(np.float64)))).sum()

    # exact-arithmetic gradient: the oracle's formulas without BF16 rounding
    X = pg.encode(s[:, 0:3], s[:, 4:7], s[:, 8:11], bounds).astype(np.float64)
    Wt, b = pg.split(params)
    hs, h = [X], X
    for l in range(4):
        z = h @ Wt[l].astype(np.float64).T + b[l]
        h = np.maximum(z, 0) if l < 3 else z
        if l < 3:
            hs.append(h)
    g, _ = pg.loss_grad_out(h, s[:, 12:15].astype(np.float64), s[:, 3].astype(np.float64))
    dz = g
    grads = np.zeros((4, 64, 64))
    for l in range(3, -1, -1):
        grads[l] = dz.T @ hs[l]
        if l:
            dz = (dz @ Wt[l].astype(np.float64)) * (hs[l] > 0)
    for (l, o, i) in [(3, 0, 0), (3, 6, 45), (2, 5, 7), (0, 3, 39), (1, 10, 20)]:
        p1, p2 = params.astype(np.float64).copy(), params.astype(np.float64).copy()
        k = (l * 64 + o) * 64 + i
        p1[k] += 1e-6
        p2[k] -= 1e-6
        fd = (loss_fp64(p1) - loss_fp64(p2)) / 2e-6
        assert abs(fd - grads[l, o, i]) <= 1e-4 * max(1.0, abs(fd)), (l, o, i, fd, grads[l, o, i])


def _points(rng, n, lo=-1.0, hi=1.0):
    p = np.zeros((n, 12), np.float32)
    p[:, 0:3] = rng.uniform(lo, hi, (n, 3))
    p[:, 3] = 1.0
    p[:, 4:7] = _unit(rng.normal(size=(n, 3)))
    wo = _unit(rng.normal(size=(n, 3)))
    wo *= np.sign((wo * p[:, 4:7]).sum(1, keepdims=True))
    p[:, 8:11] = wo
    return p


def _sharpen(ctx, rng):
    """Initial parameters with the output layer scaled up, so lobes differ."""
    prm = ctx.guide_params()
    prm[3 * 4096:4 * 4096] *= 20.0
    prm[4 * 4096 + 3 * 64: 4 * 4096 + 4 * 64] = rng.normal(0, 1, 64)
    ctx.guide_set_params(prm)
    return prm


def _small_box(ctx):
    s, lights = guiding_box(slab_cells=24, wall_cells=4)
    ctx.upload_scene(**s)
    ctx.set_area_lights(lights)
    return s, lights


@pytest.mark.gpu
def test_guide_forward_matches_oracle(ctx):
    rng = np.random.default_rng(4)
    _small_box(ctx)
    ctx.guide_reset()
    prm = _sharpen(ctx, rng)
    pts = _points(rng, 1000)  # not a multiple of 128: ragged last tile
    got = ctx.guide_eval(pts)
    info = ctx.bvh_info()
    bounds = np.array([-1, -1, -1, 1, 1, 1], np.float32)
    ref, _ = pg.eval_points(prm, pts, bounds)
    err = np.abs(got - ref)
    assert np.quantile(err, 0.99) < 2e-2, np.quantile(err, 0.99)
    assert np.median(err) < 1e-3
    assert np.allclose(got[:, 32:64:4].sum(1), 1.0, atol=1e-4)  # weights sum to one
    assert np.all(got[:, 35] == 1.0)
    assert info["triangles"] > 0


@pytest.mark.gpu
def test_guide_gradients_match_oracle(ctx):
    rng = np.random.default_rng(5)
    _small_box(ctx)
    ctx.guide_reset()
    prm = _sharpen(ctx, rng)
    n = 700
    s = np.zeros((n, 16), np.float32)
    pts = _points(rng, n)
    s[:, 0:3], s[:, 4:7], s[:, 8:11] = pts[:, 0:3], pts[:, 4:7], pts[:, 8:11]
    s[:, 3] = rng.uniform(0.1, 2.0, n)
    s[:, 12:15] = _unit(rng.normal(size=(n, 3)))
    g, loss = ctx.guide_gradients(s)
    bounds = np.array([-1, -1, -1, 1, 1, 1], np.float32)
    ref, ref_loss = pg.gradients(prm, s, bounds)
    rel = np.linalg.norm(g - ref) / np.linalg.norm(ref)
    assert rel < 2e-2, rel
    assert abs(loss - ref_loss) / abs(ref_loss) < 1e-3
    for l in range(4):  # every layer's block gets its share
        blk = slice(l * 4096, (l + 1) * 4096)
        assert np.linalg.norm(g[blk] - ref[blk]) / np.linalg.norm(ref[blk]) < 3e-2, l


@pytest.mark.gpu
def test_guide_learns_a_direction_field(ctx):
    """Targets drawn from a vMF (kappa 20) around a position-dependent direction
    mu(x) = normalize(x + (0, 0.5, 0)): training lowers the loss and the learned
    density at mu(x) ends far above the uniform 1 / (4 pi)."""
    rng = np.random.default_rng(6)
    _small_box(ctx)
    ctx.guide_configure(seed=11, learning_rate=1e-2, batch=8192)
    ctx.guide_reset()
    n = 65536
    pts = _points(rng, n)
    mu = _unit(pts[:, 0:3] + np.array([0, 0.5, 0], np.float32))
    # vMF sample around mu (Wood / Jakob)
    u1, u2 = rng.uniform(size=n), rng.uniform(size=n)
    k = 20.0
    w = 1 + np.log(u1 + (1 - u1) * np.exp(-2 * k)) / k
    t = _unit(np.cross(mu, rng.normal(size=(n, 3))))
    b = np.cross(mu, t)
    r = np.sqrt(np.maximum(0, 1 - w * w))
    d = mu * w[:, None] + t * (r * np.cos(2 * np.pi * u2))[:, None] + b * (r * np.sin(2 * np.pi * u2))[:, None]
    s = np.zeros((n, 16), np.float32)
    s[:, 0:3], s[:, 3], s[:, 4:7], s[:, 8:11], s[:, 12:15] = pts[:, 0:3], 1.0, pts[:, 4:7], pts[:, 8:11], d
    losses = ctx.guide_train(s, 400)
    assert losses[-20:].mean() < 0.5 * losses[:5].mean(), (losses[:5], losses[-20:])
    test = _points(rng, 512)
    lob = ctx.guide_eval(test)
    mut = _unit(test[:, 0:3] + np.array([0, 0.5, 0], np.float32))
    out_w = lob[:, 32:64:4]
    norm = lob[:, 33:64:4]
    mus = lob[:, 0:32].reshape(-1, 8, 4)
    q = (out_w * norm * np.exp(mus[..., 3] * ((mus[..., :3] * mut[:, None]).sum(-1) - 1))).sum(1)
    assert np.median(q) > 10 * (1 / (4 * np.pi)), np.median(q)


def _rel_rmse(img, ref):
    return float(np.sqrt(np.mean(((img - ref) / (ref + 1e-2)) ** 2)))


@pytest.mark.gpu
def test_guided_rendering_beats_bsdf_sampling(ctx):
    """The slot box at 128^2 (light reaches the lower levels only through two
    0.2-wide slots): guided rendering with the default settings (fraction 0.5,
    waves growing 1, 2, 4, 8, 16 spp while the guide trains, 16 Adam steps
    after each wave, training weights clamped at 10x their mean, roulette on
    the BSDF-sampling throughput) against plain BSDF sampling at the same 1024
    spp, both against an FP64 plain render of 16384 spp, two render seeds
    each. Guided stays unbiased (image means within 3 %) and its relRMSE is
    well below plain's (measured: 0.058 and 0.059 against 0.128 and 0.130)."""
    _small_box(ctx)
    W = H = 128
    iv, ip = look_at((0.0, 0.0, -0.95), (0.0, 0.0, 0.5), vfov_deg=90, aspect=1.0)
    ctx.reset_accumulation()
    ctx.render_physical(iv, ip, W, H, spp=16384, max_depth=12, rr_start=3, seed=99, fp64=True)
    ref = ctx.read_accumulation_f64(W, H)
    ref = ref[..., :3] / ref[..., 3:4]
    e_plain, e_guided = [], []
    for seed in (1, 2):
        ctx.reset_accumulation()
        ctx.render_physical(iv, ip, W, H, spp=1024, max_depth=12, rr_start=3, seed=seed, wave_paths=W * H * 16)
        plain, _ = ctx.read_accumulation(W, H)
        plain = plain[..., :3] / plain[..., 3:4]
        ctx.guide_configure(fraction=0.5, train=1, warmup_waves=1, train_steps=16, batch=16384,
                            learning_rate=1e-2, weight_clamp=10.0, target=0, seed=3)
        ctx.guide_reset()
        ctx.reset_accumulation()
        ctx.render_physical(iv, ip, W, H, spp=1024, max_depth=12, rr_start=3, seed=seed, guided=True,
                            wave_paths=W * H * 16)
        guided, _ = ctx.read_accumulation(W, H)
        guided = guided[..., :3] / guided[..., 3:4]
        st = ctx.guide_stats()
        assert st["adam_steps"] >= 16 * 63 and st["last_samples"] > 10000
        assert abs(guided.mean() / ref.mean() - 1) < 0.03 and abs(plain.mean() / ref.mean() - 1) < 0.03
        e_plain.append(_rel_rmse(plain, ref))
        e_guided.append(_rel_rmse(guided, ref))
    print("relRMSE plain", e_plain, "guided", e_guided)
    assert np.mean(e_guided) < 0.6 * np.mean(e_plain)


@pytest.mark.gpu
def test_tensor_core_wait_timeout_reports_and_context_recovers(ctx):
    """The first mbarrier wait of every CTA of the forward and training kernels
    is pointed at a barrier nothing arrives at (guide_stall_test) with a limit
    of 64 polls: each CTA gives up, drains its MMA in flight, frees its TMEM and
    returns; myrt_sync reports MYRT_ERR_DEVICE_ABORT with the guide timeout bit
    (1 << 5). With the default tuning the same context then evaluates and trains
    normally, with results equal to those before the stall."""
    import myrt_b200 as mb

    rng = np.random.default_rng(12)
    _small_box(ctx)
    ctx.guide_reset()
    _sharpen(ctx, rng)
    pts = _points(rng, 700)
    ref = ctx.guide_eval(pts)
    ctx.sync()
    n = 512
    s = np.zeros((n, 16), np.float32)
    q = _points(rng, n)
    s[:, 0:3], s[:, 4:7], s[:, 8:11] = q[:, 0:3], q[:, 4:7], q[:, 8:11]
    s[:, 3] = 1.0
    s[:, 12:15] = _unit(rng.normal(size=(n, 3)))
    g_ref, loss_ref = ctx.guide_gradients(s)
    ctx.sync()
    try:
        ctx.set_tuning(guide_poll_limit=64, guide_stall_test=1)
        ctx.guide_eval(pts)
        with pytest.raises(mb.MyrtError, match="0x00000020") as e:
            ctx.sync()
        assert e.value.code == mb.MYRT_ERR_DEVICE_ABORT
        ctx.guide_gradients(s)
        with pytest.raises(mb.MyrtError, match="0x00000020"):
            ctx.sync()
    finally:
        ctx.set_tuning()
    ctx.sync()  # the error word was cleared by the report
    assert np.array_equal(ctx.guide_eval(pts), ref)
    g, loss = ctx.guide_gradients(s)
    ctx.sync()
    # per-warp bias sums meet in shared-memory atomics, so the last bits may move
    np.testing.assert_allclose(g, g_ref, rtol=1e-5, atol=1e-7)
    assert abs(loss - loss_ref) <= 1e-5 * abs(loss_ref)
