"""numpy restatement of the guide network (myrt_b200/csrc/guide.cu): encoding,
MLP forward with the device's BF16 rounding points, vMF mixture, the loss
-w log q(d | x) and its gradient by backpropagation.

TEST INFRASTRUCTURE ONLY (checker of the tensor-core kernels). Imported by
tests/ only.
"""
from __future__ import annotations

import numpy as np

LOBES = 8
LAYERS = 4
W = 64
N_PARAMS = LAYERS * W * W + LAYERS * W
KAPPA_MIN, KAPPA_MAX = 0.01, 1000.0


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(x, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out).astype(np.float32)


def split(params):
    p = np.asarray(params, np.float32)
    return p[: LAYERS * W * W].reshape(LAYERS, W, W), p[LAYERS * W * W:].reshape(LAYERS, W)


def encode(pos, nrm, wo, bounds) -> np.ndarray:
    lo, hi = np.asarray(bounds[:3], np.float32), np.asarray(bounds[3:], np.float32)
    c = np.float32(0.5) * (lo + hi)
    h = np.float32(0.5) * (hi - lo)
    inv = np.where(h > 0, np.float32(1) / np.where(h > 0, h, 1), np.float32(1)).astype(np.float32)
    pn = np.clip((np.asarray(pos, np.float32) - c) * inv, -1, 1).astype(np.float32)
    n = pn.shape[0]
    f = np.zeros((n, 64), np.float64)
    f[:, 0:3] = pn
    for fr in range(6):
        ang = np.pi * pn.astype(np.float64) * (1 << fr)
        for k in range(3):
            f[:, 3 + 6 * fr + 2 * k] = np.sin(ang[:, k])
            f[:, 4 + 6 * fr + 2 * k] = np.cos(ang[:, k])
    f[:, 39:42] = nrm
    f[:, 42:45] = wo
    f[:, 45] = 1.0
    return f.astype(np.float32)


def forward(params, X):
    """Returns (H list (bf16-rounded inputs of each layer), out float64)."""
    Wt, b = split(params)
    Wb = bf16(Wt).astype(np.float64)
    H = [bf16(X)]
    z = None
    for l in range(LAYERS):
        z = (H[l].astype(np.float64) @ Wb[l].T + b[l]).astype(np.float32)
        if l < LAYERS - 1:
            H.append(bf16(np.maximum(z, 0)))
    return H, z.astype(np.float64)


def mixture(out):
    o = np.asarray(out, np.float64)
    logits = o[:, 0::5][:, :LOBES]
    x = o[:, 1::5][:, :LOBES]
    m = np.stack([o[:, 2 + 5 * k: 5 + 5 * k] for k in range(LOBES)], 1)  # [n, 8, 3]
    w = np.exp(logits - logits.max(1, keepdims=True))
    w /= w.sum(1, keepdims=True)
    sp = np.where(x > 20, x, np.log1p(np.exp(np.minimum(x, 20))))
    kap = sp + KAPPA_MIN
    dk = 1 / (1 + np.exp(-x))
    clamp = kap > KAPPA_MAX
    kap = np.where(clamp, KAPPA_MAX, kap)
    dk = np.where(clamp, 0.0, dk)
    ln = np.linalg.norm(m, axis=2)
    mu = np.where(ln[..., None] > 1e-6, m / np.maximum(ln, 1e-30)[..., None], np.array([0, 0, 1.0]))
    return w, kap, mu, ln, dk


def vmf_norm(k):
    return k / (-2 * np.pi * np.expm1(-2 * k))


def lobes_array(out):
    """Device lobe layout [n, 64]: 8 x (mu, kappa), 8 x (w, norm, cdf, valid)."""
    w, kap, mu, _, _ = mixture(out)
    n = w.shape[0]
    res = np.zeros((n, 64))
    for k in range(LOBES):
        res[:, 4 * k: 4 * k + 3] = mu[:, k]
        res[:, 4 * k + 3] = kap[:, k]
        res[:, 32 + 4 * k] = w[:, k]
        res[:, 33 + 4 * k] = vmf_norm(kap[:, k])
        res[:, 34 + 4 * k] = 1.0 if k == LOBES - 1 else w[:, : k + 1].sum(1)
    res[:, 35] = 1.0
    return res


def pdf(out, d):
    w, kap, mu, _, _ = mixture(out)
    c = np.einsum("nkc,nc->nk", mu, d)
    return (w * vmf_norm(kap) * np.exp(kap * (c - 1))).sum(1)


def loss_grad_out(out, d, wgt):
    """d loss / d out (40 used) for loss_i = -w_i log q_i; float64."""
    w, kap, mu, ln, dk = mixture(out)
    c = np.einsum("nkc,nc->nk", mu, d)
    fk = vmf_norm(kap) * np.exp(kap * (c - 1))
    q = (w * fk).sum(1)
    g = np.zeros((out.shape[0], 64))
    ok = (wgt > 0) & (q > 1e-30)
    gq = np.where(ok, -wgt / np.where(ok, q, 1), 0.0)
    for k in range(LOBES):
        wf = w[:, k] * fk[:, k]
        g[:, 5 * k] = gq * w[:, k] * (fk[:, k] - q)
        dlnc = 1 / kap[:, k] - 2 / np.expm1(2 * kap[:, k])
        g[:, 5 * k + 1] = gq * wf * (dlnc + (c[:, k] - 1)) * dk[:, k]
        gm = gq * wf * kap[:, k]
        dmu = gm[:, None] * d
        proj = (dmu * mu[:, k]).sum(1)
        good = ln[:, k] > 1e-6
        g[:, 5 * k + 2: 5 * k + 5] = np.where(good[:, None], (dmu - proj[:, None] * mu[:, k]) /
                                               np.maximum(ln[:, k], 1e-30)[:, None], 0.0)
    loss = np.where(ok, -wgt * np.log(np.where(ok, q, 1)), 0.0).sum()
    return g, loss


def gradients(params, samples, bounds):
    """Parameter gradient of sum_i -w_i log q(d_i | x_i) with the device's
    rounding points (BF16 activations and output gradients); float64."""
    s = np.asarray(samples, np.float32).reshape(-1, 16)
    X = encode(s[:, 0:3], s[:, 4:7], s[:, 8:11], bounds)
    H, out = forward(params, X)
    g, loss = loss_grad_out(out, s[:, 12:15].astype(np.float64), s[:, 3].astype(np.float64))
    Wt, _ = split(params)
    Wb = bf16(Wt).astype(np.float64)
    dW = np.zeros((LAYERS, W, W))
    db = np.zeros((LAYERS, W))
    dz = bf16(g.astype(np.float32)).astype(np.float64)
    db[3] = dz.sum(0)
    for l in range(LAYERS - 1, -1, -1):
        dW[l] = dz.T @ H[l].astype(np.float64)
        if l > 0:
            dh = (dz @ Wb[l]).astype(np.float32)
            dz = bf16(np.where(H[l] > 0, dh, 0).astype(np.float32)).astype(np.float64)
            db[l - 1] = dz.sum(0)
    return np.concatenate([dW.ravel(), db.ravel()]), loss


def eval_points(params, points, bounds):
    p = np.asarray(points, np.float32).reshape(-1, 12)
    X = encode(p[:, 0:3], p[:, 4:7], p[:, 8:11], bounds)
    _, out = forward(params, X)
    return lobes_array(out), out
