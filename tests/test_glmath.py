"""The library's GLSL built-ins (myrt_b200/csrc/glmath.hpp): sin, cos, atan,
exp and pow as the reference shading, the forward resolve and the
post-processing passes compute them.

CPU: the host build of the header against float64 numpy (error in float32 ulps
of the exact value): sin / cos <= 2 for |x| < 1e5, atan <= 2.5, exp <= 1
(subnormal results within one unit of 2^-149), pow <= 4.5 on the exponents the
passes use, and the special values.
GPU: the device evaluation equals the host build bit for bit (NaN payloads
aside: the host and the device write different default NaNs).
"""
import numpy as np
import pytest

import pyoracle as po


def _ulps(got, exact):
    """|got - exact| in units of the float32 spacing at the exact value."""
    sp = np.spacing(np.abs(exact.astype(np.float32))).astype(np.float64)
    return np.abs(got.astype(np.float64) - exact) / sp


def _inputs():
    rng = np.random.default_rng(0)
    trig = np.concatenate([rng.uniform(-7, 7, 400000), rng.uniform(-1e4, 1e4, 100000),
                           rng.uniform(-1e-3, 1e-3, 20000), np.linspace(0, 2 * np.pi, 4097)]).astype(np.float32)
    at = np.concatenate([rng.uniform(-3, 3, 200000),
                         np.exp(rng.uniform(-20, 20, 200000)) * rng.choice([-1, 1], 200000)]).astype(np.float32)
    ex = rng.uniform(-103, 88, 400000).astype(np.float32)
    pw = np.concatenate([rng.uniform(0, 2, 200000), np.exp(rng.uniform(-30, 30, 200000))]).astype(np.float32)
    return trig, at, ex, pw


def test_sin_cos_atan_accuracy():
    trig, at, _, _ = _inputs()
    x64 = trig.astype(np.float64)
    assert _ulps(po.glsl_eval("sin", trig), np.sin(x64)).max() <= 2.0
    assert _ulps(po.glsl_eval("cos", trig), np.cos(x64)).max() <= 2.0
    assert _ulps(po.glsl_eval("atan", at), np.arctan(at.astype(np.float64))).max() <= 2.5


def test_exp_pow_accuracy():
    _, _, ex, pw = _inputs()
    exact = np.exp(ex.astype(np.float64))
    got = po.glsl_eval("exp", ex)
    normal = exact > 2.0 ** -126
    assert _ulps(got[normal], exact[normal]).max() <= 1.0
    assert (np.abs(got[~normal] - exact[~normal]) / 2.0 ** -149).max() <= 1.0
    for y in (5.0, 2.2, 1.3, 0.5, -1.7):
        exact = np.power(pw.astype(np.float64), np.float64(np.float32(y)))
        ok = (exact > 2.0 ** -126) & (exact < 3e38)
        assert _ulps(po.glsl_eval("pow", pw, y)[ok], exact[ok]).max() <= 4.5, y


def test_special_values():
    nan, inf = np.nan, np.inf
    s = po.glsl_eval("sin", [0.0, -0.0, inf, nan])
    assert s[0] == 0 and np.signbit(s[1]) and np.isnan(s[2:]).all()
    a = po.glsl_eval("atan", [0.0, -0.0, inf, -inf, 1.0, -1.0])
    assert a[0] == 0 and np.signbit(a[1])
    assert a[2] == np.float32(np.pi / 2) and a[3] == -np.float32(np.pi / 2)
    assert a[4] == np.float32(np.pi / 4) and a[5] == -np.float32(np.pi / 4)
    p = po.glsl_eval("pow", [0.0, 1.0, 0.5, 2.0, inf, 0.0, -1.0, 7.0], [5, 3, 0, 10, 2, -1, 2, nan])
    assert list(p[:6]) == [0.0, 1.0, 1.0, 1024.0, inf, inf] and np.isnan(p[6:]).all()
    e = po.glsl_eval("exp", [0.0, -200.0, 200.0, nan])
    assert e[0] == 1.0 and e[1] == 0.0 and e[2] == inf and np.isnan(e[3])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["sin", "cos", "atan", "exp", "pow"])
def test_device_equals_host(ctx, name):
    trig, at, ex, pw = _inputs()
    specials = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1e-30, -1e-30, 1e30, 2.0 ** -140], np.float32)
    if name in ("sin", "cos"):
        x = np.concatenate([trig, specials])
    elif name == "atan":
        x = np.concatenate([at, specials])
    elif name == "exp":
        x = np.concatenate([ex, specials])
    else:
        x = np.concatenate([pw, pw, pw, np.abs(specials)])
    y = None
    if name == "pow":
        n = pw.size
        y = np.concatenate([np.full(n, 5.0), np.full(n, 2.2), np.full(n, 1.3), np.full(specials.size, 0.5)])
        y = y.astype(np.float32)
    got = ctx.glsl_builtin(name, x, y)
    ref = po.glsl_eval(name, x, y)
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    ok = ~np.isnan(ref)
    assert np.array_equal(got[ok].view(np.uint32), ref[ok].view(np.uint32))
