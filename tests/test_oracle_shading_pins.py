"""The restated shading functions (oracle_render.cpp) against known answers from
the reference's own GLSL compiled as C++ (tests/golden/glsl_kat.npz)."""
import ctypes as C

import numpy as np

import pyoracle as po


def test_wang_hash(golden):
    k = golden("glsl_kat.npz")
    a, out = k["wang_in"], k["wang_out"]
    assert all(po.oracle().orc_wang_hash(int(x)) == int(y) for x, y in zip(a, out))


def test_random_stream(golden):
    k = golden("glsl_kat.npz")
    tex, px, seeds, streams, states = k["tex"], k["rs_px"], k["rs_seed"], k["rs_stream"], k["rs_state"]
    for i in range(px.shape[0]):
        out = np.zeros(32, np.float32)
        st = C.c_uint32()
        po.oracle().orc_random_stream(tex.ctypes.data, 1024, int(px[i, 0]), int(px[i, 1]), int(seeds[i]), 32,
                                      out.ctypes.data, C.byref(st))
        assert st.value == states[i]
        assert np.array_equal(out, streams[i])


def test_transform_pack_sphere(golden):
    k = golden("glsl_kat.npz")
    v, n, ref = k["tlw_v"], k["tlw_n"], k["tlw_out"]
    for i in range(v.shape[0]):
        out = np.zeros(3, np.float32)
        vi, ni = np.ascontiguousarray(v[i]), np.ascontiguousarray(n[i])
        po.oracle().orc_transform_local_to_world(vi.ctypes.data, ni.ctypes.data, out.ctypes.data)
        assert np.array_equal(out, ref[i])
    cin, cout = k["pack_in"], k["pack_out"]
    for i in range(cin.shape[0]):
        ci = np.ascontiguousarray(cin[i])
        assert po.oracle().orc_pack_unorm4x8(ci.ctypes.data) == cout[i]
    so, sd, sc, sr, st = k["sph_o"], k["sph_d"], k["sph_c"], k["sph_r"], k["sph_t"]
    for i in range(so.shape[0]):
        a, b, c = (np.ascontiguousarray(x[i]) for x in (so, sd, sc))
        t = po.oracle().orc_intersect_sphere(a.ctypes.data, b.ctypes.data, c.ctypes.data, float(sr[i]))
        assert np.float32(t) == st[i] or (np.isnan(t) and np.isnan(st[i]))


def test_material_bounce_and_eval(golden):
    k = golden("glsl_kat.npz")
    mats, tv, nrm, rng_in, rng_out = k["mat"], k["mat_tv"], k["mat_n"], k["mat_rng_in"], k["mat_rng_out"]
    gen, refl, pdf, lobe, resample = k["mat_gen"], k["mat_refl"], k["mat_pdf"], k["mat_lobe"], k["mat_resample"]
    ltd, nee_refl, nee_pdf = k["mat_ltd"], k["mat_nee_refl"], k["mat_nee_pdf"]
    for i in range(mats.shape[0]):
        io = np.ascontiguousarray(rng_in[i]).copy()
        g = np.zeros(3, np.float32)
        rf = np.zeros(3, np.float32)
        pd, lb, rs = C.c_float(), C.c_int(), C.c_float()
        m, t, nn = (np.ascontiguousarray(x[i]) for x in (mats, tv, nrm))
        po.oracle().orc_material_bounce_eval(m.ctypes.data, io.ctypes.data, t.ctypes.data, nn.ctypes.data,
                                             g.ctypes.data, rf.ctypes.data, C.byref(pd), C.byref(lb), C.byref(rs))
        assert np.array_equal(io, rng_out[i])
        assert lb.value == lobe[i]
        np.testing.assert_array_equal(g, gen[i])
        np.testing.assert_array_equal(rf, refl[i])
        assert np.float32(pd.value) == pdf[i] or (np.isnan(pd.value) and np.isnan(pdf[i]))
        assert np.float32(rs.value) == resample[i]
        l = np.ascontiguousarray(ltd[i])
        rf2 = np.zeros(3, np.float32)
        pd2 = C.c_float()
        po.oracle().orc_material_eval(m.ctypes.data, int(lb.value), float(rs.value), l.ctypes.data, t.ctypes.data,
                                      nn.ctypes.data, rf2.ctypes.data, C.byref(pd2))
        np.testing.assert_array_equal(rf2, nee_refl[i])
        assert np.float32(pd2.value) == nee_pdf[i] or (np.isnan(pd2.value) and np.isnan(nee_pdf[i]))
