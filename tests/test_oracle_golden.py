"""CPU: the oracle pinned to the reference.

* against golden fixtures taken from the reference (tests/golden, made by tests/golden/make_golden.py):
  the spline test vectors of splinepractice/*.csv, draws of the reference's SFMT engine, and outputs
  of its compiled primitives;
* against the reference's compiled primitives directly when oracle/_ref is present (this container).
"""
import ctypes as C
import hashlib
import json
import math
import os

import numpy as np
import pytest

import oracle_bridge as ob
import simpler_b200 as sb

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gold(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


def fp(a):
    return C.c_void_p(a.ctypes.data)


def _olib():
    lib = ob.oracle()
    f = C.c_float
    vp = C.c_void_p
    lib.orc_hg_sample.argtypes = [f, vp, C.c_uint64, C.c_int, vp]
    lib.orc_hg_f.argtypes = [f, vp, vp]
    lib.orc_hg_f.restype = f
    lib.orc_hemisphere.argtypes = [f, f, vp]
    lib.orc_fresnel.argtypes = [f, f, f]
    lib.orc_fresnel.restype = f
    lib.orc_refract.argtypes = [vp, vp, f, vp]
    lib.orc_coordinate_system.argtypes = [vp, vp, vp]
    lib.orc_bsdf_sample.argtypes = [f, f, vp, vp, C.c_uint64, C.c_int, vp]
    lib.orc_lens_propagate.argtypes = [vp, f, f, C.c_int, vp, vp, vp]
    return lib


# ---- SFMT ------------------------------------------------------------------------------------------
def test_sfmt_matches_reference_engine_fixture():
    lib = ob.oracle()
    for seed, draws in gold("sfmt.json")["draws"].items():
        a = np.zeros(len(draws), np.float32)
        lib.orc_sfmt_floats(C.c_uint64(int(seed)), len(draws), fp(a))
        assert np.array_equal(a, np.array(draws, np.float32)), seed


@pytest.mark.skipif(ob.ref_prims() is None, reason="reference primitives not built here")
def test_sfmt_matches_reference_engine_live():
    lib, ref = ob.oracle(), ob.ref_prims()
    rng = np.random.default_rng(0)
    for seed in rng.integers(0, 2 ** 62, size=12):
        a = np.zeros(2500, np.float32)
        b = np.zeros(2500, np.float32)
        lib.orc_sfmt_floats(C.c_uint64(int(seed)), 2500, fp(a))
        ref.ref_sfmt_float(C.c_uint64(int(seed)), 2500, fp(b))
        assert np.array_equal(a, b), seed


def test_philox_known_answer():
    # Philox-4x32-10, key (0, 0), counter (0, 0, 0, 0) -> 0x6627e8d5 0xe169c58d 0xbc57ac4c 0x9b00dbd8
    # (the Random123 known-answer vector); the first draw is its first word >> 8 / 2^24
    lib = ob.oracle()
    a = np.zeros(4, np.float32)
    lib.orc_philox_floats(C.c_uint64(0), C.c_uint64(0), 4, fp(a))
    words = [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert np.array_equal(a, np.array([(w >> 8) / 16777216.0 for w in words], np.float32))


# ---- primitives --------------------------------------------------------------------------------------
def _close(a, b, tol=2e-5):
    # the reference primitives are built with -ffast-math (FMA contraction); sin(theta) from
    # sqrt(1 - cos^2) amplifies a 1-ulp difference in cos(theta) near the poles
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.all(np.abs(a - b) <= tol * np.maximum(1.0, np.abs(b)))


def test_primitives_match_reference_fixture():
    lib = _olib()
    g = gold("primitives.json")
    for gg, d, seed, skip, out, _c in g["hg"]:
        d = np.array(d, np.float32)
        o = np.zeros(3, np.float32)
        lib.orc_hg_sample(gg, fp(d), C.c_uint64(seed), skip, fp(o))
        assert _close(o, out), (gg, seed)
    for gg, d, o2, val in g["hg_f"]:
        d, o2 = np.array(d, np.float32), np.array(o2, np.float32)
        assert _close(lib.orc_hg_f(gg, fp(d), fp(o2)), val, 1e-5)
    for u0, u1, h in g["hemisphere"]:
        o = np.zeros(3, np.float32)
        lib.orc_hemisphere(u0, u1, fp(o))
        assert _close(o, h)
    for ci, ct, eta, val in g["fresnel"]:
        # random cosines include near-zero denominators (values up to 1e5): relative tolerance
        assert abs(lib.orc_fresnel(ci, ct, eta) - val) <= 1e-4 * max(1.0, abs(val))
    for a, n, eta, ok, b in g["refract"]:
        a, n = np.array(a, np.float32), np.array(n, np.float32)
        o = np.zeros(3, np.float32)
        assert lib.orc_refract(fp(a), fp(n), eta, fp(o)) == ok
        assert _close(o, b)
    for d, bb, cc in g["coord"]:
        d = np.array(d, np.float32)
        ob1, oc = np.zeros(3, np.float32), np.zeros(3, np.float32)
        lib.orc_coordinate_system(fp(d), fp(ob1), fp(oc))
        assert _close(ob1, bb) and _close(oc, cc)
    for a, n, seed, skip, out in g["bsdf"]:
        a, n = np.array(a, np.float32), np.array(n, np.float32)
        o = np.zeros(3, np.float32)
        lib.orc_bsdf_sample(1.0, 1.3333, fp(a), fp(n), C.c_uint64(seed), skip, fp(o))
        assert _close(o, out), (seed, skip)
    pm = g["pmf"]
    cdf = np.zeros(len(pm["pdf"]) + 1, np.float32)
    idx = np.zeros(len(pm["u"]), np.int32)
    pdf = np.array(pm["pdf"], np.float64)
    u = np.array(pm["u"], np.float32)
    ob.oracle().orc_texture_cdf(fp(pdf), len(pdf), fp(cdf), len(u), fp(u), fp(idx))
    assert np.array_equal(cdf, np.array(pm["cdf"], np.float32))
    assert idx.tolist() == pm["idx"]
    for pos, dirv, act, ok, p2, d2, tot in g["lens"]:
        origin = np.array([0.005, 0.0, 0.0], np.float32)
        p, d = np.array(pos, np.float32), np.array(dirv, np.float32)
        t = np.zeros(1, np.float32)
        assert lib.orc_lens_propagate(fp(origin), 0.0015, 0.015, act, fp(p), fp(d), fp(t)) == ok
        assert _close(p, p2) and _close(d, d2) and _close(t, [tot])


@pytest.mark.skipif(ob.ref_prims() is None, reason="reference primitives not built here")
def test_hg_and_bsdf_match_reference_live():
    lib, ref = _olib(), ob.ref_prims()
    rng = np.random.default_rng(5)
    for k in range(500):
        d = rng.standard_normal(3).astype(np.float32)
        d /= np.linalg.norm(d)
        a, b = np.zeros(3, np.float32), np.zeros(3, np.float32)
        lib.orc_hg_sample(0.85, fp(d), C.c_uint64(k), k % 7, fp(a))
        ref.ref_hg_sample(0.85, fp(d), C.c_uint64(k), k % 7, fp(b))
        assert _close(a, b)
        n = np.zeros(3, np.float32)
        n[k % 3] = -1.0 if k % 2 else 1.0
        v = (rng.standard_normal(3) * 1.3).astype(np.float32)
        lib.orc_bsdf_sample(1.0, 1.3333, fp(v), fp(n), C.c_uint64(k), k % 3, fp(a))
        ref.ref_bsdf_sample(1.0, 1.3333, fp(v), fp(n), C.c_uint64(k), k % 3, fp(b))
        assert _close(a, b)


# ---- splines (splinepractice golden vectors) ---------------------------------------------------------
def test_spline_1d_golden():
    g = gold("spline1d.json")
    lib = ob.oracle()
    data = np.array(g["data"], np.float64)
    t = np.array(g["t"], np.float64)
    xmin, xmax = math.sqrt(g["xmin_sq"]), math.sqrt(g["xmax_sq"])
    for deriv, key in [(0, "value"), (1, "d1"), (2, "d2")]:
        out = np.zeros(len(t))
        lib.orc_spline1d(fp(data), len(data), xmin, xmax, deriv, len(t), fp(t), fp(out))
        ref = np.array(g[key])
        # the CSV holds 6 significant digits
        assert np.all(np.abs(out - ref) <= 2e-5 * np.maximum(1.0, np.abs(ref))), (key, np.abs(out - ref).max())


def test_spline_kernels_golden():
    g = gold("kernel.json")
    lib = ob.oracle()
    lib.orc_bspline_kernel.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    x = np.array(g["x"], np.float64)
    for d, key in [(0, "k0"), (1, "k1"), (2, "k2")]:
        out = np.zeros(len(x))
        lib.orc_bspline_kernel(d, len(x), fp(x), fp(out))
        ref = np.array(g[key])
        # kernel.csv holds 6 significant digits
        assert np.all(np.abs(out - ref) <= 1e-5 * np.maximum(np.abs(ref), 1e-3)), (key, np.abs(out - ref).max())


def test_spline_3d_golden():
    g = gold("spline3d.json")
    lib = ob.oracle()
    data = np.array(g["data"], np.float64)
    coeff = np.zeros(1000)
    dims = np.array([10, 10, 10], np.int32)
    lib.orc_spline_prefilter3d(fp(data), fp(dims), 64, fp(coeff))
    # coefficients3d.csv row (k, i) holds coeff[i + 10 j + 100 k] for j = 0..9
    rows = np.array(g["coeff_rows"]).reshape(10, 10, 10)       # [k, i, j]
    ours = coeff.reshape(10, 10, 10)                            # [k, j, i]
    assert np.allclose(ours.transpose(0, 2, 1), rows, rtol=1e-9, atol=1e-9)
    pts = np.array(g["points"])
    vals = np.array(g["values"])
    xmin = np.array([1.0, 1.0, 1.0])
    xmax = np.array([10.0, 10.0, 10.0])
    for c, (dx, dy, dz) in enumerate(g["derivs"]):
        out = np.zeros(len(pts))
        lib.orc_spline3d_value(fp(coeff), fp(dims), fp(xmin), fp(xmax), dx, dy, dz, len(pts), fp(pts), fp(out))
        assert np.allclose(out, vals[:, c], rtol=1e-8, atol=1e-9), (c, np.abs(out - vals[:, c]).max())


def test_product_prefilter_matches_oracle():
    rng = np.random.default_rng(1)
    n = np.array([9, 7, 11], np.int32)
    s = (1.3333 + 1e-3 * rng.standard_normal((11, 7, 9))).astype(np.float32)
    got = np.zeros_like(s)
    sb._lib.check(sb.load().smp_spline_prefilter(fp(s), fp(n), fp(got)))
    ref = np.zeros(s.size)
    s64 = s.astype(np.float64)
    ob.oracle().orc_spline_prefilter3d(fp(s64), fp(n), 32, fp(ref))
    assert np.allclose(got.reshape(-1), ref, rtol=0, atol=2e-6)


def test_product_texture_cdf_matches_oracle():
    tex = sb.bernoulli_texture(64, 0.5, 1)
    got = np.zeros(tex.size + 1, np.float32)
    sb._lib.check(sb.load().smp_texture_cdf(fp(tex), 64, 64, fp(got)))
    ref = np.zeros(tex.size + 1, np.float32)
    idx = np.zeros(1, np.int32)
    u = np.zeros(1, np.float32)
    ob.oracle().orc_texture_cdf(fp(tex), tex.size, fp(ref), 1, fp(u), fp(idx))
    assert np.array_equal(got, ref)


def test_disk_texture_matches_reference_file():
    g = gold("textures.json")["Disk_501"]
    tex = sb.disk_texture()
    assert list(tex.shape) == g["shape"]
    assert hashlib.sha256(tex.astype("<f8").tobytes()).hexdigest() == g["sha256_f64_le"]
