"""Test-side bridge to the CPU oracle (oracle/liboracle.so): the checker, never the product."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from simpler_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE = os.path.join(ROOT, "oracle", "liboracle.so")
ORACLE_FAST = os.path.join(ROOT, "oracle", "liboracle_fast.so")
REF_PRIMS = os.path.join(ROOT, "oracle", "_ref", "libref_prims.so")

_libs = {}


def oracle(fast: bool = False) -> C.CDLL:
    path = ORACLE_FAST if fast else ORACLE
    if path in _libs:
        return _libs[path]
    lib = C.CDLL(path)
    P = C.POINTER
    vp = C.c_void_p
    lib.orc_render.argtypes = [P(L.SceneDesc), P(L.MediumDesc), P(L.FieldDesc), P(L.RenderOpts), C.c_int, C.c_int,
                               C.c_int64, C.c_int64, C.c_int64, vp, vp, vp, vp]
    lib.orc_sfmt_floats.argtypes = [C.c_uint64, C.c_int, vp]
    lib.orc_sfmt_u64.argtypes = [C.c_uint64, C.c_int, vp]
    lib.orc_philox_floats.argtypes = [C.c_uint64, C.c_uint64, C.c_int, vp]
    lib.orc_field_eval.argtypes = [P(L.FieldDesc), C.c_double, C.c_int, C.c_int64, vp, vp, vp]
    lib.orc_texture_cdf.argtypes = [vp, C.c_int, vp, C.c_int, vp, vp]
    lib.orc_spline_prefilter3d.argtypes = [vp, vp, C.c_int, vp]
    lib.orc_spline1d.argtypes = [vp, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, vp, vp]
    lib.orc_spline3d_value.argtypes = [vp, vp, vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp]
    _libs[path] = lib
    return lib


def ref_prims() -> C.CDLL | None:
    """The reference's own compiled primitives (oracle/_ref), when they were built."""
    if not os.path.exists(REF_PRIMS):
        return None
    if REF_PRIMS in _libs:
        return _libs[REF_PRIMS]
    lib = C.CDLL(REF_PRIMS)
    f = C.c_float
    vp = C.c_void_p
    lib.ref_sfmt_float.argtypes = [C.c_uint64, C.c_int, vp]
    lib.ref_hg_sample.argtypes = [f, vp, C.c_uint64, C.c_int, vp]
    lib.ref_hg_sample.restype = f
    lib.ref_hg_f.argtypes = [f, vp, vp]
    lib.ref_hg_f.restype = f
    lib.ref_hemisphere.argtypes = [f, f, vp]
    lib.ref_fresnel.argtypes = [f, f, f]
    lib.ref_fresnel.restype = f
    lib.ref_refract.argtypes = [vp, vp, f, vp]
    lib.ref_coordinate_system.argtypes = [vp, vp, vp]
    lib.ref_bsdf_sample.argtypes = [f, f, vp, vp, C.c_uint64, C.c_int, vp]
    lib.ref_pmf_sample.argtypes = [vp, C.c_int, C.c_int, vp, vp, vp]
    lib.ref_pmf_sample.restype = C.c_long
    lib.ref_lens_propagate.argtypes = [vp, f, f, C.c_int, vp, vp, vp]
    lib.ref_lens_deflect.argtypes = [vp, f, f, vp, vp, vp]
    _libs[REF_PRIMS] = lib
    return lib


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def oracle_trace(setup, first: int, n: int, weight_photons: int, uniforms=None, offsets=None, real_bits: int = 32,
                 threads: int = 0, records: bool = True, image: bool = True, fast: bool = False):
    """Run the CPU restatement; returns (records array or None, film (z,y,x) or None)."""
    lib = oracle(fast)
    sc, md, fd, op = setup.descs()
    recs = (L.PhotonRecord * n)() if records else None
    img = np.zeros(setup.film_shape(), dtype=np.float64) if image else None
    u = o = None
    if uniforms is not None:
        u = np.ascontiguousarray(uniforms, dtype=np.float32)
        o = np.ascontiguousarray(offsets, dtype=np.int64)
    rc = lib.orc_render(C.byref(sc), C.byref(md), C.byref(fd), C.byref(op), real_bits, threads, first, n,
                        weight_photons, _p(u), _p(o), C.cast(recs, C.c_void_p) if recs is not None else None,
                        _p(img))
    assert rc == 0, rc
    from simpler_b200.render import records_to_arrays
    return (records_to_arrays(recs) if recs is not None else None), img


def oracle_fd_gradient(setup, index: int, h: float, n: int, G: np.ndarray, threads: int = 0) -> float:
    """FP64 reference gradient: the central difference of sum(G * film) in field parameter `index`
    (simpler_b200.field_params order) with the FP64 restatement on common random numbers (the same
    Philox photons 0..n-1 on both sides). The step is the difference of the two parameter values as
    the renders receive them (with_field_params stores spline coefficients in float32, so there it
    is the float32 rounding of +-h; Bessel and plane-wave parameters stay float64)."""
    import simpler_b200 as sb
    th = sb.field_params(setup)
    tp, tm = th.copy(), th.copy()
    tp[index] += h
    tm[index] -= h
    sp, sm = sb.with_field_params(setup, tp), sb.with_field_params(setup, tm)
    dh = float(sb.field_params(sp)[index]) - float(sb.field_params(sm)[index])
    _, ip = oracle_trace(sp, 0, n, n, records=False, real_bits=64, threads=threads)
    _, im = oracle_trace(sm, 0, n, n, records=False, real_bits=64, threads=threads)
    return float(((ip - im) * G).sum()) / dh


def oracle_field(setup, scaling: float, points: np.ndarray, real_bits: int = 64):
    return oracle_field_desc(setup.field_desc(), scaling, points, real_bits)


def oracle_field_desc(fd, scaling: float, points: np.ndarray, real_bits: int = 64):
    lib = oracle()
    pts = np.ascontiguousarray(points, dtype=np.float64)
    n = np.zeros(len(pts))
    g = np.zeros((len(pts), 3))
    assert lib.orc_field_eval(C.byref(fd), scaling, real_bits, len(pts), _p(pts), _p(n), _p(g)) == 0
    return n, g


def sfmt_streams(seed_base: int, first: int, n: int, per_photon: int):
    """Per-photon SFMT uniform streams (photon i seeded with seed_base + i, as photon.cpp:313),
    packed for injection: (uniforms, offsets)."""
    lib = oracle()
    u = np.zeros((n, per_photon), dtype=np.float32)
    for k in range(n):
        lib.orc_sfmt_floats(C.c_uint64(seed_base + first + k), per_photon, C.c_void_p(u[k].ctypes.data))
    offsets = np.arange(n + 1, dtype=np.int64) * per_photon
    return u.reshape(-1), offsets
