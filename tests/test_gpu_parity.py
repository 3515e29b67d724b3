"""GPU march vs the CPU oracle, photon by photon, on the reference's own uniform streams.

Each photon i draws from SFMT-19937 seeded with i (renderer/src/photon.cpp:313); the streams are
generated by the oracle's SFMT restatement (pinned to the reference engine in test_oracle.py)
and injected into both implementations. Tolerances (the acceptance bounds of this path): positions 1e-4 mm, directions
1e-5 rad; splat values 1e-4 relative. Photons whose discrete events differ (a Fresnel coin flip
or a refinement decision within an FP32 rounding of its threshold) are counted, not hidden.
"""
import numpy as np
import pytest

import oracle_bridge as ob
import parity
import simpler_b200 as sb
from simpler_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _check(setup, n, min_ok=0.98, min_events=0.995, per_photon=256, img_tol=5e-4, real_bits=32):
    return parity.check(setup, n, min_ok=min_ok, min_events=min_events, per_photon=per_photon, img_tol=img_tol,
                        real_bits=real_bits)


def test_parity_bessel_mode0_plain_small():
    _check(sb.config_plain_small(rng=L.RNG_STREAM), 2000)


def test_parity_bessel_mode1_mixed_precision():
    s = sb.config_precision(rng=L.RNG_STREAM, spatial_x=64, spatial_y=64, path_length_bins=16)
    _check(s, 600, per_photon=1024)


def test_parity_bessel_mode2_with_gaps_and_bounces():
    s = sb.config_plain_small(rng=L.RNG_STREAM, mode=2, n_max=2e-3, n_clip=1.5e-3, phi_min=0.3, phi_max=2.0,
                              emitter_gap=0.002, sensor_gap=0.001, use_bounce_decomposition=True,
                              path_length_bins=8)
    _check(s, 1500)


def test_parity_no_direct_maxdepth():
    s = sb.config_plain_small(rng=L.RNG_STREAM, use_direct=False, max_depth=3, sigma_t=400.0, albedo=0.8)
    _check(s, 1500)


def test_parity_planewave():
    s = sb.config_planewave(rng=L.RNG_STREAM, phi_min=0.0, phi_max=6.283185307179586)
    _check(s, 1500)


def test_parity_sources():
    s = sb.config_plain_small(rng=L.RNG_STREAM, field_type=L.FIELD_SOURCES, f_u=2e6, n_scaling=2.15e-5,
                              theta_sources=6, trans_z_sources=5, radius=0.0508, chordlength=0.0127,
                              center1=(0.0, 0.0, -0.0508), center2=(0.0, -0.0508, 0.0), phase1=np.pi,
                              phase2=np.pi, er_stepsize=5e-5, sigma_t=100.0)
    _check(s, 400)


def _spline_setup(**kw):
    rng = np.random.default_rng(4)
    n = 12
    samples = 1.3333 + 1e-3 * rng.standard_normal((n, n, n)).astype(np.float32)
    coeff = np.zeros_like(samples)
    import ctypes as C
    lib = sb.load()
    dims = np.array([n, n, n], dtype=np.int32)
    assert lib.smp_spline_prefilter(C.c_void_p(samples.ctypes.data), C.c_void_p(dims.ctypes.data),
                                    C.c_void_p(coeff.ctypes.data)) == 0
    return sb.config_plain_small(rng=L.RNG_STREAM, field_type=L.FIELD_SPLINE, grid_coeff=coeff,
                                 grid_min=(-0.006, -0.006, -0.006), grid_max=(0.006, 0.006, 0.006), **kw)


def test_parity_spline():
    _check(_spline_setup(er_stepsize=2e-5), 800)


def test_parity_philox_many_photons_per_lane():
    # every lane traces many photons in turn: per-photon state must not leak between them
    s = sb.config_plain_small(rng=L.RNG_PHILOX, seed=7)
    n_gpu, n_cmp = 400_000, 3000
    g, _ = sb.trace_photons(s, 0, n_gpu, n_gpu, with_image=False)
    g = sb.records_to_arrays(g)
    assert (g["photon"] == np.arange(n_gpu)).all()
    r, _ = ob.oracle_trace(s, 0, n_cmp, n_gpu, image=False)
    parity.accept(g[:n_cmp], r)
    # the tail of the range as well
    r2, _ = ob.oracle_trace(s, n_gpu - n_cmp, n_cmp, n_gpu, image=False)
    c2 = parity.compare_records(g[n_gpu - n_cmp:], r2)
    assert c2["same_events"].mean() >= 0.995, parity.summary(c2)


def test_plan_render_film_matches_oracle_same_streams():
    # the plan path (persistent launch, Philox) against the restatement on the same streams
    s = sb.config_plain_small(rng=L.RNG_PHILOX, seed=3, spatial_x=32, spatial_y=32, path_length_bins=8)
    n = 30_000
    p = sb.Plan(s)
    img, st = p.render(n)
    p.close()
    assert st.photons == n
    _, rimg = ob.oracle_trace(s, 0, n, n, records=False)
    rel = np.abs(img - rimg).sum() / np.abs(rimg).sum()
    assert rel < 2e-3, rel
    assert abs(img.sum() / rimg.sum() - 1.0) < 1e-3


@pytest.mark.gpu
def test_fp32_march_image_against_fp64_oracle():
    """The precision form (FP32 march, FP64 path length and film) against the FP64 restatement on
    the same Philox photons: relative image RMSE within 1 %."""
    s = sb.config_plain_small(rng=L.RNG_PHILOX, seed=5, spatial_x=32, spatial_y=32, path_length_bins=8,
                              precision_mode=L.PREC_MIXED)
    n = 20_000
    img, st = sb.render(s, n)
    assert st.photons == n
    _, ref = ob.oracle_trace(s, 0, n, n, records=False, real_bits=64)
    rmse = np.sqrt(((img - ref) ** 2).sum() / (ref ** 2).sum())
    print(f"relative image RMSE against the FP64 oracle: {rmse:.3e}")
    assert rmse < 1e-2, rmse


def test_field_probe_matches_oracle():
    rng = np.random.default_rng(0)
    pts = rng.uniform(-0.005, 0.005, size=(4000, 3))
    pts[:10, 1:] = 0.0                          # on the axis
    pts[10:20, 1:] *= 1e-5                      # near the axis
    cases = [
        (sb.config_plain_small(), 0.7),
        (sb.config_plain_small(mode=1, n_max=2e-3), -0.4),
        (sb.config_plain_small(mode=2, n_max=2e-3, f_u=2e6), 1.0),
        (sb.config_planewave(), 0.3),
        (_spline_setup(), 0.0),
    ]
    for setup, s in cases:
        gn, gg = sb.field_eval(setup, s, pts)
        rn, rg = ob.oracle_field(setup, s, pts, real_bits=64)
        dn = np.abs(gn - rn)
        # a few FP32 ulps of n ~ 1.33 (64 taps are summed for the spline)
        assert dn.max() < (1e-6 if setup.field_type == L.FIELD_SPLINE else 4e-7), (setup.field_type, setup.mode, dn.max())
        scale = np.abs(rg).max()
        assert np.abs(gg - rg).max() < 2e-4 * scale + 1e-6, (setup.field_type, setup.mode, np.abs(gg - rg).max(), scale)


def test_step_cap_is_reported_and_context_survives():
    s = sb.config_plain_small(step_cap=50)
    with pytest.raises(sb.SmpError) as e:
        sb.render(s, 1000)
    assert e.value.code == L.SMP_ERR_STEP_CAP
    img, st = sb.render(sb.config_plain_small(), 2000)
    assert st.photons == 2000 and np.isfinite(img).all()


def test_stream_exhaustion_is_reported():
    s = sb.config_plain_small(rng=L.RNG_STREAM)
    n = 64
    u = np.full(n * 3, 0.5, dtype=np.float32)
    off = np.arange(n + 1, dtype=np.int64) * 3
    with pytest.raises(sb.SmpError) as e:
        sb.trace_photons(s, 0, n, n, uniforms=u, offsets=off)
    assert e.value.code == L.SMP_ERR_STREAM
