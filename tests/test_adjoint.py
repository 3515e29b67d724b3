"""The adjoint (gradient of sum(G * film) over the field parameters) against common-random-number
finite differences of the forward render.

The adjoint is the pathwise derivative: per photon, random numbers and discrete events are held
fixed. Two finite-difference checks isolate exactly that quantity:

* direct light only (albedo 0): every photon marches source -> sensor face -> film with no
  discrete event that depends on the field, so the CRN difference of two renders is the pathwise
  derivative itself;
* full scattering: photon records at theta +- h; photons whose discrete event sequence (end code,
  uniforms drawn, depth, splat count and depths) is the same in both runs are differenced photon
  by photon ("matched paths"). Photons whose sequence changes -- an escape instead of a scatter, a
  Fresnel reflection instead of a transmission -- carry the boundary term that a pathwise
  derivative does not contain; they are a fraction O(h) of the photons.

Tolerances are set by the finite differences' own noise (FP32 marches: the rounding of each
photon's path changes with the parameters), measured at these photon counts and steps.
"""
import numpy as np
import pytest

import simpler_b200 as sb
from simpler_b200 import _lib as L


def smooth_weights(s):
    z, y, x = s.film_shape()
    X, Y = np.meshgrid(np.arange(x) / x, np.arange(y) / y)
    g = 1.0 + 0.5 * np.sin(2 * np.pi * 3 * X) * np.cos(2 * np.pi * 2 * Y)
    return np.broadcast_to(g, (z, y, x)).copy()


def camera(s):
    sc = s.scene_desc()
    d = np.array(sc.view_dir[:]); h = np.array(sc.view_horizontal[:])
    d /= np.linalg.norm(d); h /= np.linalg.norm(h)
    return np.array(sc.view_origin[:]), h, np.cross(d, h), np.array(sc.view_plane[:])


def photon_objective(s, rec, G):
    """Per-photon sum(G * film contribution) from its splat records (addEnergyToImage's bilinear
    split, scene.cpp:782-829)."""
    o, h, v, plane = camera(s)
    Z, Y, X = G.shape
    J = np.zeros(len(rec))
    lo, hi = s.path_length_min, s.path_length_max
    for k in range(rec["splats"].shape[1]):
        idx = np.nonzero(k < rec["n_splats"])[0]
        sp = rec["splats"][idx, k]
        p = sp["p"].astype(np.float64)
        pl = sp["pathlength"]
        ok = (pl > lo) & (pl < hi)
        idx, p, pl, val = idx[ok], p[ok], pl[ok], sp["value"][ok]
        x = ((p @ h - o[1]) / plane[0] + 0.5) * X
        y = ((p @ v - o[2]) / plane[1] + 0.5) * Y
        iz = np.floor((pl - lo) / (hi - lo) * Z).astype(np.int64)
        ix = np.floor(x).astype(np.int64); iy = np.floor(y).astype(np.int64)
        fx, fy = x - ix, y - iy

        def g(a, b):
            inb = (a >= 0) & (a < X) & (b >= 0) & (b < Y) & (iz >= 0) & (iz < Z)
            out = np.zeros(len(a))
            out[inb] = G[iz[inb], b[inb], a[inb]]
            return out

        w = ((1 - fx) * (1 - fy) * g(ix, iy) + fx * (1 - fy) * g(ix + 1, iy) + (1 - fx) * fy * g(ix, iy + 1)
             + fx * fy * g(ix + 1, iy + 1))
        np.add.at(J, idx, val * w)
    return J


def signature_match(a, b):
    same = (a["end"] == b["end"]) & (a["draws"] == b["draws"]) & (a["depth"] == b["depth"]) & (a["n_splats"] == b["n_splats"])
    for k in range(a["splats"].shape[1]):
        same &= (a["splats"][:, k]["depth"] == b["splats"][:, k]["depth"]) | (k >= a["n_splats"])
    return same


def matched_fd(s, sp, sm, n, G):
    """sum over matched photons of J(theta + h) - J(theta - h)."""
    rp = sb.records_to_arrays(sb.trace_photons(sp, 0, n, n, with_image=False)[0])
    rm = sb.records_to_arrays(sb.trace_photons(sm, 0, n, n, with_image=False)[0])
    same = signature_match(rp, rm)
    Jp, Jm = photon_objective(s, rp, G), photon_objective(s, rm, G)
    return float((Jp[same] - Jm[same]).sum()), float(same.mean())


def stepped(theta, i, h):
    tp, tm = theta.copy(), theta.copy()
    tp[i] += h
    tm[i] -= h
    return tp, tm, float(np.float32(tp[i]) - np.float32(tm[i]))


# ---- CPU -----------------------------------------------------------------------------------------
def test_param_layout():
    pw = sb.config_planewave()
    assert sb.param_count(pw) == 2 * len(pw.wave_amp)
    th = sb.field_params(pw)
    np.testing.assert_array_equal(th, list(pw.wave_amp) + list(pw.wave_phase))
    pw2 = sb.with_field_params(pw, th * 2.0)
    assert pw2.wave_amp == tuple(2.0 * a for a in pw.wave_amp)
    sp = sb.config_spline(n=8)
    assert sb.param_count(sp) == 8 ** 3
    c = sb.field_params(sp)
    np.testing.assert_array_equal(sb.with_field_params(sp, c).grid_coeff, sp.grid_coeff)
    assert sb.param_count(sb.config_plain_small()) == 3   # Bessel: n_max, phi_min, phi_max
    with pytest.raises(L.SmpError):
        sb.param_count(sb.config_plain_small(mode=3))    # orders above 2: no adjoint built
    with pytest.raises(L.SmpError):
        sb.param_count(sb.config_sources())
    g = sb.roi_weights(pw, 32)
    assert g.shape == pw.film_shape() and g.sum() == 32 * 32 * pw.path_length_bins


def test_fp64_reference_gradient_is_stable():
    """The FP64 reference gradient (central differences of the FP64 restatement on the same photons)
    does not depend on its step: direct light, plane-wave amplitude and phase."""
    import oracle_bridge as ob
    s = sb.config_planewave(albedo=0.0, precision_mode=L.PREC_MIXED, spatial_x=64, spatial_y=64, path_length_bins=8)
    G = smooth_weights(s)
    a1, a2 = (ob.oracle_fd_gradient(s, 0, h, 400, G) for h in (1e-6, 2e-6))
    assert abs(a1) > 1e-3 * _direct_light_scale(s, G), a1        # a real signal, not 0 == 0
    assert abs(a1 - a2) <= 1e-4 * abs(a1), (a1, a2)
    p1, p2 = (ob.oracle_fd_gradient(s, 2, h, 400, G) for h in (2e-4, 4e-4))
    assert abs(p1) > 1e-6 * _direct_light_scale(s, G), p1
    assert abs(p1 - p2) <= 1e-2 * abs(p1), (p1, p2)


def _direct_light_scale(s, G):
    """sum(G * film) of the direct light (photons 0..399, FP64 oracle): the objective's own size, to
    which a gradient is compared when it must be clearly nonzero."""
    import oracle_bridge as ob
    _, img = ob.oracle_trace(s, 0, 400, 400, records=False, real_bits=64)
    return float((img * G).sum())


def test_adjoint_stats_layout():
    assert sb.check_layout()["smp_adjoint_stats"][0] == 112


# ---- GPU -----------------------------------------------------------------------------------------
@pytest.mark.gpu
def test_planewave_direct_light_fd():
    s = sb.config_planewave(albedo=0.0, precision_mode=L.PREC_MIXED)      # FP64 film (see the Bessel test)
    G = smooth_weights(s)
    n = 200_000
    grad, st = sb.adjoint(s, n, G)
    assert st.photons == n and st.replay_mismatch == 0 and st.dropped == 0 and st.aborted == 0
    _, fst = sb.render(s, n)
    assert st.er_steps_forward == fst.er_steps            # phase A traces the render's own photons
    th = sb.field_params(s)
    for i, h, tol in [(0, 3e-5, 1e-3), (2, 3e-2, 1e-3)]:   # amplitude and phase of wave 0
        tp, tm, dh = stepped(th, i, h)
        fp, _ = sb.render(sb.with_field_params(s, tp), n)
        fm, _ = sb.render(sb.with_field_params(s, tm), n)
        fd = float(((fp - fm) * G).sum()) / dh
        assert abs(grad[i] - fd) <= tol * abs(fd), (i, grad[i], fd)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["planewave", "bessel1"])
def test_adjoint_against_fp64_reference_gradient(case):
    """smp_plan_adjoint (FP32 march, pathwise derivative) against the FP64 reference gradient:
    central differences of the FP64 restatement on the same Philox photons (direct light, so no
    discrete event depends on the field), to 1e-3 relative."""
    import oracle_bridge as ob
    if case == "planewave":
        s = sb.config_planewave(albedo=0.0, precision_mode=L.PREC_MIXED, spatial_x=64, spatial_y=64,
                                path_length_bins=8)
        params = [(0, 1e-6), (1, 1e-6), (2, 2e-4), (3, 2e-4)]
        G = smooth_weights(s)
    else:
        # mode 1 deflects the beam along z (film rows): a row ramp measures the deflection. (A
        # smooth symmetric weighting cancels the two sides of the axis to 1e-8 of the objective,
        # below the march's own discrete refinement, and no finite difference resolves it.)
        s = sb.config_plain_small(albedo=0.0, mode=1, n_max=2e-3, n_clip=4e-3, phi_min=0.3, phi_max=1.5,
                                  precision_mode=L.PREC_MIXED, spatial_x=64, spatial_y=64, path_length_bins=8)
        params = [(0, 1e-6), (1, 3e-4), (2, 3e-4)]
        z, y, x = s.film_shape()
        G = np.broadcast_to((np.arange(y) - y / 2)[None, :, None] / y, (z, y, x)).copy()
    n = 4000
    plan = sb.Plan(s)
    grad, st = plan.adjoint(G, 0, n, n)
    plan.close()
    assert st.photons == n and st.dropped == 0 and st.replay_mismatch == 0
    ref = np.array([ob.oracle_fd_gradient(s, i, h, n, G) for i, h in params])
    got = np.array([grad[i] for i, _ in params])
    for (i, _), a, r in zip(params, got, ref):
        print(f"{case} parameter {i}: adjoint {a:.8e}, FP64 reference {r:.8e}, relative {abs(a - r) / abs(r):.2e}")
    # 1e-3 relative per group of parameters of one kind (amplitudes, phases): a component much
    # smaller than its group's largest carries the group's absolute FP32 error
    groups = [[0, 1], [2, 3]] if case == "planewave" else [[0], [1, 2]]
    for grp in groups:
        err = np.linalg.norm(got[grp] - ref[grp]) / np.linalg.norm(ref[grp])
        print(f"{case} parameters {grp}: relative error {err:.2e}")
        assert err <= 1e-3, (grp, got[grp], ref[grp])


@pytest.mark.gpu
def test_planewave_scattering_matched_fd():
    s = sb.config_planewave(max_depth=7)                 # <= 8 splats per photon: all in the records
    G = sb.roi_weights(s, 32)
    n = 300_000
    grad, st = sb.adjoint(s, n, G)
    assert st.replay_mismatch == 0 and st.dropped == 0
    th = sb.field_params(s)
    for i, h, tol in [(0, 3e-5, 0.08), (1, 3e-5, 0.03), (2, 3e-2, 0.02)]:
        tp, tm, dh = stepped(th, i, h)
        fd, frac = matched_fd(s, sb.with_field_params(s, tp), sb.with_field_params(s, tm), n, G)
        assert frac > 0.99
        fd /= dh
        assert abs(grad[i] - fd) <= tol * abs(fd), (i, grad[i], fd)


@pytest.mark.gpu
def test_planewave_wave_counts_agree():
    """The sweep runs a two-wave instance for fields of at most two waves and an eight-wave one
    otherwise: a third wave of amplitude 0 leaves every photon as it is, so the eight-wave
    gradient of the first two waves equals the two-wave gradient (up to the order of the float
    sums), and the third wave's amplitude derivative is that of a field it does not yet change."""
    s2 = sb.config_planewave(max_depth=7)
    k = 2.0 * np.pi * 1e6 / 1500.0
    s3 = sb.config_planewave(max_depth=7, wave_amp=s2.wave_amp + (0.0,), wave_k=s2.wave_k + ((k, 0.0, 0.0),),
                             wave_phase=s2.wave_phase + (0.5,))
    G = sb.roi_weights(s2, 32)
    n = 200_000
    g2, st2 = sb.adjoint(s2, n, G)
    g3, st3 = sb.adjoint(s3, n, G)
    assert st2.replay_mismatch == 0 and st3.replay_mismatch == 0 and st2.dropped == 0 and st3.dropped == 0
    assert st2.points == st3.points and st2.splats == st3.splats
    first = [0, 1, 3, 4]                             # a_0, a_1, phase_0, phase_1 of the three-wave layout
    np.testing.assert_allclose(g3[first], g2, rtol=1e-4, atol=1e-6 * np.abs(g2).max())
    assert abs(g3[2]) > 1e-3 * np.abs(g2[:2]).max()  # d/da_2 at a_2 = 0
    assert g3[5] == 0.0                              # d/dphase_2 carries a factor a_2 = 0


@pytest.mark.gpu
def test_bessel_direct_light_fd():
    """Bessel mode 1 at a fixed phase (s = sin 1 for every photon; n_clip = 2 n_max, so no photon is
    clamped on either side of the step): amplitude, and the phase window moved as a whole. (Mode 0
    is a poor finite-difference case: its radially symmetric focusing gives photons on opposite
    sides of the axis contributions of opposite sign that cancel to about 1 % of their size.)"""
    # FP64 film: direct light lands in a single path-length bin, where FP32 film atomics (thousands
    # per pixel, in no fixed order) would round away the difference being measured
    s = sb.config_plain_small(albedo=0.0, mode=1, n_max=2e-3, n_clip=4e-3, phi_min=1.0, phi_max=1.0,
                              precision_mode=L.PREC_MIXED)
    G = smooth_weights(s)
    n = 1_000_000
    grad, st = sb.adjoint(s, n, G)
    assert st.replay_mismatch == 0 and st.dropped == 0
    th = sb.field_params(s)
    # amplitude (a 5 % step: smaller ones are dominated by the march's FP32 rounding at this signal)
    tp, tm, dh = stepped(th, 0, 1e-4)
    fd = float(((sb.render(sb.with_field_params(s, tp), n)[0] - sb.render(sb.with_field_params(s, tm), n)[0]) * G).sum()) / dh
    assert abs(grad[0] - fd) <= 2e-2 * abs(fd), (grad[0], fd)
    # the phase window shifted as a whole: d/dphi_min + d/dphi_max
    tp, tm = th.copy(), th.copy()
    tp[1:] += 0.05
    tm[1:] -= 0.05
    fd = float(((sb.render(sb.with_field_params(s, tp), n)[0] - sb.render(sb.with_field_params(s, tm), n)[0]) * G).sum()) / 0.1
    assert abs(grad[1] + grad[2] - fd) <= 3e-2 * abs(fd), (grad[1] + grad[2], fd)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
def test_bessel_scattering_matched_fd(mode):
    s = sb.config_plain_small(mode=mode, n_max=2e-3, n_clip=4e-3, max_depth=7)
    G = sb.roi_weights(s, 32)
    n = 300_000
    grad, st = sb.adjoint(s, n, G)
    assert st.replay_mismatch == 0 and st.dropped == 0
    tp, tm, dh = stepped(sb.field_params(s), 0, 2e-5)
    fd, frac = matched_fd(s, sb.with_field_params(s, tp), sb.with_field_params(s, tm), n, G)
    assert frac > 0.99
    fd /= dh
    assert abs(grad[0] - fd) <= 3e-2 * abs(fd), (grad[0], fd)


@pytest.mark.gpu
def test_spline_direction_fd():
    """All 262144 coefficients at once: the gradient dotted with a random perturbation."""
    n = 100_000
    s = sb.config_spline(albedo=0.0, precision_mode=L.PREC_MIXED)
    G = smooth_weights(s)
    grad, st = sb.adjoint(s, n, G)
    assert st.replay_mismatch == 0 and st.dropped == 0
    th = sb.field_params(s)
    u = np.random.default_rng(1).standard_normal(th.shape) * 1e-3
    cp, cm = (th + 0.03 * u).astype(np.float32), (th - 0.03 * u).astype(np.float32)
    pred = float(grad @ (cp.astype(np.float64) - cm.astype(np.float64)))
    fp, _ = sb.render(sb.with_field_params(s, cp), n)
    fm, _ = sb.render(sb.with_field_params(s, cm), n)
    fd = float(((fp - fm) * G).sum())
    assert abs(pred - fd) <= 1e-2 * abs(fd), (pred, fd)

    s = sb.config_spline(max_depth=7)
    G = sb.roi_weights(s, 32)
    n = 50_000
    grad, st = sb.adjoint(s, n, G)
    assert st.replay_mismatch == 0
    rng = np.random.default_rng(1)
    rng.standard_normal(th.shape)
    u = rng.standard_normal(th.shape) * 1e-3
    cp, cm = (th + 0.03 * u).astype(np.float32), (th - 0.03 * u).astype(np.float32)
    pred = float(grad @ (cp.astype(np.float64) - cm.astype(np.float64)))
    fd, frac = matched_fd(s, sb.with_field_params(s, cp), sb.with_field_params(s, cm), n, G)
    assert frac > 0.99
    assert abs(pred - fd) <= 3e-2 * abs(fd), (pred, fd)


@pytest.mark.gpu
def test_plan_adjoint_and_autograd():
    import torch
    from simpler_b200.pybind.autograd import render_torch
    s = sb.config_planewave()
    n = 50_000
    G = sb.roi_weights(s, 32)
    g1, _ = sb.adjoint(s, n, G)
    p = sb.Plan(s)
    try:
        g2, _ = p.adjoint(G, 0, n, n)
        # two halves of the photon range add up to the whole
        ga, _ = p.adjoint(G, 0, n // 2, n)
        gb, _ = p.adjoint(G, n // 2, n - n // 2, n)
    finally:
        p.close()
    np.testing.assert_allclose(g2, g1, rtol=1e-6)
    np.testing.assert_allclose(ga + gb, g1, rtol=1e-6)
    theta = torch.tensor(sb.field_params(s), requires_grad=True)
    film = render_torch(theta, s, n)
    assert film.is_cuda                                                              # no host round trip
    ref, _ = sb.render(s, n)
    np.testing.assert_allclose(film.detach().cpu().numpy(), ref, rtol=1e-5, atol=1e-12)   # FP32 film atomics
    (film * torch.from_numpy(G).to(film.device)).sum().backward()
    np.testing.assert_allclose(theta.grad.numpy(), g1, rtol=1e-6)
