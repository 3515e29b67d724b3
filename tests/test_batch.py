"""The batched sweep (smp_render_batch): many field / medium configurations over one scene in
one slot pool. Photon j of instance i draws the stream (seed_i, j), so each instance's film is the
single render of that configuration with that seed, up to float rounding: the sweep evaluates the
Bessel field on one branch-free path for every order, which rounds differently from the
order-specific closed forms of a single render."""
import dataclasses

import numpy as np
import pytest

import simpler_b200 as sb
from simpler_b200 import _lib as L


def _instances():
    return [
        dict(mode=0, n_max=1e-3, n_clip=1e-3, f_u=848e3, n_photons=20000, seed=5),
        dict(mode=1, n_max=2e-3, n_clip=2e-3, f_u=1.5e6, phi_min=0.0, phi_max=1.0, n_photons=7000, seed=6),
        dict(mode=2, n_max=1.5e-3, n_clip=1e-3, f_u=0.6e6, sigma_t=200.0, albedo=0.8, g=0.7,
             n_photons=13000, seed=7),
        dict(mode=1, n_max=1e-3, n_clip=1e-3, f_u=1e6, n_photons=0, seed=8),
    ]


def test_batch_sweep_config():
    setup, insts = sb.config_batch_sweep(n_inst=256, seed=2)
    assert len(insts) == 256
    modes = {i["mode"] for i in insts}
    assert modes == {0, 1, 2}
    assert all(1e5 <= i["n_photons"] <= 1e7 for i in insts)
    assert all(0.5e6 <= i["f_u"] <= 2e6 and 0.0 <= i["n_max"] <= 2e-3 for i in insts)
    assert len({i["seed"] for i in insts}) == 256
    assert setup.film_shape() == (32, 128, 128)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [L.PREC_MIXED, L.PREC_FP32])
def test_batch_matches_single_renders(prec):
    setup = sb.config_plain_small(spatial_x=32, spatial_y=32, path_length_bins=8, precision_mode=prec)
    insts = _instances()
    films, st = sb.render_batch(setup, insts)
    assert films.shape == (len(insts),) + setup.film_shape()
    assert st.photons == sum(i["n_photons"] for i in insts)
    for i, inst in enumerate(insts):
        over = {k: v for k, v in inst.items() if k != "n_photons"}
        if inst["n_photons"] == 0:
            assert not films[i].any()
            continue
        ref, rst = sb.render(dataclasses.replace(setup, **over), inst["n_photons"])
        assert ref.sum() > 0
        np.testing.assert_allclose(films[i], ref, rtol=1e-4, atol=1e-6 * ref.max())
        assert abs(films[i].sum() / ref.sum() - 1.0) < 1e-5


@pytest.mark.gpu
def test_batch_rejects_other_fields():
    setup = sb.config_plain_small(spatial_x=16, spatial_y=16, path_length_bins=4)
    with pytest.raises(sb.SmpError):
        sb.render_batch(setup, [dict(field_type=L.FIELD_PLANEWAVE, wave_amp=(1e-3,), wave_k=((0.0, 1e3, 0.0),),
                                     wave_phase=(0.0,), n_photons=100, seed=1)])
