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


def test_batch_rejects_mixed_refinement_levels():
    """The number of refinement levels is shared by a sweep's instances; a sweep that mixes them is
    refused before anything is allocated."""
    setup = sb.config_plain_small(spatial_x=16, spatial_y=16, path_length_bins=4)
    with pytest.raises(sb.SmpError, match="refinement levels"):
        sb.render_batch(setup, [dict(n_photons=10, seed=1), dict(precision=3, n_photons=10, seed=2)])


@pytest.mark.gpu
def test_batch_instances_keep_their_own_steps():
    """Each instance marches with its own er_stepsize: its film is the single render at that step."""
    setup = sb.config_plain_small(spatial_x=32, spatial_y=32, path_length_bins=8)
    insts = _instances()[:3]
    for inst, h in zip(insts, (1e-5, 4e-5, 2.5e-5)):
        inst["er_stepsize"] = h
    films, st = sb.render_batch(setup, insts)
    steps = 0
    for i, inst in enumerate(insts):
        over = {k: v for k, v in inst.items() if k != "n_photons"}
        ref, rst = sb.render(dataclasses.replace(setup, **over), inst["n_photons"])
        steps += rst.er_steps
        np.testing.assert_allclose(films[i], ref, rtol=1e-4, atol=1e-6 * ref.max())
    # the sweep's order-general field path rounds differently, which moves a few refinement steps
    assert abs(st.er_steps / steps - 1.0) < 1e-5, (st.er_steps, steps)


def _rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


@pytest.mark.gpu
def test_tune_batch_steps_within_budget_and_against_fp64_oracle():
    """The step-size autotuner (smp_batch_tune_steps) on an FP32 sweep: every chosen step is a listed
    multiple of the instance's own step and at most an eighth of its ultrasound wavelength, its
    error (measured in the mixed form) within the budget; and against the FP64 oracle at the nominal
    step on the same photons the tuned FP32 films stay within 1 % relative RMSE (the bound the
    batched form is held to) and within the budget of the larger of the budget and the nominal-step
    FP32 film's own error."""
    from oracle_bridge import oracle_trace
    n = 10000
    setup = sb.config_plain_small()
    assert setup.precision_mode == L.PREC_FP32
    insts = [
        dict(mode=2, n_max=2e-3, n_clip=2e-3, f_u=2e6, n_photons=n, seed=11),
        dict(mode=1, n_max=1e-3, n_clip=1e-3, f_u=1e6, phi_max=3.0, n_photons=n, seed=12),
        dict(mode=0, n_max=1.5e-3, n_clip=1.5e-3, f_u=0.55e6, n_photons=n, seed=13),
        dict(mode=0, n_max=0.0, n_clip=0.0, f_u=0.7e6, n_photons=n, seed=14),
    ]
    budget = 2e-3
    steps, rmse, rounds = sb.tune_batch_steps(setup, insts, budget, n_sample=n)
    assert rounds >= 2                       # the reference and at least one trial
    mults = steps / setup.er_stepsize
    for i, inst in enumerate(insts):
        m = round(mults[i])
        assert abs(mults[i] - m) < 1e-9 and m in (1, 2, 3, 4, 6, 8, 12, 16, 24, 32), mults
        assert m == 1 or steps[i] <= setup.speed_u / inst["f_u"] / 8.0 * (1 + 1e-12)
        assert 0.0 <= rmse[i] <= budget
    assert mults.max() >= 4, mults           # the low-frequency instances take much larger steps
    nominal, _ = sb.render_batch(setup, insts)
    tuned, _ = sb.render_batch(setup, [dict(inst, er_stepsize=float(h)) for inst, h in zip(insts, steps)])
    for i in (0, 2, 3):
        over = {k: v for k, v in insts[i].items() if k != "n_photons"}
        _, ref = oracle_trace(dataclasses.replace(setup, **over), 0, n, n, records=False, real_bits=64)
        e_tuned, e_nominal = _rel(tuned[i], ref), _rel(nominal[i], ref)
        assert e_tuned <= 1e-2, (i, e_tuned, e_nominal, mults[i])
        assert e_tuned <= max(budget, e_nominal) + budget, (i, e_tuned, e_nominal, mults[i])


def test_tune_batch_steps_rejects_bad_arguments():
    """The step tuner's argument checks run before any device work."""
    setup, insts = sb.config_batch_sweep(n_inst=2)
    with pytest.raises(sb.SmpError, match="n_sample"):
        sb.tune_batch_steps(setup, insts, 2e-3, n_sample=0)
    with pytest.raises(sb.SmpError, match="rmse_budget"):
        sb.tune_batch_steps(setup, insts, 0.0)
