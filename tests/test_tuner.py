"""The slot pool's autotuner (smp_plan_tune): trial traces over march-kernel block size, slots per
lane and chunk, the winner cached per process. The schedule changes only the order in which photons
are traced, so a tuned render's film and counts equal an untuned render's on the same photons."""
import numpy as np
import pytest

import simpler_b200 as sb
from simpler_b200 import _lib as L

pytestmark = pytest.mark.gpu


def test_tune_picks_a_candidate_caches_it_and_keeps_the_film():
    s = sb.config_precision(seed=21, spatial_x=64, spatial_y=64, path_length_bins=16)
    n = 300_000
    ref, rst = sb.render(s, n)                  # untuned defaults
    p = sb.Plan(s)
    t = p.tune(200_000)
    assert t.march_block in (128, 256) and t.slots_per_lane in (2, 4, 6, 8) and t.chunk in (64, 96, 128, 192)
    assert t.trials == 19 and t.ms > 0 and t.paths_per_s > 0      # 16 + 1 at 256 threads + the two best again
    film, st = p.render(n)
    p.close()
    assert (st.march_block, st.slots_per_lane, st.chunk, st.tuned) == (t.march_block, t.slots_per_lane, t.chunk, 1)
    assert st.photons == rst.photons == n and st.er_steps == rst.er_steps and st.splats == rst.splats
    assert np.abs(film - ref).sum() <= 1e-12 * np.abs(ref).sum()     # FP64 film: atomic order only
    # a second plan of the same configuration takes the cached schedule without trials
    q = sb.Plan(s)
    t2 = q.tune(200_000)
    q.close()
    assert t2.trials == 0
    assert (t2.march_block, t2.slots_per_lane, t2.chunk) == (t.march_block, t.slots_per_lane, t.chunk)


def test_tune_rejects_other_kernels():
    p = sb.Plan(sb.config_plain_small(kernel=L.KERNEL_PLAIN))
    with pytest.raises(sb.SmpError) as e:
        p.tune(1000)
    p.close()
    assert e.value.code == L.SMP_ERR_UNSUPPORTED


def test_batch_reports_its_schedule():
    setup, insts = sb.config_batch_sweep(n_inst=6, seed=5, scale=0.02)
    films, st = sb.render_batch(setup, insts)
    assert st.tuned == 1 and st.chunk in (64, 96, 128, 192) and st.slots_per_lane in (2, 4, 6, 8)
    assert st.photons == sum(i["n_photons"] for i in insts)


def _rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def test_plan_tune_step_within_budget_and_against_fp64_oracle():
    """The step-size autotuner of a plan (smp_plan_tune_step). On the plain small scene (Bessel mode
    0, 848 kHz: an eighth of its wavelength is 22 times the 0.01 mm step) it takes a multiple of at
    least 4; the film at the tuned step is within the budget of the film at the plan's own step on
    the same photons and within 1 % relative RMSE of the FP64 oracle at the own step; set_field
    restores the field's step. On the plane-wave configuration the step stays a listed multiple below
    an eighth of the 1.5 mm wavelength."""
    from oracle_bridge import oracle_trace
    n, budget = 20000, 2e-3
    s = sb.config_plain_small(precision_mode=L.PREC_MIXED)
    p = sb.Plan(s)
    nominal, _ = p.render(n)
    step, rmse = p.tune_step(n, budget)
    m = step / s.er_stepsize
    assert abs(m - round(m)) < 1e-4 and round(m) in (4, 6, 8, 12, 16), m
    assert step <= s.speed_u / s.f_u / 8.0 * (1 + 1e-6)
    assert 0.0 < rmse <= budget
    tuned, st = p.render(n)
    assert _rel(tuned, nominal) <= budget * 1.05, (_rel(tuned, nominal), rmse)
    _, ref = oracle_trace(s, 0, n, n, records=False, real_bits=64)
    e_tuned, e_nominal = _rel(tuned, ref), _rel(nominal, ref)
    assert e_tuned <= 1e-2 and e_tuned <= e_nominal + budget, (e_tuned, e_nominal)
    p.set_field(s)
    again, _ = p.render(n)
    assert np.abs(again - nominal).sum() <= 1e-12 * np.abs(nominal).sum()     # the own step again
    p.close()
    # the FP32 form: the search runs on a mixed-form copy of the plan, so the float path length's
    # own rounding does not hold the step at its own value
    f = sb.config_plain_small()
    assert f.precision_mode == L.PREC_FP32
    r = sb.Plan(f)
    nominal32, _ = r.render(n)
    step, rmse = r.tune_step(n, budget)
    m = step / f.er_stepsize
    assert abs(m - round(m)) < 1e-4 and round(m) in (4, 6, 8, 12, 16), m
    assert 0.0 < rmse <= budget
    tuned32, _ = r.render(n)
    r.close()
    e_tuned, e_nominal = _rel(tuned32, ref), _rel(nominal32, ref)
    assert e_tuned <= 1e-2 and e_tuned <= max(budget, e_nominal) + budget, (e_tuned, e_nominal)
    w = sb.config_planewave()
    q = sb.Plan(w)
    step, rmse = q.tune_step(10000, budget)
    q.close()
    m = step / w.er_stepsize
    assert abs(m - round(m)) < 1e-4 and round(m) in (1, 2, 3, 4, 6, 8, 12, 16), m
    assert step <= 2.0 * np.pi / np.linalg.norm(w.wave_k[0]) / 8.0 * (1 + 1e-6)
    assert 0.0 <= rmse <= budget


def test_plan_tune_step_rejects_bad_arguments():
    p = sb.Plan(sb.config_plain_small(spatial_x=16, spatial_y=16, path_length_bins=4))
    with pytest.raises(sb.SmpError, match="n_sample"):
        p.tune_step(0, 1e-3)
    with pytest.raises(sb.SmpError, match="rmse_budget"):
        p.tune_step(1000, -1.0)
    p.close()
