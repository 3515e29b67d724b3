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
