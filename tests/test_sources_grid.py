"""The point-source field (rif_sources, scene.cpp:139-195) sampled on a tricubic grid
(`sources_to_spline`) against the direct sum over every source, at random points of the medium."""
import numpy as np
import pytest

import simpler_b200 as sb
from simpler_b200 import _lib as L


def test_sources_to_spline_rejects_other_fields():
    with pytest.raises(ValueError):
        sb.sources_to_spline(sb.config_plain_small())


def test_grid_offset_in_layout():
    assert [f for f, _ in L.FieldDesc._fields_][-1] == "grid_offset"
    assert sb.check_layout()["smp_field_desc"][0] == C_sizeof_field_desc()


def C_sizeof_field_desc():
    import ctypes as C
    return C.sizeof(L.FieldDesc)


@pytest.mark.gpu
def test_sources_grid_matches_direct_sum():
    s = sb.config_sources()
    pts = np.random.default_rng(0).uniform(-0.0049, 0.0049, size=(20000, 3))
    nd, gd = sb.field_eval(s, 0.0, pts)
    errs = []
    for n in (64, 96):
        sp = sb.sources_to_spline(s, n)
        assert sp.field_type == L.FIELD_SPLINE and sp.grid_offset == s.n_o
        ns, gs = sb.field_eval(sp, 0.0, pts)
        # n: within a couple of float ulps of n ~ 1.3333 (the direct sum's own resolution) of a
        # 1.8e-5 field
        assert np.abs(ns - nd).max() <= 4 * 1.2e-7
        errs.append(np.abs(gs - gd).max() / np.abs(gd).max())
    assert errs[1] < 2e-3 and errs[1] < errs[0]     # measured 3.0e-3, 6.7e-4


@pytest.mark.gpu
def test_sources_grid_renders():
    s = sb.sources_to_spline(sb.config_sources(), 64)
    img, st = sb.render(s, 20000)
    assert st.photons == 20000 and st.nan_photons == 0 and img.sum() > 0
