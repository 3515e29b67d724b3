"""Merging and resuming renders (helperScripts/mergeMultipleRenderings.cpp's job, with photon
weights): the Python and C++ mergers on synthetic films, the reference helper's per-bin file set,
and on the GPU a resumed render against one render of all the photons."""
import os
import subprocess

import numpy as np
import pytest

import simpler_b200 as sb
from simpler_b200 import _lib as L
from simpler_b200 import merge, pfm

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MERGE = os.path.join(ROOT, "simpler_b200", "bin", "merge_renderings")


def test_photon_weighted_mean():
    rng = np.random.default_rng(0)
    a, b, c = rng.random((3, 4, 5, 6))
    m = merge.merge_films([a, b, c], [1e6, 3e6, 0])
    np.testing.assert_allclose(m, (a + 3 * b) / 4, rtol=1e-15)
    np.testing.assert_allclose(merge.merge_films([a, b], [7, 7]), (a + b) / 2, rtol=1e-15)
    with pytest.raises(ValueError):
        merge.merge_films([a, b], [1])
    with pytest.raises(ValueError):
        merge.merge_films([a, rng.random((2, 2, 2))], [1, 1])


def test_reference_bin_files_python_and_cli(tmp_path):
    """<prefix>_<i>_<j>.pfm sets: the equal-weight mean (the helper's running mean would give
    rendering 0 weight 2/3 of two), by the Python merger and by bin/merge_renderings."""
    rng = np.random.default_rng(1)
    prefix = str(tmp_path / "run")
    imgs = rng.random((3, 2, 6, 5))                 # renderings x bins x y x
    for i in range(3):
        for j in range(2):
            pfm.write_pfm(f"{prefix}_{i}_{j}.pfm", imgs[i, j])
    stack = merge.merge_reference_bins(prefix, 3, 2, photons=[1, 2, 1], write=False)
    np.testing.assert_allclose(stack, (imgs[0] + 2 * imgs[1] + imgs[2]) / 4, rtol=1e-15)
    res = subprocess.run([MERGE, f"prefix={prefix}", "renderings=3", "pathLengthBins=2"], capture_output=True,
                         text=True, timeout=60)
    assert res.returncode == 0, res.stderr
    for j in range(2):
        np.testing.assert_allclose(pfm.read_pfm(f"{prefix}_mean_{j}.pfm"), imgs[:, j].mean(axis=0), rtol=1e-15)
    res = subprocess.run([MERGE, "bogus=1"], capture_output=True, text=True, timeout=60)
    assert res.returncode != 0 and "Unknown variable in the input argument:bogus" in res.stderr


def test_pfm3d_cli_and_module(tmp_path):
    rng = np.random.default_rng(2)
    a, b = rng.random((2, 3, 4, 5))
    pa, pb = str(tmp_path / "a.pfm3d"), str(tmp_path / "b.pfm3d")
    pfm.write_pfm3d(pa, a)
    pfm.write_pfm3d(pb, b)
    out = str(tmp_path / "m.pfm3d")
    res = subprocess.run([MERGE, "pfm3d", out, pa + ":1000", pb + ":3000"], capture_output=True, text=True, timeout=60)
    assert res.returncode == 0, res.stderr
    np.testing.assert_allclose(pfm.read_pfm3d(out), (a + 3 * b) / 4, rtol=1e-14)
    out2 = str(tmp_path / "m2.pfm3d")
    assert merge.main([out2, pa + ":1", pb + ":1"]) == 0
    np.testing.assert_allclose(pfm.read_pfm3d(out2), (a + b) / 2, rtol=1e-15)


@pytest.mark.gpu
def test_resume_equals_one_render():
    """Photon k draws stream (seed, k): photons [0, N) then [N, N + M) merged with weights N, M
    are the photons of one N + M render. The films agree to the rounding of the per-photon weight
    Li T / N, which is a float and differs between the three renders (a few 1e-7)."""
    setup = sb.config_plain_small(spatial_x=32, spatial_y=32, path_length_bins=8, precision_mode=L.PREC_MIXED)
    full, _ = sb.render(setup, 30000)
    first, _ = sb.render(setup, 12000)
    resumed, st = merge.resume(setup, first, 12000, 18000)
    assert st.photons == 18000
    np.testing.assert_allclose(resumed, full, rtol=2e-6, atol=1e-9 * full.max())
