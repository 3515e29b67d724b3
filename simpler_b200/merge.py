"""Merging and resuming renders: the replacement for helperScripts/mergeMultipleRenderings.cpp.

Every film a render writes is an average over its photons (each splat carries Li T / N), so films
of independent renders of one scene merge as the photon-weighted mean

    merged = sum_i N_i film_i / sum_i N_i

The reference helper (mergeMultipleRenderings.cpp:207-231) updates a running mean as
mean = (mean (i+1) + x_i) / (i+2) for the i-th extra rendering, which gives the first rendering
twice the weight it should have (for two renderings, 2/3 instead of 1/2); it also assumes equal
photon budgets. `merge_films` weights by photon count and `merge_reference_bins` reads the
helper's per-bin PFM sets (`<prefix>_<i>_<j>.pfm`) with the corrected weights.

Resuming: photon k of a render draws the Philox stream (seed, k), so tracing photons
[N, N + M) and merging with weights N and M gives the film a single N + M photon render gives.

    python -m simpler_b200.merge out.pfm3d a.pfm3d:1000000 b.pfm3d:4000000
"""
from __future__ import annotations

import os
import sys

import numpy as np

from . import pfm


def merge_films(films, photons) -> np.ndarray:
    """Photon-weighted mean of films rendered with `photons[i]` photons each."""
    films = [np.asarray(f, dtype=np.float64) for f in films]
    w = np.asarray(photons, dtype=np.float64)
    if len(films) != len(w) or len(films) == 0:
        raise ValueError("one photon count per film")
    if np.any(w < 0) or w.sum() <= 0:
        raise ValueError("photon counts must be non-negative with a positive sum")
    shape = films[0].shape
    out = np.zeros(shape, dtype=np.float64)
    for f, n in zip(films, w):
        if f.shape != shape:
            raise ValueError(f"film shapes differ: {f.shape} vs {shape}")
        out += f * n
    return out / w.sum()


def merge_pfm3d(out_path: str, paths, photons) -> np.ndarray:
    """Merge PFM3D files (image.cpp:161-206 layout) and write the result."""
    merged = merge_films([pfm.read_pfm3d(p) for p in paths], photons)
    pfm.write_pfm3d(out_path, merged)
    return merged


def merge_reference_bins(prefix: str, renderings: int, bins: int, photons=None, write: bool = True):
    """The reference helper's file set: `<prefix>_<i>_<j>.pfm` for rendering i and path-length
    bin j (2-D PFMs). Returns the merged (bins, y, x) stack and, with `write`, writes
    `<prefix>_mean_<j>.pfm` as the helper does -- with photon weights (equal by default)."""
    w = np.ones(renderings) if photons is None else np.asarray(photons, dtype=np.float64)
    out = []
    for j in range(bins):
        films = [pfm.read_pfm(f"{prefix}_{i}_{j}.pfm") for i in range(renderings)]
        m = merge_films(films, w)
        out.append(m)
        if write:
            pfm.write_pfm(f"{prefix}_mean_{j}.pfm", m)
    return np.stack(out)


def resume(setup, film: np.ndarray, photons_done: int, photons_more: int, stream: int = 0):
    """Continue a render of `setup` that holds `photons_done` photons: trace photons
    [photons_done, photons_done + photons_more) and merge. Returns (film, stats of the new part)."""
    from .render import Plan
    p = Plan(setup)
    try:
        p.clear(stream)
        p.trace(photons_done, photons_more, photons_more, stream)
        new = p.read_image()
        st = p.stats()
    finally:
        p.close()
    return merge_films([film, new], [photons_done, photons_more]), st


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) < 2:
        sys.stderr.write("usage: python -m simpler_b200.merge OUT.pfm3d IN.pfm3d[:PHOTONS] ...\n")
        return 2
    out, ins = argv[0], argv[1:]
    paths, counts = [], []
    for a in ins:
        path, _, n = a.rpartition(":") if ":" in a and not os.path.exists(a) else (a, "", "1")
        paths.append(path)
        counts.append(float(n))
    merge_pfm3d(out, paths, counts)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
