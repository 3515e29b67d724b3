"""The texture CDF's guide table (the event kernel's new-photon texel search). For 2^k buckets of u,
entry b is the lower bound of b / 2^k in the CDF; a u in bucket b has its lower bound between the
entries of b and b + 1, so the search narrowed to them returns the texel the full binary search
returns. Checked here on the library's own CDFs (smp_texture_cdf, no GPU) of the two bench textures,
with the guide built by the rule the plan uses."""
import ctypes as C

import numpy as np

import simpler_b200 as sb
from simpler_b200 import _lib as L


def _cdf(tex: np.ndarray) -> np.ndarray:
    t = np.ascontiguousarray(tex, dtype=np.float64)
    out = np.zeros(t.size + 1, dtype=np.float32)
    L.check(L.load().smp_texture_cdf(C.c_void_p(t.ctypes.data), t.shape[1], t.shape[0], C.c_void_p(out.ctypes.data)))
    return out


def _guide(cdf: np.ndarray):
    n1 = cdf.size
    assert np.all(cdf[1:] >= cdf[:-1])                 # the plan builds a guide only for these
    bits = 8
    while (1 << bits) < n1 - 1 and bits < 20:
        bits += 1
    G = 1 << bits
    edges = (np.arange(G + 1, dtype=np.float32) / np.float32(G)).astype(np.float32)
    g = np.searchsorted(cdf, edges, side="left")      # first i with not (cdf[i] < edge)
    return np.concatenate([g, [n1]]), bits


def _lower_bound(cdf, u, lo, hi):
    while lo < hi:
        mid = (lo + hi) >> 1
        if cdf[mid] < u:
            lo = mid + 1
        else:
            hi = mid
    return lo


def test_guided_search_finds_the_full_search_texel():
    rng = np.random.default_rng(7)
    for tex in (sb.disk_texture(), sb.bernoulli_texture(64, 0.5, 1)):
        cdf = _cdf(tex)
        guide, bits = _guide(cdf)
        G = 1 << bits
        us = np.concatenate([rng.random(20000, dtype=np.float32),
                             cdf[rng.integers(0, cdf.size, 5000)],            # on CDF values
                             np.float32([0.0, np.nextafter(np.float32(1.0), np.float32(0.0))])])
        width = 0
        for u in us.astype(np.float32):
            b = min(int(np.float32(u * np.float32(G))), G)
            lo, hi = int(guide[b]), int(guide[b + 1])
            assert _lower_bound(cdf, u, lo, hi) == _lower_bound(cdf, u, 0, cdf.size), (u, lo, hi)
            width = max(width, hi - lo)
        assert width < cdf.size // 16                 # the buckets narrow the search
