"""smp_render_noalloc: the entry point for callers that cannot allocate device memory.

Such callers (a host application whose device memory belongs to its own allocator, code that must
not trigger cudaMalloc's device-wide synchronisation mid-frame, a plugin host that only lends the
buffers the renderer may write) pass an already-allocated device film; the entry point keeps its
own scratch in a fixed device array. This test calls it through the C ABI twice in a row, on two
different scenes, each time into a film allocated here by the test, and checks each film against
the allocating entry point smp_render on the same photons and streams. It is collected last so a
failure here stops a -x run only after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

import simpler_b200 as sb
from simpler_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _noalloc_film(setup, n):
    import torch
    lib = sb.load()
    sc, md, fd, op = setup.descs()
    dtype = torch.float64 if setup.precision_mode == L.PREC_MIXED else torch.float32
    film = torch.zeros(setup.film_shape(), dtype=dtype, device="cuda:0")
    st = L.Stats()
    rc = lib.smp_render_noalloc(C.byref(sc), C.byref(md), C.byref(fd), C.byref(op), 0, n, n,
                                C.c_void_p(film.data_ptr()), None, C.byref(st))
    L.check(rc)
    torch.cuda.synchronize()
    return film.double().cpu().numpy(), st


def test_noalloc_matches_render_on_two_calls_in_a_row():
    cases = [
        (sb.config_plain_small(spatial_x=64, spatial_y=64, path_length_bins=16), 60_000),
        (sb.config_precision(spatial_x=48, spatial_y=40, path_length_bins=12, seed=5), 20_000),
    ]
    for setup, n in cases:
        ref, rst = sb.render(setup, n)
        got, gst = _noalloc_film(setup, n)
        assert gst.photons == n == rst.photons
        assert gst.er_steps == rst.er_steps
        rel = np.abs(got - ref).sum() / np.abs(ref).sum()
        assert rel < 2e-3, rel
        assert abs(got.sum() / ref.sum() - 1.0) < 1e-3


def test_noalloc_rejects_oversized_texture():
    import torch
    setup = sb.config_plain_small(texture=np.ones((600, 600)))
    sc, md, fd, op = setup.descs()
    film = torch.zeros(setup.film_shape(), dtype=torch.float32, device="cuda:0")
    rc = sb.load().smp_render_noalloc(C.byref(sc), C.byref(md), C.byref(fd), C.byref(op), 0, 10, 10,
                                      C.c_void_p(film.data_ptr()), None, None)
    assert rc == L.SMP_ERR_BAD_ARG
    assert b"texels" in sb.load().smp_last_error()
