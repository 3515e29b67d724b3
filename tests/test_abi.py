"""CPU: libsimpler_b200.so loads, exports every entry point of include/simpler_b200.h, its structs
match the ctypes mirrors, and host-side argument checks fail loudly without touching a GPU."""
import ctypes as C
import os
import re

import numpy as np

import simpler_b200 as sb
from simpler_b200 import _lib as L

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "simpler_b200.h")


def declared_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|size_t|const char \*|int64_t)\s*\*?\s*(smp_\w+)\s*\(", src, re.M)))


def test_every_declared_symbol_is_exported():
    lib = sb.load()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(L.EXPORTS) == names


def test_struct_layouts_match():
    sizes = sb.check_layout()
    assert sizes["smp_photon_record"][0] == C.sizeof(L.PhotonRecord)


def test_version_and_errors_without_device():
    lib = sb.load()
    assert lib.smp_version() == 1
    s = sb.config_plain_small()
    sc, md, fd, op = s.descs()
    img = np.zeros(s.film_shape())
    if lib.smp_device_count() == 0:
        rc = lib.smp_render(C.byref(sc), C.byref(md), C.byref(fd), C.byref(op), 10, C.c_void_p(img.ctypes.data), None)
        assert rc == L.SMP_ERR_NO_DEVICE
        assert b"device" in lib.smp_last_error()


def test_bad_arguments_are_rejected_before_any_device_work():
    lib = sb.load()
    s = sb.config_plain_small()
    sc, md, fd, op = s.descs()
    sc.x_res = 0
    img = np.zeros(8)
    assert lib.smp_render(C.byref(sc), C.byref(md), C.byref(fd), C.byref(op), 10, C.c_void_p(img.ctypes.data), None) == L.SMP_ERR_BAD_ARG
    sc, md, fd, op = s.descs()
    fd.er_stepsize = 0.0
    assert lib.smp_render(C.byref(sc), C.byref(md), C.byref(fd), C.byref(op), 10, C.c_void_p(img.ctypes.data), None) == L.SMP_ERR_BAD_ARG
    sc, md, fd, op = s.descs()
    fd.mode = 99                 # above the largest built order
    ptr = C.c_void_p()
    rc = lib.smp_plan_create(C.byref(sc), C.byref(md), C.byref(fd), C.byref(op), C.byref(ptr))
    assert rc in (L.SMP_ERR_UNSUPPORTED, L.SMP_ERR_NO_DEVICE)
    assert lib.smp_texture_cdf(None, 4, 4, None) == L.SMP_ERR_BAD_ARG
    assert lib.smp_spline_prefilter(None, None, None) == L.SMP_ERR_BAD_ARG
    # the adjoint's entry points check their arguments before touching a device
    g = np.zeros(4)
    assert lib.smp_plan_adjoint(None, 0, 10, 10, C.c_void_p(img.ctypes.data), C.c_void_p(g.ctypes.data), None) == L.SMP_ERR_BAD_ARG
    sc, md, fd, op = s.descs()
    sc.x_res = 0
    assert lib.smp_render_adjoint(C.byref(sc), C.byref(md), C.byref(fd), C.byref(op), 10, C.c_void_p(img.ctypes.data),
                                  C.c_void_p(g.ctypes.data), None) == L.SMP_ERR_BAD_ARG
    sc, md, fd, op = sb.config_sources().descs()
    assert lib.smp_adjoint_param_count(C.byref(fd)) == L.SMP_ERR_UNSUPPORTED
    assert lib.smp_adjoint_param_count(None) == L.SMP_ERR_BAD_ARG


def test_sizeof_unknown_is_zero():
    assert sb.load().smp_sizeof(b"nope") == 0
