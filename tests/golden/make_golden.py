"""Generate the golden fixtures in this directory from the reference checkout.

Run in the container that has the reference (default /root/reference) and the reference's own
primitives built under oracle/_ref (oracle/ref/build_ref.sh):

    python tests/golden/make_golden.py [reference-root]

Writes:
  spline1d.json   inputs of renderer/samples/spline_tests.cpp:8-11 and a subset of
                  splinepractice/interpolate1d.csv (value, d1, d2 on t = -30..44 step 0.01)
  spline3d.json   the 10x10x10 input array of spline_tests.cpp:100, splinepractice/coefficients3d.csv
                  and a subset of splinepractice/interpolate3d.csv (7 derivative combinations)
  kernel.json     a subset of splinepractice/kernel.csv (cubic B-spline kernels k0, k1, k2)
  sfmt.json       float draws of the reference's SFMT engine (renderer/src/rng_sse.cpp) per seed
  primitives.json outputs of the reference's compiled phase.cpp / warp.cpp / util.h / bsdf.cpp /
                  pmf.h / lens.cpp for fixed inputs and seeds
  textures.json   sha256 of renderer/images/Disk_501.pfm's texels
"""
import ctypes as C
import hashlib
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
# the reference checkout: the first argument, else $SIMPLER_REFERENCE_ROOT, else /root/reference
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SIMPLER_REFERENCE_ROOT", "/root/reference")


def read(rel):
    with open(os.path.join(REF, rel)) as f:
        return f.read()


def csv_floats(rel):
    vals = []
    for line in read(rel).splitlines():
        for tok in line.replace(",", " ").split():
            vals.append(float(tok))
    return vals


def dump(name, obj):
    with open(os.path.join(HERE, name), "w") as f:
        json.dump(obj, f, separators=(",", ":"))


def spline1d():
    src = read("renderer/samples/spline_tests.cpp")
    x = [float(v) for v in re.search(r"Float x\[\] = \{([^}]*)\};", src).group(1).split(",")]
    vals = np.array(csv_floats("splinepractice/interpolate1d.csv"))
    n = len(vals) // 3
    t = -30.0 + 0.01 * np.arange(n)
    idx = np.arange(0, n, 13)
    dump("spline1d.json", {"data": x, "xmin_sq": 13, "xmax_sq": 803, "t": t[idx].tolist(),
                           "value": vals[idx].tolist(), "d1": vals[n + idx].tolist(), "d2": vals[2 * n + idx].tolist(),
                           "source": "renderer/samples/spline_tests.cpp:8-30, splinepractice/interpolate1d.csv"})


def spline3d():
    src = read("renderer/samples/spline_tests.cpp")
    m = re.search(r"//\s*Float x\[\] = \{([^}]*)\};\s*\n//\s*int N\[\] = \{10, 10, 10\}", src)
    data = [float(v) for v in m.group(1).split(",")]
    assert len(data) == 1000
    coeff = csv_floats("splinepractice/coefficients3d.csv")
    assert len(coeff) == 1000
    interp = np.array(csv_floats("splinepractice/interpolate3d.csv")).reshape(-1, 7)
    pts = []
    for tz in np.arange(-1.0, 12.001, 1.5):
        for ty in np.arange(1.0, 12.001, 1.5):
            for tx in np.arange(1.0, 12.001, 1.5):
                pts.append((tx, ty, tz))
    pts = np.array(pts)
    assert len(pts) == len(interp)
    dump("spline3d.json", {"data": data, "coeff_rows": coeff, "points": pts.tolist(), "values": interp.tolist(),
                           "derivs": [[0, 0, 0], [1, 0, 0], [2, 0, 0], [0, 2, 0], [0, 0, 1], [0, 1, 1], [1, 0, 1]],
                           "source": "renderer/samples/spline_tests.cpp:98-130, splinepractice/coefficients3d.csv, "
                                     "splinepractice/interpolate3d.csv"})


def kernel():
    rows = np.array(csv_floats("splinepractice/kernel.csv")).reshape(-1, 2)
    n = len(rows) // 3
    idx = np.arange(0, n, 7)
    dump("kernel.json", {"x": rows[idx, 0].tolist(), "k0": rows[idx, 1].tolist(), "k1": rows[n + idx, 1].tolist(),
                         "k2": rows[2 * n + idx, 1].tolist(), "source": "splinepractice/kernel.csv"})


def ref_lib():
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_bridge
    lib = oracle_bridge.ref_prims()
    if lib is None:
        raise SystemExit("oracle/_ref/libref_prims.so missing: run oracle/ref/build_ref.sh first")
    return lib


def f32p(a):
    return C.c_void_p(a.ctypes.data)


def sfmt():
    lib = ref_lib()
    out = {}
    for seed in [0, 1, 2, 3, 17, 12345, 999999, 2 ** 40 + 7]:
        a = np.zeros(700, np.float32)
        lib.ref_sfmt_float(C.c_uint64(seed), 700, f32p(a))
        out[str(seed)] = a.tolist()
    dump("sfmt.json", {"draws": out, "source": "renderer/src/rng_sse.cpp (compiled by oracle/ref/build_ref.sh)"})


def primitives():
    lib = ref_lib()
    rng = np.random.default_rng(11)
    out = {"hg": [], "hg_f": [], "hemisphere": [], "fresnel": [], "refract": [], "coord": [], "bsdf": [],
           "pmf": [], "lens": [], "source": "renderer/src/{phase,warp,bsdf,lens}.cpp, include/{util,pmf}.h"}
    for k in range(200):
        g = float(rng.choice([0.0, 0.3, 0.85, 0.9, -0.5]))
        d = rng.standard_normal(3).astype(np.float32)
        d /= np.linalg.norm(d)
        o = np.zeros(3, np.float32)
        c = lib.ref_hg_sample(g, f32p(d), C.c_uint64(k), k % 5, f32p(o))
        out["hg"].append([g, d.tolist(), k, k % 5, o.tolist(), c])
        o2 = rng.standard_normal(3).astype(np.float32)
        o2 /= np.linalg.norm(o2)
        out["hg_f"].append([g, d.tolist(), o2.tolist(), lib.ref_hg_f(g, f32p(d), f32p(o2))])
        u0, u1 = float(np.float32(rng.random())), float(np.float32(rng.random()))
        h = np.zeros(3, np.float32)
        lib.ref_hemisphere(u0, u1, f32p(h))
        out["hemisphere"].append([u0, u1, h.tolist()])
        ci, ct, eta = [float(np.float32(v)) for v in (rng.uniform(-1, 1), rng.uniform(-1, 1), rng.choice([1.3333, 0.75, 1.0]))]
        out["fresnel"].append([ci, ct, eta, lib.ref_fresnel(ci, ct, eta)])
        n = np.zeros(3, np.float32)
        n[k % 3] = 1.0 if (k // 3) % 2 else -1.0
        a = (rng.standard_normal(3) * [1.0, 1.0, 1.0]).astype(np.float32)
        if k % 4 == 0:
            a *= 1.3333
        b = np.zeros(3, np.float32)
        ok = lib.ref_refract(f32p(a), f32p(n), eta, f32p(b))
        out["refract"].append([a.tolist(), n.tolist(), eta, int(ok), b.tolist()])
        bb, cc = np.zeros(3, np.float32), np.zeros(3, np.float32)
        lib.ref_coordinate_system(f32p(d), f32p(bb), f32p(cc))
        out["coord"].append([d.tolist(), bb.tolist(), cc.tolist()])
        ob = np.zeros(3, np.float32)
        lib.ref_bsdf_sample(1.0, 1.3333, f32p(a), f32p(n), C.c_uint64(1000 + k), k % 3, f32p(ob))
        out["bsdf"].append([a.tolist(), n.tolist(), 1000 + k, k % 3, ob.tolist()])
    pdf = np.array([0, 0, 1, 2, 0, 3, 0, 0, 5, 1, 0], dtype=np.float64)
    us = np.array([0.0, 1e-7, 0.05, 0.1, 0.25, 0.5, 0.75, 0.9, 0.99, 0.9999999], dtype=np.float32)
    idx = np.zeros(len(us), np.int64)
    cdf = np.zeros(len(pdf) + 1, np.float32)
    lib.ref_pmf_sample(f32p(pdf), len(pdf), len(us), f32p(us), f32p(idx), f32p(cdf))
    out["pmf"] = {"pdf": pdf.tolist(), "u": us.tolist(), "idx": idx.tolist(), "cdf": cdf.tolist()}
    for k in range(40):
        origin = np.array([0.005, 0.0, 0.0], np.float32)
        pos = np.array([0.006, rng.uniform(-1e-3, 1e-3), rng.uniform(-1e-3, 1e-3)], np.float32)
        dirv = np.array([-1.0, rng.uniform(-0.1, 0.1), rng.uniform(-0.1, 0.1)], np.float32)
        dirv /= np.linalg.norm(dirv)
        tot = np.zeros(1, np.float32)
        p2, d2 = pos.copy(), dirv.copy()
        ok = lib.ref_lens_propagate(f32p(origin), 0.0015, 0.015, k % 2, f32p(p2), f32p(d2), f32p(tot))
        out["lens"].append([pos.tolist(), dirv.tolist(), k % 2, int(ok), p2.tolist(), d2.tolist(), float(tot[0])])
    dump("primitives.json", out)


def textures():
    d = open(os.path.join(REF, "renderer/images/Disk_501.pfm"), "rb").read()
    tex = np.frombuffer(d[-501 * 501 * 8:], dtype="<f8").reshape(501, 501)
    dump("textures.json", {"Disk_501": {"shape": [501, 501], "sha256_f64_le": hashlib.sha256(tex.tobytes()).hexdigest(),
                                        "sum": float(tex.sum()), "source": "renderer/images/Disk_501.pfm"}})


if __name__ == "__main__":
    spline1d()
    spline3d()
    kernel()
    sfmt()
    primitives()
    textures()
    print("golden fixtures written to", HERE)
