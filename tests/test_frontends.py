"""The reference's front-ends over the B200 library: file formats, the key=value command line of
renderer/samples/renderer3d_sample.cpp, the JSON settings of simplER.cpp, and the pybind modules.

CPU tests parse and assemble descriptors only (the binaries' --dry-run); the GPU tests render
through each front-end and compare with the Python entry point on the same photons.
"""
import ctypes as C
import json
import math
import os
import sys
import subprocess

import numpy as np
import pytest

import simpler_b200 as sb
from simpler_b200 import _lib as L
from simpler_b200 import pfm
from simpler_b200 import build as _build

# the reference's modules under their own names: their directory goes on sys.path, as the reference's
# build directory does for its users, and `import scene_pybind` is unchanged
sys.path.insert(0, _build.PYBIND_DIR)
import image_pybind  # noqa: E402
import medium_pybind  # noqa: E402
import phase_pybind  # noqa: E402
import photon_pybind  # noqa: E402
import scene_pybind  # noqa: E402
import tvector_pybind  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "simpler_b200", "bin")


def run_bin(name, args, cwd):
    res = subprocess.run([os.path.join(BIN, name), *args], capture_output=True, text=True, cwd=cwd, timeout=120)
    return res.returncode, res.stdout, res.stderr


def parse_dump(text):
    out = {}
    for line in text.splitlines():
        if " = " in line:
            k, v = line.split(" = ", 1)
            out[k.strip()] = v.strip()
    return out


@pytest.fixture
def texture_file(tmp_path):
    tex = sb.disk_texture(41, 300)
    path = tmp_path / "disk.pfm"
    pfm.write_pfm(str(path), tex)
    return str(path), tex


# ---- file formats -----------------------------------------------------------------------------

def test_pfm_texture_round_trip(tmp_path):
    tex = np.random.default_rng(0).random((7, 5))
    p = str(tmp_path / "t.pfm")
    pfm.write_pfm(p, tex)
    raw = open(p, "rb").read()
    assert raw.startswith(b"Pf\n5 7\n-1\n")
    # stored bottom row first (image.h:232-238 flips on read)
    stored = np.frombuffer(raw[-7 * 5 * 8:], "<f8").reshape(7, 5)
    np.testing.assert_array_equal(stored, tex[::-1])
    np.testing.assert_array_equal(pfm.read_pfm(p), tex)


def test_pfm3d_layout(tmp_path):
    film = np.arange(4 * 3 * 2, dtype=np.float64).reshape(4, 3, 2)
    p = str(tmp_path / "f.pfm3d")
    pfm.write_pfm3d(p, film)
    raw = open(p, "rb").read()
    assert raw[:raw.index(b"-1\n") + 3] == b"Pf\n2 3 4\n-1\n"       # image.cpp:176-195
    np.testing.assert_array_equal(np.frombuffer(raw[-film.nbytes:], "<f8"), film.reshape(-1))
    np.testing.assert_array_equal(pfm.read_pfm3d(p), film)


def test_vol_round_trip(tmp_path):
    g = np.random.default_rng(1).random((4, 5, 6)).astype(np.float32)
    p = str(tmp_path / "g.vol")
    pfm.write_vol(p, g, (-1.0, -2.0, -3.0), (1.0, 2.0, 3.0))
    v, lo, hi = pfm.read_vol(p)
    np.testing.assert_array_equal(v, g)
    assert lo == (-1.0, -2.0, -3.0) and hi == (1.0, 2.0, 3.0)


# ---- renderer3d (key=value) -------------------------------------------------------------------

def test_renderer3d_dry_run_matches_setup(texture_file, tmp_path):
    path, tex = texture_file
    rc, out, err = run_bin("renderer3d", ["--dry-run", f"projectorTexture={path}", "sigmaT=111.1", "albedo=0.9",
                                          "gVal=0.9", "mode=1", "n_max=2e-3", "spatialX=64", "spatialY=32",
                                          "pathLengthBins=16", "pathLengthMax=0.05", "emitter_gap=0.002",
                                          "sensor_gap=0.001", "emitter_distance=0.01", "printInputs=false",
                                          "useDirect=TRUE"], str(tmp_path))
    assert rc == 0, err
    d = parse_dump(out)
    assert d["scene.medium_l"] == "-0.015 -5 -5" and d["scene.medium_r"] == "0.015 5 5"
    assert float(d["scene.light_origin"].split()[0]) == pytest.approx(0.015 + f32(0.01), abs=1e-8)
    assert d["scene.texture"] == f"{tex.shape[1]} x {tex.shape[0]}"
    assert d["scene.film"] == "64 32 16"
    assert d["field.type"] == "0" and d["field.mode"] == "1"
    assert float(d["field.egap_end_x"]) == pytest.approx(float(np.float32(0.015) - np.float32(0.002)), abs=1e-9)
    assert float(d["field.sgap_begin_x"]) == pytest.approx(float(np.float32(-0.015) + np.float32(0.001)), abs=1e-9)
    assert d["opts.use_direct"] == "1"
    assert d["output"] == "USOCTRendering.pfm3d"


@pytest.mark.parametrize("args,msg", [
    (["bogus"], "should be in the format arg=value"),
    (["nosuchkey=1"], "Unknown variable in the input argument:nosuchkey"),
    (["useDirect=maybe"], "useDirect should be either true or false; Argument maybe not recognized"),
    (["center1=1,2"], "Three input coordinates required for center1"),
    (["emitter_gap=0.02", "sensor_gap=0.02"], "sum of sensor and emitter gaps is more than the medium size"),
    (["emitter_gap=0.05"], "invalid gap between the emitter and the US"),
    (["emitter_lens_active=true"], "emitter_distance should be strictly positive"),
    (["phi_min=2", "phi_max=1"], "phi_max must be greater than or equal to phi min"),
    (["stricts=true", "sigmaT=1"], "crashing as one or more inputs is absent"),
])
def test_renderer3d_errors(args, msg, tmp_path):
    rc, out, err = run_bin("renderer3d", ["--dry-run", *args], str(tmp_path))
    assert rc != 0
    assert msg in err


def test_renderer3d_strict_lists_missing(tmp_path):
    rc, _, err = run_bin("renderer3d", ["--dry-run", "stricts=true", "sigmaT=1", "albedo=0.9"], str(tmp_path))
    assert rc != 0
    assert "gVal is not specified" in err and "sigmaT is not specified" not in err
    assert "n_max is not specified" in err      # rif_analytical block (renderer3d_sample.cpp:668-690)


def test_renderer3d_sources_inferred(texture_file, tmp_path):
    path, _ = texture_file
    rc, out, err = run_bin("renderer3d", ["--dry-run", f"projectorTexture={path}", "n_scaling=2e-5",
                                          "center1=0,0,-0.0508", "printInputs=false"], str(tmp_path))
    assert rc == 0, err
    d = parse_dump(out)
    assert d["field.type"] == "1"
    assert d["field.f_u"] == "5000000"         # rif_sources defaults (renderer3d_sample.cpp:117-136)


# ---- simplER (JSON) -----------------------------------------------------------------------------

def settings(texture):
    return {
        "stricts": True, "rendering_type": "rif_sources", "threads": -1, "emitter_gap": 0.0, "sensor_gap": 0.0,
        "use_bounce_decomposition": False, "print_inputs": False, "projector_texture": texture,
        "film_parameters": {"path_length": {"min": 0.0, "max": 1e5, "bins": 1}, "spatial": {"x": 96, "y": 96}},
        "adoc_geometry_parameters": {"half_theta_limit": 0.0, "emitter_size": 0.001, "sensor_size": 0.001,
                                     "emitter_distance": 0.0, "sensor_distance": 0.0},
        "scattering_parameters": {"sigma_t": 0.0, "albedo": 0.9, "g_val": 0.9},
        "rendering_parameters": {"num_photons": 10000, "use_direct": True, "max_depth": -1, "max_pathlength": 1e5,
                                 "use_angular_sampling": True},
        "importance_sampling_parameters": {"distribution": "none", "g_or_kappa": 1.0},
        "scene_parameters": {"medium_lx": -0.00635, "medium_rx": 0.00635},
        "rif_parameters": {"f_u": 2e6, "speed_u": 1500.0, "precision": 4, "rr_weight": 1e-3, "er_stepsize": 1e-4,
                           "direct_to_l": 1e-6, "use_initialization_hack": False, "n_o": 1.3333,
                           "n_scaling": 2.15e-5, "n_coeff": 1, "radius": 0.0508, "center1": [0.0, 0.0, -0.0508],
                           "center2": [0.0, -0.0508, 0.0], "active1": True, "active2": True,
                           "phase1": math.pi, "phase2": math.pi, "chordlength": 0.0127, "theta_sources": 10,
                           "trans_z_sources": 5},
        "lens_parameters": {"emitter_lens_aperture": 0.3, "emitter_lens_focal_length": 0.3,
                            "emitter_lens_active": False, "sensor_lens_aperture": 0.3,
                            "sensor_lens_focal_length": 0.3, "sensor_lens_active": False},
    }


def test_simpler_json_dry_run(texture_file, tmp_path):
    path, _ = texture_file
    cfg = tmp_path / "fus.json"
    cfg.write_text(json.dumps(settings(path), indent=2))
    rc, out, err = run_bin("simplER", ["--dry-run", str(cfg)], str(tmp_path))
    assert rc == 0, err
    d = parse_dump(out)
    assert d["field.type"] == "1"
    assert d["scene.film"] == "96 96 1"
    assert d["scene.medium_l"].split()[0] == "-0.00635"
    assert d["output"].startswith("rif_sources_") and d["output"].endswith(".pfm3d")


def test_simpler_json_strict_missing(texture_file, tmp_path):
    path, _ = texture_file
    s = settings(path)
    del s["rif_parameters"]["radius"]
    cfg = tmp_path / "bad.json"
    cfg.write_text(json.dumps(s))
    rc, _, err = run_bin("simplER", ["--dry-run", str(cfg)], str(tmp_path))
    assert rc != 0 and "rif_parameters.radius" in err
    s["stricts"] = False
    cfg.write_text(json.dumps(s))
    rc, _, err = run_bin("simplER", ["--dry-run", str(cfg)], str(tmp_path))
    assert rc == 0, err


def test_simpler_json_bad_type(texture_file, tmp_path):
    path, _ = texture_file
    s = settings(path)
    s["rendering_type"] = "rif_magic"
    cfg = tmp_path / "bad.json"
    cfg.write_text(json.dumps(s))
    rc, _, err = run_bin("simplER", ["--dry-run", str(cfg)], str(tmp_path))
    assert rc != 0 and "Invalid rendering_type: 'rif_magic'" in err


# ---- pybind modules ---------------------------------------------------------------------------

def pybind_scene(texture_path, setup):
    """The reference's rif_analytical Scene constructor arguments for a Setup (scene.h:47-105)."""
    V3, V2 = tvector_pybind.Vec3f, tvector_pybind.Vec2f
    s = setup
    ang = float(np.float32(math.pi))
    return scene_pybind.Scene(
        s.ior, V3(*s.medium_l), V3(*s.medium_r), V3(s.medium_r[0] + s.emitter_distance, 0, 0),
        V3(math.cos(ang), math.sin(ang), 0), s.half_theta_limit, texture_path, V2(s.emitter_size, s.emitter_size),
        s.Li, V3(s.medium_l[0] - s.sensor_distance, 0, 0), V3(-1, 0, 0), V3(0, -1, 0),
        V2(s.sensor_size, s.sensor_size), V2(s.path_length_min, s.path_length_max), s.use_bounce_decomposition,
        "vmf", 4.0, V3(s.medium_r[0], 0, 0), s.emitter_lens_aperture, s.emitter_lens_focal_length,
        s.emitter_lens_active, V3(s.medium_l[0], 0, 0), s.sensor_lens_aperture, s.sensor_lens_focal_length,
        s.sensor_lens_active,
        s.f_u, s.speed_u, s.n_o, s.n_max, s.n_clip, s.phi_min, s.phi_max, s.mode,
        V3(-1, 0, 0), V3(0, 0, 1), V3(0, 0, 0), s.er_stepsize, s.direct_tol, s.rr_weight, s.precision,
        float(np.float32(s.medium_r[0]) - np.float32(s.emitter_gap)),
        float(np.float32(s.medium_l[0]) + np.float32(s.sensor_gap)), s.use_initialization_hack)


def f32(x):
    return float(np.float32(x))


def test_pybind_scene_descriptors(texture_file):
    path, tex = texture_file
    setup = sb.config_plain_small(texture=tex, spatial_x=16, spatial_y=16, path_length_bins=4)
    sc = pybind_scene(path, setup)
    ref_s, ref_f = setup.scene_desc(), setup.field_desc()
    got_s, got_f = descs(sc)
    for name in ("medium_l", "medium_r", "light_origin", "light_dir", "view_origin", "view_dir", "view_horizontal",
                 "emitter_lens_origin", "sensor_lens_origin", "pathlength_range", "light_plane", "view_plane"):
        assert list(getattr(got_s, name)) == [f32(v) for v in getattr(ref_s, name)], name
    assert (got_s.tex_x, got_s.tex_y) == (ref_s.tex_x, ref_s.tex_y)
    np.testing.assert_array_equal(sc.texture, tex)
    for name in ("type", "mode", "precision", "f_u", "speed_u", "n_o", "n_max", "n_clip", "phi_min", "phi_max",
                 "er_stepsize", "egap_end_x", "sgap_begin_x"):
        assert getattr(got_f, name) == pytest.approx(f32(getattr(ref_f, name)), rel=1e-7), name
    sc.set_n_max(5e-4)
    sc.set_f_u(1e6)
    got_s, got_f = descs(sc)
    assert got_f.n_max == f32(5e-4) and got_f.f_u == 1e6
    assert sc.form == "rif_analytical"


def descs(sc):
    """The compiled Scene's C-ABI descriptors (smp_scene_desc, smp_field_desc) as ctypes structs."""
    b_s, b_f = sc.descriptors()
    return L.SceneDesc.from_buffer_copy(b_s), L.FieldDesc.from_buffer_copy(b_f)


def test_pybind_scene_forms(texture_file, tmp_path):
    path, _ = texture_file
    with pytest.raises(TypeError):
        scene_pybind.Scene(1.0, 2.0)
    img = image_pybind.SmallImage(4, 4, 2)
    assert (img.get_x_res(), img.get_y_res(), img.getZRes()) == (4, 4, 2)
    img.pixels[1, 2, 3] = 7.0
    assert img.get_pixel(3, 2, 1) == 7.0
    view = np.asarray(img)                                # buffer protocol: the same memory, no copy
    assert view.shape == (2, 4, 4) and view[1, 2, 3] == 7.0
    view[0, 0, 0] = 2.5
    assert img.get_pixel(0, 0, 0) == 2.5
    img.writePFM3D(str(tmp_path / "img.pfm3d"))
    np.testing.assert_array_equal(pfm.read_pfm3d(str(tmp_path / "img.pfm3d")), view)
    med = medium_pybind.Medium(100.0, 0.9, phase_pybind.henyey_greenstein(0.9))
    assert med.getSigmaT() == 100.0 and med.phase.getG() == f32(0.9)
    v = tvector_pybind.Vec3f(1.0, 2.0, 3.0)
    assert [v.index(i) for i in range(3)] == [1.0, 2.0, 3.0]


def test_explicit_source_arcs_match_chord():
    """Explicit theta/trans_z ranges equal to the chord-derived ones give the same field."""
    s = sb.Setup(field_type=L.FIELD_SOURCES, theta_sources=6, trans_z_sources=5, radius=0.0508, chordlength=0.0127,
                 center1=(0.0, 0.0, -0.0508), center2=(0.0, -0.0508, 0.0), n_scaling=2e-5, f_u=2e6)
    a = s.field_desc()
    b = s.field_desc()
    half = math.asin(0.0127 / (2 * 0.0508))
    b.theta_min, b.theta_max, b.trans_z_min, b.trans_z_max = -half, half, -0.0127 / 2, 0.0127 / 2
    import oracle_bridge
    pts = np.random.default_rng(4).uniform(-4e-3, 4e-3, (64, 3))
    na, ga = oracle_bridge.oracle_field_desc(a, 0.7, pts)
    nb, gb = oracle_bridge.oracle_field_desc(b, 0.7, pts)
    np.testing.assert_allclose(na, nb, rtol=1e-6)
    np.testing.assert_allclose(ga, gb, rtol=1e-4, atol=1e-6 * np.abs(ga).max())


# ---- GPU: rendering through the front-ends -------------------------------------------------------

@pytest.mark.gpu
def test_renderer3d_renders_same_film(texture_file, tmp_path):
    path, tex = texture_file
    args = [f"projectorTexture={path}", "sigmaT=111.1", "albedo=0.9", "gVal=0.9", "mode=0", "n_max=1e-3",
            "spatialX=32", "spatialY=32", "pathLengthBins=8", "pathLengthMax=0.1", "numPhotons=20000",
            "mediumLx=-0.005", "mediumRx=0.005", "mediumLy=-0.005", "mediumRy=0.005", "mediumLz=-0.005",
            "mediumRz=0.005", "er_stepsize=1e-5", "precision=4", "emitter_size=0.001", "sensor_size=0.01",
            "phi_min=0", "phi_max=6.283185307179586", "useDirect=true", "renderPrecision=mixed",
            "outFilePrefix=out", "printInputs=false"]
    rc, out, err = run_bin("renderer3d", args, str(tmp_path))
    assert rc == 0, err
    film = pfm.read_pfm3d(str(tmp_path / "out.pfm3d"))
    setup = sb.Setup(texture=tex, sigma_t=f32(111.1), albedo=f32(0.9), g=f32(0.9), mode=0, n_max=f32(1e-3),
                     n_clip=1e-3, spatial_x=32, spatial_y=32, path_length_bins=8, path_length_max=0.1,
                     er_stepsize=f32(1e-5), precision=4, phi_min=0.0, phi_max=f32(2 * math.pi),
                     medium_l=(-0.005,) * 3, medium_r=(0.005,) * 3, use_direct=True,
                     emitter_size=f32(0.001), sensor_size=f32(0.01), precision_mode=L.PREC_MIXED,
                     use_initialization_hack=True, use_bounce_decomposition=True, half_theta_limit=12.8e-3)
    ref, _ = sb.render(setup, 20000)
    assert ref.sum() > 0
    np.testing.assert_allclose(film, ref, rtol=1e-9, atol=1e-12 * ref.max())     # FP64 atomics: order only


@pytest.mark.gpu
def test_pybind_renderer_matches_render(texture_file):
    path, tex = texture_file
    setup = sb.config_plain_small(texture=tex, spatial_x=32, spatial_y=32, path_length_bins=8,
                                  precision_mode=L.PREC_MIXED, use_direct=True)
    sc = pybind_scene(path, setup)
    img = image_pybind.SmallImage(32, 32, 8)
    med = medium_pybind.Medium(setup.sigma_t, setup.albedo, phase_pybind.henyey_greenstein(setup.g))
    r = photon_pybind.Renderer(-1, -1.0, True, True, 8, precision=L.PREC_MIXED)
    r.renderImage(img, med, sc, 20000)
    # the Setup path with every Float argument rounded as the pybind layer rounds it
    for k in ("sigma_t", "albedo", "g", "f_u", "n_max", "n_clip", "phi_min", "phi_max", "er_stepsize", "n_o",
              "speed_u", "emitter_size", "sensor_size", "ior", "path_length_min", "path_length_max",
              "emitter_lens_aperture", "emitter_lens_focal_length", "sensor_lens_aperture",
              "sensor_lens_focal_length", "half_theta_limit", "Li"):
        setattr(setup, k, f32(getattr(setup, k)))
    setup.medium_l = tuple(f32(v) for v in setup.medium_l)
    setup.medium_r = tuple(f32(v) for v in setup.medium_r)
    ref, _ = sb.render(setup, 20000)
    assert ref.sum() > 0 and r.last_stats["photons"] == 20000
    np.testing.assert_allclose(img.pixels, ref, rtol=1e-9, atol=1e-12 * ref.max())
