// pybind_types.h -- the C++ classes behind the reference's six Python modules
// (renderer/pybindFiles/{tvector,phase,medium,image,scene,photon}_pybind.cpp), over this library's C
// ABI. Each module registers its own classes; the others take them as arguments (photon_pybind's
// renderImage takes the SmallImage, Medium and Scene of image_pybind, medium_pybind and scene_pybind),
// exactly as the reference's modules share their C++ types, so the classes are defined once, here,
// with default visibility.
#pragma once
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/simpler_b200.h"
#include "../host/smp_host.h"

#define SMP_PYBIND_EXPORT __attribute__((visibility("default")))

namespace smp_pybind {

namespace py = pybind11;

// tvec::TVector2<Float>, TVector3<Float>, TVector3<int> (renderer/include/tvector.h)
struct SMP_PYBIND_EXPORT Vec2f {
    float x = 0.0f, y = 0.0f;
};
struct SMP_PYBIND_EXPORT Vec3f {
    float x = 0.0f, y = 0.0f, z = 0.0f;
    // TVector3::index (tvector.h:327-329)
    float index(int i) const {
        if (i < 0 || i > 2) throw py::index_error("Vec3f.index: 0, 1 or 2");
        return i == 0 ? x : (i == 1 ? y : z);
    }
};
struct SMP_PYBIND_EXPORT Vec3i {
    int x = 0, y = 0, z = 0;
};

// pfunc::henyey_greenstein (renderer/include/phase.h)
struct SMP_PYBIND_EXPORT HenyeyGreenstein {
    float g = 0.0f;
};

// med::Medium (renderer/include/medium.h:24-38): sigma_t, albedo and the phase function
struct SMP_PYBIND_EXPORT Medium {
    float sigma_t = 0.0f, albedo = 0.0f;
    HenyeyGreenstein phase;
};

// image::Image3<double> (renderer/include/image.h:290-340), the pybind build's SmallImage: x*y*z
// doubles, index z*X*Y + y*X + x
struct SMP_PYBIND_EXPORT SmallImage {
    int xres = 0, yres = 0, zres = 0;
    std::vector<double> pixels;
    SmallImage(int x, int y, int z) : xres(x), yres(y), zres(z) {
        if (x <= 0 || y <= 0 || z <= 0) throw py::value_error("SmallImage: resolutions must be positive");
        pixels.assign(size_t(x) * y * z, 0.0);
    }
    // Image3::get_pixel (image.h:309-312) reads index z*X*Y + y*Y + x: the film's (x, y, z) when
    // X == Y, as the reference's own films are; the same index is read here
    double get_pixel(int x, int y, int z) const {
        if (x < 0 || x >= xres || y < 0 || y >= yres || z < 0 || z >= zres)
            throw py::index_error("get_pixel: coordinate out of range");
        return pixels[size_t(z) * xres * yres + size_t(y) * yres + x];
    }
};

// scn::Scene<TVector3> (renderer/include/scene.h:47-105) as the descriptors it amounts to
struct SMP_PYBIND_EXPORT Scene {
    std::string form;               // rif_analytical, rif_interpolated or rif_sources
    smp_scene_desc scene;
    smp_field_desc field;
    smp_host::Texture texture;
    std::vector<float> coeff;       // prefiltered spline coefficients (rif_interpolated)
    std::string distribution;       // final-angle importance sampling: carried, unused by the march
    float g_or_kappa = 0.0f;
    Scene() {
        std::memset(&scene, 0, sizeof(scene));
        std::memset(&field, 0, sizeof(field));
    }
};

inline float f32(py::handle h) { return py::cast<float>(h); }

inline Vec3f as_vec3(py::handle h) {
    if (py::isinstance<Vec3f>(h)) return py::cast<Vec3f>(h);
    py::sequence s = py::reinterpret_borrow<py::sequence>(h);
    if (s.size() != 3) throw py::type_error("expected a tvector_pybind.Vec3f or three numbers");
    Vec3f v;
    v.x = f32(s[0]); v.y = f32(s[1]); v.z = f32(s[2]);
    return v;
}
inline Vec2f as_vec2(py::handle h) {
    if (py::isinstance<Vec2f>(h)) return py::cast<Vec2f>(h);
    py::sequence s = py::reinterpret_borrow<py::sequence>(h);
    if (s.size() != 2) throw py::type_error("expected a tvector_pybind.Vec2f or two numbers");
    Vec2f v;
    v.x = f32(s[0]); v.y = f32(s[1]);
    return v;
}
inline void put3(double *dst, const Vec3f &v) { dst[0] = v.x; dst[1] = v.y; dst[2] = v.z; }
inline void put2(double *dst, const Vec2f &v) { dst[0] = v.x; dst[1] = v.y; }

[[noreturn]] inline void raise_smp(int rc, const char *what) {
    throw std::runtime_error(std::string(what) + ": simpler_b200 error " + std::to_string(rc) + ": " + smp_last_error());
}

}  // namespace smp_pybind
