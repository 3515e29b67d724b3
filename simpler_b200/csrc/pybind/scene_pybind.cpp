// scene_pybind -- the reference's scene module (renderer/pybindFiles/scene_pybind.cpp):
// Scene(<the positional arguments of renderer/include/scene.h:47-105>) and the ultrasound setters
// set_f_u, set_n_max, set_n_scaling, set_phase1, set_phase2 (scene.h:179-219).
//
// The reference compiles one constructor form per build (USE_RIF_SOURCES, USE_RIF_INTERPOLATED);
// this module takes each of them and tells them apart by argument count:
//   43 arguments: rif_analytical   (..., f_u, speed_u, n_o, n_max, n_clip, phi_min, phi_max, mode, ...)
//   44 arguments: rif_interpolated (the analytical form plus rifgridFile, a .vol grid, last)
//   53 arguments: rif_sources      (..., f_u, speed_u, n_o, n_scaling, n_coeff, radius, center1,
//                                   center2, active1, active2, phase1, phase2, theta_min, theta_max,
//                                   theta_sources, trans_z_min, trans_z_max, trans_z_sources, ...)
// Vectors are tvector_pybind.Vec3f / Vec2f (or plain sequences); every Float argument is rounded to
// single precision as the reference's Float build rounds it. The film resolution is not part of a
// Scene: photon_pybind.Renderer.renderImage takes it from the SmallImage it fills.
#include "pybind_types.h"

using namespace smp_pybind;

namespace {

const int kCommon = 25, kTail = 10;

std::unique_ptr<Scene> make_scene(const py::args &a) {
    const int n = int(a.size());
    auto sc = std::make_unique<Scene>();
    if (n == kCommon + 8 + kTail) sc->form = "rif_analytical";
    else if (n == kCommon + 8 + kTail + 1) sc->form = "rif_interpolated";
    else if (n == kCommon + 18 + kTail) sc->form = "rif_sources";
    else
        throw py::type_error("Scene: expected 43, 44 or 53 positional arguments (scene.h:47-105), got " +
                             std::to_string(n));
    smp_scene_desc &s = sc->scene;
    s.ior = f32(a[0]);
    put3(s.medium_l, as_vec3(a[1]));
    put3(s.medium_r, as_vec3(a[2]));
    put3(s.light_origin, as_vec3(a[3]));
    put3(s.light_dir, as_vec3(a[4]));
    s.half_theta_limit = f32(a[5]);
    std::string err;
    if (!smp_host::read_pfm_texture(py::cast<std::string>(a[6]), sc->texture, err)) throw std::runtime_error(err);
    put2(s.light_plane, as_vec2(a[7]));
    s.Li = f32(a[8]);
    put3(s.view_origin, as_vec3(a[9]));
    put3(s.view_dir, as_vec3(a[10]));
    put3(s.view_horizontal, as_vec3(a[11]));
    put2(s.view_plane, as_vec2(a[12]));
    put2(s.pathlength_range, as_vec2(a[13]));
    s.use_bounce_decomposition = py::cast<bool>(a[14]) ? 1 : 0;
    sc->distribution = py::cast<std::string>(a[15]);
    sc->g_or_kappa = f32(a[16]);
    put3(s.emitter_lens_origin, as_vec3(a[17]));
    s.emitter_lens_aperture = f32(a[18]);
    s.emitter_lens_focal_length = f32(a[19]);
    s.emitter_lens_active = py::cast<bool>(a[20]) ? 1 : 0;
    put3(s.sensor_lens_origin, as_vec3(a[21]));
    s.sensor_lens_aperture = f32(a[22]);
    s.sensor_lens_focal_length = f32(a[23]);
    s.sensor_lens_active = py::cast<bool>(a[24]) ? 1 : 0;
    s.tex_x = sc->texture.x;
    s.tex_y = sc->texture.y;
    s.texture = sc->texture.texels.data();

    smp_field_desc &f = sc->field;
    int t = kCommon;
    f.f_u = f32(a[t]);
    f.speed_u = f32(a[t + 1]);
    f.n_o = f32(a[t + 2]);
    if (sc->form == "rif_sources") {
        f.type = SMP_FIELD_SOURCES;
        f.n_scaling = f32(a[t + 3]);
        f.n_coeff = py::cast<int>(a[t + 4]);
        f.radius = f32(a[t + 5]);
        put3(f.center1, as_vec3(a[t + 6]));
        put3(f.center2, as_vec3(a[t + 7]));
        f.active1 = py::cast<bool>(a[t + 8]) ? 1 : 0;
        f.active2 = py::cast<bool>(a[t + 9]) ? 1 : 0;
        f.phase1 = f32(a[t + 10]);
        f.phase2 = f32(a[t + 11]);
        f.theta_min = f32(a[t + 12]);
        f.theta_max = f32(a[t + 13]);
        f.theta_sources = py::cast<int>(a[t + 14]);
        f.trans_z_min = f32(a[t + 15]);
        f.trans_z_max = f32(a[t + 16]);
        f.trans_z_sources = py::cast<int>(a[t + 17]);
        if (!(f.theta_max > f.theta_min)) throw py::value_error("Scene: theta_max must exceed theta_min");
        t += 18;
    } else {
        f.type = SMP_FIELD_BESSEL;
        f.n_max = f32(a[t + 3]);
        f.n_clip = f32(a[t + 4]);
        f.phi_min = f32(a[t + 5]);
        f.phi_max = f32(a[t + 6]);
        f.mode = py::cast<int>(a[t + 7]);
        t += 8;
    }
    // the ultrasound frame the kernels are built for (renderer3d_sample.cpp:839-841, rif_base.h:146-148)
    const Vec3f uz = as_vec3(a[t]), ux = as_vec3(a[t + 1]), pu = as_vec3(a[t + 2]);
    if (!(uz.x == -1.0f && uz.y == 0.0f && uz.z == 0.0f && ux.x == 0.0f && ux.y == 0.0f && ux.z == 1.0f &&
          pu.x == 0.0f && pu.y == 0.0f && pu.z == 0.0f))
        throw std::runtime_error("Scene: the ultrasound frame must be axis_uz=(-1,0,0), axis_ux=(0,0,1), p_u=(0,0,0)");
    f.er_stepsize = f32(a[t + 3]);
    f.direct_tol = f32(a[t + 4]);
    f.rr_weight = f32(a[t + 5]);
    f.precision = py::cast<int>(a[t + 6]);
    f.egap_end_x = f32(a[t + 7]);
    f.sgap_begin_x = f32(a[t + 8]);
    f.use_initialization_hack = py::cast<bool>(a[t + 9]) ? 1 : 0;
    if (sc->form == "rif_interpolated") {
        // rif_interpolated (rif_interpolated.h:46-104): the .vol grid, prefiltered as Spline<3>::build3d
        smp_host::Vol vol;
        if (!smp_host::read_vol(py::cast<std::string>(a[t + 10]), vol, err)) throw std::runtime_error(err);
        sc->coeff.assign(vol.data.size(), 0.0f);
        const int32_t dims[3] = {vol.n[0], vol.n[1], vol.n[2]};
        int rc = smp_spline_prefilter(vol.data.data(), dims, sc->coeff.data());
        if (rc) raise_smp(rc, "Scene: spline prefilter");
        f.type = SMP_FIELD_SPLINE;
        for (int i = 0; i < 3; ++i) {
            f.grid_n[i] = vol.n[i];
            f.grid_min[i] = vol.min[i];
            f.grid_max[i] = vol.max[i];
        }
        f.grid_coeff = sc->coeff.data();
    }
    return sc;
}

py::tuple descriptors(const Scene &sc) {
    return py::make_tuple(py::bytes(reinterpret_cast<const char *>(&sc.scene), sizeof(sc.scene)),
                          py::bytes(reinterpret_cast<const char *>(&sc.field), sizeof(sc.field)));
}

}  // namespace

PYBIND11_MODULE(scene_pybind, m) {
    m.doc() = "scene pybind module";
    py::module_::import("tvector_pybind");
    py::class_<Scene>(m, "Scene")
        .def(py::init([](const py::args &a) { return make_scene(a); }))
        // setters (scene.h:179-219); k = 2 pi f_u / speed_u follows f_u as rif_base.h:144-154 derives it
        .def("set_f_u", [](Scene &s, float v) { s.field.f_u = v; })
        .def("set_n_max", [](Scene &s, float v) { s.field.n_max = v; })
        .def("set_n_scaling", [](Scene &s, float v) { s.field.n_scaling = v; })
        .def("set_phase1", [](Scene &s, float v) { s.field.phase1 = v; })
        .def("set_phase2", [](Scene &s, float v) { s.field.phase2 = v; })
        .def("getUSFrequency", [](const Scene &s) { return s.field.f_u; })
        .def_readonly("form", &Scene::form)
        // the texture as rows after the PFM flip (texel y * X + x), and the C-ABI descriptors as bytes
        // (smp_scene_desc, smp_field_desc; their pointers are this Scene's own buffers)
        .def_property_readonly("texture", [](py::object self) {
            Scene &s = self.cast<Scene &>();
            const py::ssize_t d = sizeof(double);
            return py::array_t<double>({py::ssize_t(s.texture.y), py::ssize_t(s.texture.x)}, {d * s.texture.x, d},
                                       s.texture.texels.data(), self);
        })
        .def("descriptors", &descriptors);
}
