// photon_pybind -- the reference's photon module (renderer/pybindFiles/photon_pybind.cpp):
// Renderer(maxDepth, maxPathlength, useDirect, useAngularSampling, threads)
//     .renderImage(image_pybind.SmallImage, medium_pybind.Medium, scene_pybind.Scene, numPhotons)
// -- photon::Renderer::renderImage (renderer/src/photon.cpp:267-340) on the B200 kernels through
// smp_render, which overwrites every pixel of the image as the reference's merge of its per-thread
// images does. The film is written in place (no copy) and the GIL is released during the render.
// `threads` is accepted and unused (the render runs on one GPU); keyword-only extensions choose the
// device, the Philox seed (photon i draws stream (seed, i)), the film precision and the kernel.
#include "pybind_types.h"

using namespace smp_pybind;

namespace {

struct Renderer {
    int max_depth = -1;
    float max_pathlength = -1.0f;
    bool use_direct = false, use_angular_sampling = true;
    int threads = 0, device = 0, precision = SMP_PREC_FP32, kernel = SMP_KERNEL_POOL;
    unsigned long long seed = 0;
    smp_stats last{};

    void render_image(SmallImage &img, const Medium &md, const Scene &sc, long long n_photons) {
        smp_scene_desc s = sc.scene;
        s.x_res = img.xres;
        s.y_res = img.yres;
        s.z_res = img.zres;
        smp_medium_desc m;
        m.sigma_t = md.sigma_t;
        m.albedo = md.albedo;
        m.g = md.phase.g;
        smp_render_opts o;
        std::memset(&o, 0, sizeof(o));
        o.max_depth = max_depth;
        o.max_pathlength = max_pathlength;
        o.use_direct = use_direct ? 1 : 0;
        o.use_angular_sampling = use_angular_sampling ? 1 : 0;
        o.rng = SMP_RNG_PHILOX;
        o.precision = precision;
        o.device = device;
        o.seed = seed;
        o.kernel = kernel;
        smp_stats st{};
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = smp_render(&s, &m, &sc.field, &o, n_photons, img.pixels.data(), &st);
        }
        if (rc) raise_smp(rc, "renderImage");
        last = st;
    }
};

}  // namespace

PYBIND11_MODULE(photon_pybind, m) {
    m.doc() = "photon pybind module";
    py::module_::import("image_pybind");
    py::module_::import("medium_pybind");
    py::module_::import("scene_pybind");
    py::class_<Renderer>(m, "Renderer")
        .def(py::init([](int max_depth, float max_pathlength, bool use_direct, bool use_angular, long long threads,
                         int device, unsigned long long seed, int precision, int kernel) {
                 Renderer r;
                 r.max_depth = max_depth;
                 r.max_pathlength = max_pathlength;
                 r.use_direct = use_direct;
                 r.use_angular_sampling = use_angular;
                 r.threads = int(threads);
                 r.device = device;
                 r.seed = seed;
                 r.precision = precision;
                 r.kernel = kernel;
                 return r;
             }),
             py::arg("maxDepth"), py::arg("maxPathlength"), py::arg("useDirect"), py::arg("useAngularSampling"),
             py::arg("threads"), py::kw_only(), py::arg("device") = 0, py::arg("seed") = 0ULL,
             py::arg("precision") = int(SMP_PREC_FP32), py::arg("kernel") = int(SMP_KERNEL_POOL))
        .def("renderImage", &Renderer::render_image, py::arg("img"), py::arg("medium"), py::arg("scene"),
             py::arg("numPhotons"))
        // statistics of the last render: photons, ER steps, splats
        .def_property_readonly("last_stats", [](const Renderer &r) {
            py::dict d;
            d["photons"] = r.last.photons;
            d["er_steps"] = r.last.er_steps;
            d["splats"] = r.last.splats;
            d["kernel_ms"] = r.last.kernel_ms;
            return d;
        });
}
