// plain.cuh -- the plain GPU kernel: one thread per photon, launched once over all photons.
//
// This is the structure of the reference's own GPU renderer (renderer/src/cuda_renderer.cu:681-708
// `renderPhotons`, launched at :713-725 with one thread per photon in 16 x 16 blocks): every thread
// traces its photon from genRay to termination, with no persistence, no regeneration of finished
// lanes and no separation of the march from the discrete logic, and splats with plain atomics. Its
// per-photon arithmetic is this library's own (march_step, run_events), so its photons and films are
// those of the slot-pool path; the difference between the two is scheduling alone. It is the
// denominator of the speed-up the production paths are measured against, and a renderer in its own
// right (smp_render_opts.kernel = SMP_KERNEL_PLAIN).
#pragma once
#include "march.cuh"

namespace smp {

static constexpr int kPlainBlock = 256;      // the reference's dim3(16, 16)

template <int FK>
__global__ void __launch_bounds__(kPlainBlock) plain_kernel(const __grid_constant__ KParams P) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    LaneStats S;
    if (t < P.n_photons) {
        Lane L;
        L.idx = P.first_photon + t;
        L.end = 0;
        L.inst = nullptr;
        L.tab = P.field.btab;                 // the Bessel table read from global memory
        int st = run_events<FK>(L, P, EV_NEW);
        while (st == ST_MARCH) {
            while (!march_step<FK>(L, P)) {
            }
            st = run_events<FK>(L, P, EV_MARCH_END);
        }
        finish_photon_stats<FK>(L, S);
    }
    flush_stats(S, P, lane);
}

}  // namespace smp
