// k_wave.cu -- the slot-pool kernels (wavefront.cuh): march (blocks of 128 or 256 threads, FP32 or
// FP64 path length), event and tail kernels, instantiated per field kind.
#include <cuda_runtime.h>

#include "dispatch.h"
#include "wavefront.cuh"

namespace smp {

template <int B>
static WaveFn wf_march_fn_b(int fk, bool fp64) {
    switch (fk) {
        case FK_BESSEL0: return fp64 ? wf_march_kernel<FK_BESSEL0, 1, B> : wf_march_kernel<FK_BESSEL0, 0, B>;
        case FK_BESSEL1: return fp64 ? wf_march_kernel<FK_BESSEL1, 1, B> : wf_march_kernel<FK_BESSEL1, 0, B>;
        case FK_BESSEL2: return fp64 ? wf_march_kernel<FK_BESSEL2, 1, B> : wf_march_kernel<FK_BESSEL2, 0, B>;
        case FK_BESSELN: return fp64 ? wf_march_kernel<FK_BESSELN, 1, B> : wf_march_kernel<FK_BESSELN, 0, B>;
        case FK_PLANEWAVE: return fp64 ? wf_march_kernel<FK_PLANEWAVE, 1, B> : wf_march_kernel<FK_PLANEWAVE, 0, B>;
        case FK_SOURCES: return fp64 ? wf_march_kernel<FK_SOURCES, 1, B> : wf_march_kernel<FK_SOURCES, 0, B>;
        case FK_SPLINE: return fp64 ? wf_march_kernel<FK_SPLINE, 1, B> : wf_march_kernel<FK_SPLINE, 0, B>;
        case FK_BATCH: return fp64 ? wf_march_kernel<FK_BATCH, 1, B> : wf_march_kernel<FK_BATCH, 0, B>;
        default: return nullptr;
    }
}

WaveFn wf_march_fn(int fk, bool fp64, int block, bool bricks) {
    if (fk == FK_SPLINE && bricks) {
        if (block == 256) return fp64 ? wf_march_spline_kernel<1, 256> : wf_march_spline_kernel<0, 256>;
        return fp64 ? wf_march_spline_kernel<1, 128> : wf_march_spline_kernel<0, 128>;
    }
    return block == 256 ? wf_march_fn_b<256>(fk, fp64) : wf_march_fn_b<128>(fk, fp64);
}

WaveFn wf_event_fn(int fk) {
    switch (fk) {
        case FK_BESSEL0: return wf_event_kernel<FK_BESSEL0>;
        case FK_BESSEL1: return wf_event_kernel<FK_BESSEL1>;
        case FK_BESSEL2: return wf_event_kernel<FK_BESSEL2>;
        case FK_BESSELN: return wf_event_kernel<FK_BESSELN>;
        case FK_PLANEWAVE: return wf_event_kernel<FK_PLANEWAVE>;
        case FK_SOURCES: return wf_event_kernel<FK_SOURCES>;
        case FK_SPLINE: return wf_event_kernel<FK_SPLINE>;
        case FK_BATCH: return wf_event_kernel<FK_BATCH>;
        default: return nullptr;
    }
}

WaveFn wf_finish_fn(int fk) {
    switch (fk) {
        case FK_BESSEL0: return wf_finish_kernel<FK_BESSEL0>;
        case FK_BESSEL1: return wf_finish_kernel<FK_BESSEL1>;
        case FK_BESSEL2: return wf_finish_kernel<FK_BESSEL2>;
        case FK_BESSELN: return wf_finish_kernel<FK_BESSELN>;
        case FK_PLANEWAVE: return wf_finish_kernel<FK_PLANEWAVE>;
        case FK_SOURCES: return wf_finish_kernel<FK_SOURCES>;
        case FK_SPLINE: return wf_finish_kernel<FK_SPLINE>;
        case FK_BATCH: return wf_finish_kernel<FK_BATCH>;
        default: return nullptr;
    }
}

}  // namespace smp
