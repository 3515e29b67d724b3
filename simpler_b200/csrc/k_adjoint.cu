// k_adjoint.cu -- the adjoint's checkpointing-trace and segment-replay kernels (adjoint.cuh),
// instantiated per field kind; the backward sweep is in adjoint_sweep.cu.
#include <cuda_runtime.h>

#include "adjoint.cuh"
#include "dispatch.h"

namespace smp {

AdjFn adjoint_trace_fn(int fk) {
    switch (fk) {
        case FK_BESSEL0: return adjoint_trace_kernel<FK_BESSEL0>;
        case FK_BESSEL1: return adjoint_trace_kernel<FK_BESSEL1>;
        case FK_BESSEL2: return adjoint_trace_kernel<FK_BESSEL2>;
        case FK_PLANEWAVE: return adjoint_trace_kernel<FK_PLANEWAVE>;
        case FK_SPLINE: return adjoint_trace_kernel<FK_SPLINE>;
        default: return nullptr;
    }
}

AdjRoundFn adjoint_replay_fn(int fk) {
    switch (fk) {
        case FK_BESSEL0: return adjoint_replay_kernel<FK_BESSEL0>;
        case FK_BESSEL1: return adjoint_replay_kernel<FK_BESSEL1>;
        case FK_BESSEL2: return adjoint_replay_kernel<FK_BESSEL2>;
        case FK_PLANEWAVE: return adjoint_replay_kernel<FK_PLANEWAVE>;
        case FK_SPLINE: return adjoint_replay_kernel<FK_SPLINE>;
        default: return nullptr;
    }
}

}  // namespace smp
