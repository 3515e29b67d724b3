// adjoint_sweep.cu -- the adjoint's backward-sweep kernel in a translation unit of its own, compiled
// with a*b+c contraction (every other kernel is compiled without it, so that the render's two march
// paths and the adjoint's replays of them reproduce the same photons bit for bit; the sweep only
// reads what the replays recorded).
#include <cuda_runtime.h>

#include "adjoint.cuh"

namespace smp {

AdjRoundFn adjoint_sweep_fn(int fk) {
    switch (fk) {
        case FK_BESSEL0: return adjoint_sweep_kernel<FK_BESSEL0>;
        case FK_BESSEL1: return adjoint_sweep_kernel<FK_BESSEL1>;
        case FK_BESSEL2: return adjoint_sweep_kernel<FK_BESSEL2>;
        case FK_PLANEWAVE: return adjoint_sweep_kernel<FK_PLANEWAVE>;
        case FK_SPLINE: return adjoint_sweep_kernel<FK_SPLINE>;
        default: return nullptr;
    }
}

}  // namespace smp
