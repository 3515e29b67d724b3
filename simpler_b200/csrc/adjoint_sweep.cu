// adjoint_sweep.cu -- the adjoint's backward-sweep kernel in a translation unit of its own, compiled
// with a*b+c contraction (every other kernel is compiled without it, so that the render's two march
// paths and the adjoint's replays of them reproduce the same photons bit for bit; the sweep only
// reads what the replays recorded).
#include <cuda_runtime.h>

#include "adjoint.cuh"

namespace smp {

// Resident blocks per SM: 4 (128 registers) where the kernel fits without spilling much (Bessel,
// plane waves of at most two waves: 20-25 % faster than 3), 3 for the spline and the eight-wave
// instance, whose spills at 128 registers cost what the occupancy gains.
AdjRoundFn adjoint_sweep_fn(int fk, int n_waves) {
    switch (fk) {
        case FK_BESSEL0: return adjoint_sweep_kernel<FK_BESSEL0, SMP_MAX_WAVES, 4>;
        case FK_BESSEL1: return adjoint_sweep_kernel<FK_BESSEL1, SMP_MAX_WAVES, 4>;
        case FK_BESSEL2: return adjoint_sweep_kernel<FK_BESSEL2, SMP_MAX_WAVES, 4>;
        case FK_PLANEWAVE:
            return n_waves <= 2 ? adjoint_sweep_kernel<FK_PLANEWAVE, 2, 4> : adjoint_sweep_kernel<FK_PLANEWAVE, SMP_MAX_WAVES, 3>;
        case FK_SPLINE: return adjoint_sweep_kernel<FK_SPLINE, SMP_MAX_WAVES, 3>;
        default: return nullptr;
    }
}

}  // namespace smp
