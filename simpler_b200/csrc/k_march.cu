// k_march.cu -- the persistent lane-loop kernel (march.cuh), the plain one-thread-per-photon kernel
// (plain.cuh) and the field probe, instantiated per field kind.
#include <cuda_runtime.h>

#include "dispatch.h"
#include "march.cuh"
#include "plain.cuh"

namespace smp {

MarchFn march_fn(int fk) {
    switch (fk) {
        case FK_BESSEL0: return march_kernel<FK_BESSEL0>;
        case FK_BESSEL1: return march_kernel<FK_BESSEL1>;
        case FK_BESSEL2: return march_kernel<FK_BESSEL2>;
        case FK_BESSELN: return march_kernel<FK_BESSELN>;
        case FK_PLANEWAVE: return march_kernel<FK_PLANEWAVE>;
        case FK_SOURCES: return march_kernel<FK_SOURCES>;
        case FK_SPLINE: return march_kernel<FK_SPLINE>;
        case FK_BATCH: return march_kernel<FK_BATCH>;
        default: return nullptr;
    }
}

MarchFn plain_fn(int fk) {
    switch (fk) {
        case FK_BESSEL0: return plain_kernel<FK_BESSEL0>;
        case FK_BESSEL1: return plain_kernel<FK_BESSEL1>;
        case FK_BESSEL2: return plain_kernel<FK_BESSEL2>;
        case FK_BESSELN: return plain_kernel<FK_BESSELN>;
        case FK_PLANEWAVE: return plain_kernel<FK_PLANEWAVE>;
        case FK_SOURCES: return plain_kernel<FK_SOURCES>;
        case FK_SPLINE: return plain_kernel<FK_SPLINE>;
        default: return nullptr;
    }
}

ProbeFn field_probe_fn(int fk) {
    switch (fk) {
        case FK_BESSEL0: return field_probe_kernel<FK_BESSEL0>;
        case FK_BESSEL1: return field_probe_kernel<FK_BESSEL1>;
        case FK_BESSEL2: return field_probe_kernel<FK_BESSEL2>;
        case FK_BESSELN: return field_probe_kernel<FK_BESSELN>;
        case FK_PLANEWAVE: return field_probe_kernel<FK_PLANEWAVE>;
        case FK_SOURCES: return field_probe_kernel<FK_SOURCES>;
        case FK_SPLINE: return field_probe_kernel<FK_SPLINE>;
        default: return nullptr;
    }
}

}  // namespace smp
