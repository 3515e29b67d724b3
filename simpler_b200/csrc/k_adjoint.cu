// k_adjoint.cu -- the adjoint's checkpointing-trace kernels (on the slot pool, and on the persistent
// lane loop) and segment-replay kernel (adjoint.cuh), instantiated per field kind, and the kernels
// that order a batch's photons for the replays and sweeps; the backward sweep is in adjoint_sweep.cu.
#include <cuda_runtime.h>

#include "adjoint.cuh"
#include "dispatch.h"

namespace smp {

// ---- the order in which replays and sweeps take the batch's photons ----------------------------
// A counting sort of the photons the sweep needs (differentiated, some splat reaching dJ/dfilm) by
// their trajectory length, longest first, into kOrderBuckets buckets 64 per octave wide: lanes of
// one warp then march and sweep photons of about equal length, instead of waiting for the longest
// of 32 random ones. Within a bucket the order is that of the atomics.
constexpr int kOrderBuckets = 1024;
__device__ __forceinline__ int order_bucket(int tlen) {
    // 64 buckets per octave of tlen + 1, the top one open-ended (tlen above 2^16)
    const float l = __log2f(float(tlen) + 1.0f);
    return min(kOrderBuckets - 1, int(l * 64.0f));
}
__device__ __forceinline__ bool order_needed(const AdjPhoton &r) { return r.status == PH_OK && r.hits != 0; }

__global__ void adjoint_order_count(const __grid_constant__ AdjParams A, long long n) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const AdjPhoton &r = A.photons[k];
        if (order_needed(r)) atomicAdd(A.obucket + order_bucket(r.tlen), 1u);
    }
}

// one block of kOrderBuckets threads: bucket counts -> first position of each bucket, highest first
__global__ void __launch_bounds__(kOrderBuckets) adjoint_order_scan(const __grid_constant__ AdjParams A) {
    __shared__ unsigned v[kOrderBuckets];
    const int t = threadIdx.x;
    const unsigned own = A.obucket[kOrderBuckets - 1 - t];
    v[t] = own;
    __syncthreads();
    for (int o = 1; o < kOrderBuckets; o <<= 1) {
        const unsigned x = t >= o ? v[t - o] : 0u;
        __syncthreads();
        v[t] += x;
        __syncthreads();
    }
    A.obucket[kOrderBuckets - 1 - t] = v[t] - own;       // exclusive
    if (t == kOrderBuckets - 1) *A.n_order = v[t];
}

__global__ void adjoint_order_scatter(const __grid_constant__ AdjParams A, long long n) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const AdjPhoton &r = A.photons[k];
        if (order_needed(r)) A.order[atomicAdd(A.obucket + order_bucket(r.tlen), 1u)] = int(k);
    }
}


// Fills A.order / *A.n_order for photons [0, n) of the batch (kernels above, on stream s).
cudaError_t adjoint_order(const AdjParams &A, long long n, int grid, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(A.obucket, 0, kOrderBuckets * sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    adjoint_order_count<<<grid, 256, 0, s>>>(A, n);
    adjoint_order_scan<<<1, kOrderBuckets, 0, s>>>(A);
    adjoint_order_scatter<<<grid, 256, 0, s>>>(A, n);
    return cudaGetLastError();
}

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

AdjWaveFn adjoint_trace_event_fn(int fk) {
    switch (fk) {
        case FK_BESSEL0: return adjoint_trace_event_kernel<FK_BESSEL0>;
        case FK_BESSEL1: return adjoint_trace_event_kernel<FK_BESSEL1>;
        case FK_BESSEL2: return adjoint_trace_event_kernel<FK_BESSEL2>;
        case FK_PLANEWAVE: return adjoint_trace_event_kernel<FK_PLANEWAVE>;
        case FK_SPLINE: return adjoint_trace_event_kernel<FK_SPLINE>;
        default: return nullptr;
    }
}

AdjWaveFn adjoint_trace_finish_fn(int fk) {
    switch (fk) {
        case FK_BESSEL0: return adjoint_trace_finish_kernel<FK_BESSEL0>;
        case FK_BESSEL1: return adjoint_trace_finish_kernel<FK_BESSEL1>;
        case FK_BESSEL2: return adjoint_trace_finish_kernel<FK_BESSEL2>;
        case FK_PLANEWAVE: return adjoint_trace_finish_kernel<FK_PLANEWAVE>;
        case FK_SPLINE: return adjoint_trace_finish_kernel<FK_SPLINE>;
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
