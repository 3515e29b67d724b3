// dispatch.h -- the kernels of the library, compiled in translation units of their own (k_march.cu,
// k_wave.cu, k_adjoint.cu, adjoint_sweep.cu) so that they build in parallel, and handed to the host
// code in capi.cu as function pointers per field kind.
#pragma once
#include <cuda_runtime.h>

#include "kparams.h"

namespace smp {

struct WaveParams;
struct AdjParams;

typedef void (*MarchFn)(KParams);
typedef void (*WaveFn)(KParams, WaveParams, int);
typedef void (*ProbeFn)(FieldParams, float, long long, const double *, double *, double *);
typedef void (*AdjFn)(KParams, AdjParams);
typedef void (*AdjRoundFn)(KParams, AdjParams, int);
typedef void (*AdjWaveFn)(KParams, WaveParams, AdjParams, int);

// k_march.cu
MarchFn march_fn(int fk);                        // persistent lane loop (march.cuh)
MarchFn plain_fn(int fk);                        // one thread per photon (plain.cuh)
ProbeFn field_probe_fn(int fk);                  // field at host-given points
// k_wave.cu: the slot pool (wavefront.cuh); the march kernel in blocks of 128 or 256 threads; for a
// spline plan with TMA-staged coefficient bricks (smp_render_opts.spline_bricks) the brick kernel
WaveFn wf_march_fn(int fk, bool fp64, int block, bool bricks);
WaveFn wf_event_fn(int fk);
WaveFn wf_finish_fn(int fk);
// k_adjoint.cu, adjoint_sweep.cu
AdjFn adjoint_trace_fn(int fk);                  // the trace on the persistent lane loop
AdjWaveFn adjoint_trace_event_fn(int fk);        // the trace on the slot pool: event and tail kernels
AdjWaveFn adjoint_trace_finish_fn(int fk);
AdjRoundFn adjoint_replay_fn(int fk);
AdjRoundFn adjoint_sweep_fn(int fk, int n_waves);    // n_waves: of a plane-wave field
// the batch's photons in the order replays and sweeps take them (A.order, *A.n_order)
cudaError_t adjoint_order(const AdjParams &A, long long n, int grid, cudaStream_t s);

}  // namespace smp
