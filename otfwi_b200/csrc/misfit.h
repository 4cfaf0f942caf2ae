// Device trace misfits (see misfit.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace otf {

enum MisfitKind : int {
    kMisfitL2 = 0,
    kMisfitWasserstein = 1,
    kMisfitWassersteinSoftplus = 2,
    kMisfitWassersteinQuad = 3,
    kMisfitQuadEnvelope = 4,
    kMisfitWassersteinPM = 5
};
constexpr int kNumMisfits = 6;

// quad_envelope (envelope.cu): FFT plans are created by envelope_prepare,
// which must run outside stream capture (plan creation allocates).
int64_t envelope_scratch_per_trace(int T);
int envelope_prepare(int n_traces, int T);
int launch_envelope(const float *sim, const float *obs, float *adj, double *misfit, int n, int T, void *scratch,
                    cudaStream_t st);

// Bytes of global scratch one trace needs (0 for L2).
int64_t misfit_scratch_per_trace(int kind, int T);

// sim, obs, adj: device [n_traces][T]; misfit: device [n_traces] (FP64).
int launch_misfit(int kind, const float *sim, const float *obs, float *adj, double *misfit,
                  int n_traces, int T, void *scratch, int64_t scratch_bytes, cudaStream_t st);

}  // namespace otf
