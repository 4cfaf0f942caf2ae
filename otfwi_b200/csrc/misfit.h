// Device trace misfits (see misfit.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace otf {

enum MisfitKind : int {
    kMisfitL2 = 0,
    kMisfitWasserstein = 1,
    kMisfitWassersteinSoftplus = 2,
    kMisfitWassersteinQuad = 3
};
constexpr int kNumMisfits = 4;

// Bytes of global scratch one trace needs (0 for L2).
int64_t misfit_scratch_per_trace(int kind, int T);

// sim, obs, adj: device [n_traces][T]; misfit: device [n_traces] (FP64).
int launch_misfit(int kind, const float *sim, const float *obs, float *adj, double *misfit,
                  int n_traces, int T, void *scratch, int64_t scratch_bytes, cudaStream_t st);

}  // namespace otf
