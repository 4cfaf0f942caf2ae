// quad_envelope misfit (ref:adjoint_functions.py:14-22) on the device:
//   H x   = analytic signal (scipy.signal.hilbert: FFT, one-sided weights
//           h[0] = 1, 2 on positive frequencies, h[N/2] = 1 for even N, 0 on
//           negative ones, inverse FFT)
//   e     = |H sim|^2 - |H obs|^2,   misfit = sum e^2
//   adj   = sim * e - Im(H(e * Im(H sim)))
// Per trace, in FP64: three batched complex FFT pairs (cuFFT Z2Z) and four
// small kernels. The FFT plans are created by envelope_prepare, outside any
// stream capture (plan creation allocates).
#include <cufft.h>
#include <cuda_runtime.h>
#include <map>
#include <utility>
#include "misfit.h"
#include "otf_common.cuh"

namespace otf {

namespace {

std::map<std::pair<int, int>, cufftHandle> &plans()
{
    static std::map<std::pair<int, int>, cufftHandle> p;
    return p;
}

int plan_for(int n, int T, cufftHandle *out)
{
    auto &m = plans();
    auto it = m.find({n, T});
    if (it != m.end()) {
        *out = it->second;
        return 0;
    }
    cufftHandle h;
    int len = T;
    if (cufftPlanMany(&h, 1, &len, nullptr, 1, T, nullptr, 1, T, CUFFT_Z2Z, n) != CUFFT_SUCCESS) {
        set_error_msg(3, "quad_envelope: cuFFT plan creation failed");
        return -1;
    }
    m[{n, T}] = h;
    *out = h;
    return 0;
}

// real input -> complex [n][T]
__global__ void k_env_load(const float *__restrict__ x, cufftDoubleComplex *__restrict__ z, int64_t total)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < total)
        z[i] = make_cuDoubleComplex((double)x[i], 0.0);
}

// one-sided spectrum weights, with the inverse FFT's 1/T folded in
__global__ void k_env_weights(cufftDoubleComplex *__restrict__ z, int T, int64_t total)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total)
        return;
    const int k = (int)(i % T);
    double h;
    if (k == 0 || (T % 2 == 0 && k == T / 2))
        h = 1.0;
    else if (k < (T + 1) / 2)
        h = 2.0;
    else
        h = 0.0;
    h /= (double)T;
    z[i] = make_cuDoubleComplex(z[i].x * h, z[i].y * h);
}

// e = |H sim|^2 - |H obs|^2 into e; the third transform's input e * Im(H sim)
// into c; per-trace sum of e^2 (one block per trace)
__global__ void __launch_bounds__(256) k_env_energy(const cufftDoubleComplex *__restrict__ hs,
                                                    const cufftDoubleComplex *__restrict__ ho,
                                                    double *__restrict__ e, cufftDoubleComplex *__restrict__ c,
                                                    double *__restrict__ misfit, int T)
{
    __shared__ double red[8];
    const int64_t base = (int64_t)blockIdx.x * T;
    double s = 0.0;
    for (int k = threadIdx.x; k < T; k += blockDim.x) {
        const cufftDoubleComplex a = hs[base + k], b = ho[base + k];
        const double v = (a.x * a.x + a.y * a.y) - (b.x * b.x + b.y * b.y);
        e[base + k] = v;
        c[base + k] = make_cuDoubleComplex(v * a.y, 0.0);
        s += v * v;
    }
    for (int o = 16; o > 0; o >>= 1)
        s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0)
        red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < 8; k++)
            t += red[k];
        misfit[blockIdx.x] = t;
    }
}

// adj = sim * e - Im(H c)
__global__ void k_env_adjoint(const float *__restrict__ sim, const double *__restrict__ e,
                              const cufftDoubleComplex *__restrict__ hc, float *__restrict__ adj, int64_t total)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < total)
        adj[i] = (float)((double)sim[i] * e[i] - hc[i].y);
}

}  // namespace

int64_t envelope_scratch_per_trace(int T)
{
    // three complex FP64 signals and the FP64 envelope difference
    const int64_t bytes = (int64_t)T * (3 * (int64_t)sizeof(cufftDoubleComplex) + (int64_t)sizeof(double));
    return (bytes + 255) / 256 * 256;
}

int envelope_prepare(int n_traces, int T)
{
    cufftHandle h;
    return n_traces > 0 ? plan_for(n_traces, T, &h) : 0;
}

int launch_envelope(const float *sim, const float *obs, float *adj, double *misfit, int n, int T, void *scratch,
                    cudaStream_t st)
{
    cufftHandle plan;
    if (plan_for(n, T, &plan))
        return -1;
    OTF_CHECK(cufftSetStream(plan, st) == CUFFT_SUCCESS, 3, "quad_envelope: cufftSetStream failed");
    const int64_t total = (int64_t)n * T;
    // scratch layout: A | B | C (complex [n][T]) | e (double [n][T]); the
    // per-trace blocks of the misfit scratch are reinterpreted as these arrays
    cufftDoubleComplex *A = reinterpret_cast<cufftDoubleComplex *>(scratch);
    cufftDoubleComplex *B = A + total, *C = B + total;
    double *e = reinterpret_cast<double *>(C + total);
    const unsigned nb = (unsigned)((total + 255) / 256);
    k_env_load<<<nb, 256, 0, st>>>(sim, A, total);
    k_env_load<<<nb, 256, 0, st>>>(obs, B, total);
    for (cufftDoubleComplex *z : {A, B}) {
        OTF_CHECK(cufftExecZ2Z(plan, z, z, CUFFT_FORWARD) == CUFFT_SUCCESS, 3, "quad_envelope: FFT failed");
        k_env_weights<<<nb, 256, 0, st>>>(z, T, total);
        OTF_CHECK(cufftExecZ2Z(plan, z, z, CUFFT_INVERSE) == CUFFT_SUCCESS, 3, "quad_envelope: FFT failed");
    }
    k_env_energy<<<n, 256, 0, st>>>(A, B, e, C, misfit, T);
    OTF_CHECK(cufftExecZ2Z(plan, C, C, CUFFT_FORWARD) == CUFFT_SUCCESS, 3, "quad_envelope: FFT failed");
    k_env_weights<<<nb, 256, 0, st>>>(C, T, total);
    OTF_CHECK(cufftExecZ2Z(plan, C, C, CUFFT_INVERSE) == CUFFT_SUCCESS, 3, "quad_envelope: FFT failed");
    k_env_adjoint<<<nb, 256, 0, st>>>(sim, e, C, adj, total);
    OTF_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace otf
