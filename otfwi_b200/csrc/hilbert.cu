// hilbert(): the analytic-signal routine the reference links into its
// simulator library (simulator/src/hilbert.cpp:15-79). The reference runs a
// float cuFFT C2C forward transform, zeroes spectrum indices
// [N/2, N/2 + N/2), transforms back (unnormalised) and returns
// signal90 = 2*Im(y)/N and envelope = 2*|y|/N. Here the kept-band transform
// pair is evaluated directly in FP64 (one thread per output bin), which is
// exact to FP32 output precision for the trace lengths this library handles.
#include <cuda_runtime.h>
#include <cmath>
#include "otf_common.cuh"
#include "../../include/otfwi.h"

namespace {

// forward DFT of the kept bins: spec[k] = sum_m x[m] exp(-2 pi i k m / N)
__global__ void k_dft_kept(const float *__restrict__ x, double2 *__restrict__ spec, int N, int half)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N)
        return;
    const bool kept = k < half || k >= 2 * half;
    double re = 0.0, im = 0.0;
    if (kept) {
        for (int m = 0; m < N; m++) {
            const long long km = ((long long)k * m) % N;
            double s, c;
            sincospi(2.0 * (double)km / (double)N, &s, &c);
            re += (double)x[m] * c;
            im -= (double)x[m] * s;
        }
    }
    spec[k] = make_double2(re, im);
}

// inverse (unnormalised) transform and the reference's output scaling
__global__ void k_idft_out(const double2 *__restrict__ spec, float *__restrict__ s90,
                           float *__restrict__ env, int N)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N)
        return;
    double re = 0.0, im = 0.0;
    for (int k = 0; k < N; k++) {
        const long long kn = ((long long)k * n) % N;
        double s, c;
        sincospi(2.0 * (double)kn / (double)N, &s, &c);
        re += spec[k].x * c - spec[k].y * s;
        im += spec[k].x * s + spec[k].y * c;
    }
    s90[n] = (float)(2.0 * im / N);
    env[n] = (float)(2.0 * sqrt(re * re + im * im) / N);
}

}  // namespace

extern "C" void hilbert(float *signal, float *signal90, float *envelope, int N)
{
    if (N <= 0 || !signal || !signal90 || !envelope) {
        otf::set_error_msg(1, "hilbert: invalid arguments");
        return;
    }
    float *dx = nullptr, *ds = nullptr, *de = nullptr;
    double2 *spec = nullptr;
    auto fail = [&](cudaError_t e) {
        otf::set_error((int)e, "hilbert", __FILE__, __LINE__);
    };
    cudaError_t e;
    if ((e = cudaMalloc(&dx, sizeof(float) * N)) != cudaSuccess ||
        (e = cudaMalloc(&ds, sizeof(float) * N)) != cudaSuccess ||
        (e = cudaMalloc(&de, sizeof(float) * N)) != cudaSuccess ||
        (e = cudaMalloc(&spec, sizeof(double2) * N)) != cudaSuccess) {
        fail(e);
    } else if ((e = cudaMemcpy(dx, signal, sizeof(float) * N, cudaMemcpyHostToDevice)) != cudaSuccess) {
        fail(e);
    } else {
        const int b = 128, g = (N + b - 1) / b;
        k_dft_kept<<<g, b>>>(dx, spec, N, N / 2);
        k_idft_out<<<g, b>>>(spec, ds, de, N);
        if ((e = cudaGetLastError()) != cudaSuccess ||
            (e = cudaMemcpy(signal90, ds, sizeof(float) * N, cudaMemcpyDeviceToHost)) != cudaSuccess ||
            (e = cudaMemcpy(envelope, de, sizeof(float) * N, cudaMemcpyDeviceToHost)) != cudaSuccess)
            fail(e);
    }
    cudaFree(dx);
    cudaFree(ds);
    cudaFree(de);
    cudaFree(spec);
}
