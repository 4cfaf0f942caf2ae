// Shared definitions for the Otfwi B200 library: padded field layout, error
// recording and small helpers used by every translation unit.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

namespace otf {

// Every wavefield, coefficient and gradient array is stored padded: PAD zero
// cells on each side in z and at least PAD on each side in x, rows padded to a
// multiple of 32 floats so a row starts on a 128-byte boundary. Cells outside
// the reference's update region (4 <= x < X-4, 4 <= z < Z-4) hold zero for
// the whole run, which reproduces the reference's zero-masked tile loads
// (regression_PML_single.cu:488-498) without a per-tap bounds check.
constexpr int PAD = 8;
constexpr int NT = 256;  // threads per CTA of the stencil kernels

struct Layout {
    int X = 0, Z = 0;
    int pitch = 0;     // floats per padded row
    int rows = 0;      // Z + 2*PAD
    int64_t slot = 0;  // floats per padded field slot (rows * pitch)

    static Layout make(int X, int Z)
    {
        Layout L;
        L.X = X;
        L.Z = Z;
        L.pitch = ((X + 2 * PAD) + 31) / 32 * 32;
        L.rows = Z + 2 * PAD;
        L.slot = (int64_t)L.rows * L.pitch;
        return L;
    }
    __host__ __device__ int64_t at(int x, int z) const
    {
        return (int64_t)(z + PAD) * pitch + (x + PAD);
    }
};

// ---- error recording (the reference's C-ABI returns void; errors are kept
// here and exposed through otf_last_error / otf_last_status) -------------
void set_error(int code, const char *what, const char *file, int line);
void set_error_msg(int code, const std::string &msg);
void clear_error();
int last_status();
const char *last_error();

}  // namespace otf

#define OTF_CUDA(call)                                                        \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) {                                              \
            otf::set_error((int)e_, #call, __FILE__, __LINE__);               \
            return -1;                                                        \
        }                                                                     \
    } while (0)

#define OTF_CHECK(cond, code, msg)                                            \
    do {                                                                      \
        if (!(cond)) {                                                        \
            otf::set_error_msg((code), (msg));                                \
            return -1;                                                        \
        }                                                                     \
    } while (0)
