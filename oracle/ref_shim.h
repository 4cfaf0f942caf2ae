/*
 * Forced-include header for building the reference simulator into
 * oracle/_ref/ (test infrastructure; see oracle/Makefile).
 *
 * It changes no arithmetic and no call order of the reference. It only makes
 * two of the reference's latent memory errors harmless on a shared GPU:
 *
 *  1. Out-of-range reads. simulateFrameP/simulateFrameA read the damping
 *     arrays at d_x[z][x+1] and d_z[z+1][x] for every thread of the grid
 *     (regression_PML_single.cu:505-506, 592-593), i.e. up to one row past
 *     the end of d_z, and somaFrames/calcGrad2 touch cells past the array
 *     end when X or Z is not a multiple of 32 (:326, :443). Every device
 *     allocation is padded by 1 MiB so those accesses land in owned memory.
 *
 *  2. Copies through the never-allocated `initial` pointer
 *     (regression_PML_single.cu:146, 653-656). The copy is short-circuited
 *     with the error code the runtime reports for a null pointer, so no
 *     transfer is ever queued for address 0.
 */
#ifndef OTF_REF_SHIM_H
#define OTF_REF_SHIM_H
#include <cuda_runtime.h>

static inline cudaError_t otf_ref_padded_malloc(void **p, size_t n)
{
    return ::cudaMalloc(p, n + ((size_t)1 << 20));
}
template <class T>
static inline cudaError_t otf_ref_padded_malloc(T **p, size_t n)
{
    return otf_ref_padded_malloc(reinterpret_cast<void **>(p), n);
}
static inline cudaError_t otf_ref_checked_memcpy(void *d, const void *s, size_t n,
                                                 cudaMemcpyKind k)
{
    if (d == nullptr || s == nullptr)
        return cudaErrorInvalidValue;
    return ::cudaMemcpy(d, s, n, k);
}
#define cudaMalloc otf_ref_padded_malloc
#define cudaMemcpy otf_ref_checked_memcpy
#endif
