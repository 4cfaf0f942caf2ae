/*
 * CPU oracle for the split-field PML forward / adjoint-gradient hot path.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker the parity tests, smoke()
 * and bench.py's cpu_baseline leg compare against. The product (the CUDA
 * library under otfwi_b200/) never loads it.
 *
 * It restates the reference's regression_PML_single.cu / deriv_macros.h in
 * plain C (see pml_oracle_body.h for the per-function citations), in two
 * modes built from one body:
 *   *_f32: bit-level restatement of the reference's arithmetic
 *          (FP32 fields, FP64 staggered tap sums, FP32 fused updates);
 *   *_f64: the same algorithm in FP64 throughout (the "FP64 host oracle").
 * Build: see oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* deriv_macros.h:85-95 coefficients, as the reference's double literals */
#define ORC_C0 1.196289e+00
#define ORC_C1 7.975260e-02
#define ORC_C2 9.570313e-03
#define ORC_C3 6.975446e-04

#define ORC_REAL float
#define ORC_SUF f32
#define ORC_IS_F32 1
#include "pml_oracle_body.h"
#undef ORC_REAL
#undef ORC_SUF
#undef ORC_IS_F32

#define ORC_REAL double
#define ORC_SUF f64
#define ORC_IS_F32 0
#include "pml_oracle_body.h"
#undef ORC_REAL
#undef ORC_SUF
#undef ORC_IS_F32

/* Number of OpenMP threads the oracle runs with (reported as "cores"). */
int orc_num_threads(void)
{
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Video frames of cuda_simulate(en_out = 1) (regression_PML_single.cu:
 * 660-687): after every `every`-th step t, P = Px + Pz of slot t
 * (somaFrames, :312-327) is mapped as writeFramePipe does (utils.cu:94-113):
 * min and max over the grid, offset = -min, scale = 255 / (max - min) in
 * FP32, byte = (P + offset) * scale converted to unsigned char, receivers
 * set to 255. frames [n_frames][Z][X] with n_frames = (T-1)/every; p_out
 * (optional) receives the FP32 P of every frame. */
int orc_frames_f32(int X, int Z, int T, const float *cquad, const float *constvec, const float *d_x,
                   const float *d_z, int ns, const int *sx, const int *sz, const float *src, int idx_source,
                   int nm, const int *mx, const int *mz, int every, unsigned char *frames, float *p_out)
{
    orc_fields_f32 F;
    if (every < 1 || alloc_fields_f32(&F, X, Z, T))
        return -1;
    float *integ = (float *)calloc(ns > 0 ? ns : 1, sizeof(float));
    float *rec = (float *)calloc((size_t)(nm > 0 ? nm : 1) * T, sizeof(float));
    float *img = (float *)malloc(sizeof(float) * (size_t)X * Z);
    if (!integ || !rec || !img)
        return -1;
    const size_t XZ = (size_t)X * Z;
    int f = 0;
    for (int t = 1; t < T; t++) {
        frame_p_f32(&F, t, cquad, d_x, d_z, constvec, 0);
        inject_f32(&F, t, ns, sx, sz, src, integ, 0, idx_source);
        record_f32(&F, t, nm, mx, mz, rec);
        frame_a_f32(&F, t, d_x, d_z, constvec, 0);
        if (t % every != 0)
            continue;
        const float *px = F.Px + (size_t)(t % 2) * XZ, *pz = F.Pz + (size_t)(t % 2) * XZ;
        for (size_t i = 0; i < XZ; i++)
            img[i] = px[i] + pz[i];
        float max = img[0], min = img[0];
        for (size_t i = 0; i < XZ; i++) {
            float value = img[i];
            if (value > max)
                max = value;
            if (value < min)
                min = value;
        }
        float offset = -min;
        float scale = 255.0f / (max - min);
        unsigned char *buffer = frames + (size_t)f * XZ;
        /* a constant frame makes every byte 0 * inf = NaN, whose conversion
         * is undefined in C (x86-64 code gives 0); 0 here, as on the device */
        for (size_t i = 0; i < XZ; i++)
            buffer[i] = max > min ? (unsigned char)((img[i] + offset) * scale) : 0;
        for (int i = 0; i < nm; i++)
            buffer[mx[i] + (size_t)X * mz[i]] = 255;
        if (p_out)
            memcpy(p_out + (size_t)f * XZ, img, sizeof(float) * XZ);
        f++;
    }
    free(integ);
    free(rec);
    free(img);
    free_fields_f32(&F);
    return 0;
}
