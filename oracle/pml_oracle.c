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
