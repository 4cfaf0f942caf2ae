/*
 * CPU oracle for the second-order CPML forward path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker the CPML parity tests compare the
 * CUDA library against; the product never loads it.
 *
 * Restates the reference's simulator/src/regression_CPML.cu (paths relative
 * to the Otfwi project root):
 *   :10-13   xzt (four time slots) / inbounds(., 4)
 *   :49-120  simulateFrame1: first staggered derivatives of P(t-1), CPML
 *            memory variables, divided by the half-point densities
 *   :123-207 simulateFrame2: staggered derivatives of those, second memory
 *            variables, P(t) = 2 P(t-1) - P(t-2) + lap dt^2 kappa
 *   :210-231 somaFonte: P += 4pi * c^2 * s(t) * dt^2 at the sources
 *   :238-246 gravaBufferSensores2ordem: rec(t) = P(t), from t = 0
 *   :451-531 cuda_simulate2: P(0), P(1) from `initial`, steps t >= 2
 * with the prec_deriv == 4 stencil of simulator/src/deriv_macros.h:84-108.
 *
 * Two modes from one body: *_f32 the reference's arithmetic (FP32 fields,
 * FP64 staggered sums rounded to FP32, FP32 updates with the fused
 * multiply-adds the reference's expressions contract to), *_f64 the same
 * algorithm in FP64. Build: oracle/Makefile (gcc -ffp-contract=off).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define CC0 1.196289e+00
#define CC1 7.975260e-02
#define CC2 9.570313e-03
#define CC3 6.975446e-04

#define CPML_BODY(REAL, SUF, RND, FMA)                                                                  \
    /* masked load: zero outside inbounds(., 4), as the reference's tile loaders */                    \
    static inline REAL ld_##SUF(const REAL *f, int X, int Z, int x, int z)                             \
    {                                                                                                  \
        return (x >= 4 && z >= 4 && x < X - 4 && z < Z - 4) ? f[(size_t)z * X + x] : (REAL)0;          \
    }                                                                                                  \
    /* 8-tap staggered derivative in FP64: leading product rounded, seven FMAs */                     \
    static inline double dstag_##SUF(const REAL *f, int X, int Z, int x, int z, int ddx, int ddz,    \
                                     int off)                                                          \
    {                                                                                                  \
        double s = -CC3 * (double)ld_##SUF(f, X, Z, x + (4 - off) * ddx, z + (4 - off) * ddz);        \
        s = fma(CC2, (double)ld_##SUF(f, X, Z, x + (3 - off) * ddx, z + (3 - off) * ddz), s);          \
        s = fma(-CC1, (double)ld_##SUF(f, X, Z, x + (2 - off) * ddx, z + (2 - off) * ddz), s);         \
        s = fma(CC0, (double)ld_##SUF(f, X, Z, x + (1 - off) * ddx, z + (1 - off) * ddz), s);          \
        s = fma(-CC0, (double)ld_##SUF(f, X, Z, x - off * ddx, z - off * ddz), s);                     \
        s = fma(CC1, (double)ld_##SUF(f, X, Z, x + (-1 - off) * ddx, z + (-1 - off) * ddz), s);        \
        s = fma(-CC2, (double)ld_##SUF(f, X, Z, x + (-2 - off) * ddx, z + (-2 - off) * ddz), s);       \
        s = fma(CC3, (double)ld_##SUF(f, X, Z, x + (-3 - off) * ddx, z + (-3 - off) * ddz), s);        \
        return s;                                                                                      \
    }                                                                                                  \
    int orc_cpml_simulate_##SUF(int X, int Z, int T, int ns, int ppe, const int *ps_x, const int *ps_z, \
                                int nm, const int *pm_x, const int *pm_z, float dx_, float dz_,        \
                                float dt2_, float qtpi_, const float *cquad, const float *kappa,        \
                                const float *rho_hx, const float *rho_hz, const float *Kx,             \
                                const float *ax, const float *bx, const float *Kxh, const float *axh,  \
                                const float *bxh, const float *Kz, const float *az, const float *bz,   \
                                const float *Kzh, const float *azh, const float *bzh, const float *src, \
                                const float *init, int idx, REAL *rec)                                 \
    {                                                                                                  \
        const size_t XZ = (size_t)X * Z;                                                               \
        REAL *P = (REAL *)calloc(4 * XZ, sizeof(REAL)); /* slots t % 4 */                                                \
        REAL *mx = (REAL *)calloc(XZ, sizeof(REAL)), *mz = (REAL *)calloc(XZ, sizeof(REAL));           \
        REAL *mxx = (REAL *)calloc(XZ, sizeof(REAL)), *mzz = (REAL *)calloc(XZ, sizeof(REAL));         \
        REAL *v1x = (REAL *)calloc(XZ, sizeof(REAL)), *v1z = (REAL *)calloc(XZ, sizeof(REAL));         \
        if (!P || !mx || !mz || !mxx || !mzz || !v1x || !v1z)                                          \
            return -1;                                                                                 \
        const REAL dx = (REAL)dx_, dz = (REAL)dz_, dt2 = (REAL)dt2_, qtpi = (REAL)qtpi_;               \
        for (size_t i = 0; i < 2 * XZ; i++)                                                            \
            P[i] = (REAL)init[i];                                                                      \
        for (int t = 0; t < T; t++) {                                                                  \
            REAL *Pn = P + (t % 4) * XZ;                                                               \
            const REAL *P1 = P + ((t + 3) % 4) * XZ, *P2 = P + ((t + 2) % 4) * XZ;                     \
            if (t > 1) {                                                                               \
                /* simulateFrame1 */                                                                   \
                _Pragma("omp parallel for schedule(static)") for (int z = 4; z < Z - 4; z++)           \
                for (int x = 4; x < X - 4; x++)                                                       \
                {                                                                                      \
                    const size_t i = (size_t)z * X + x;                                                \
                    const REAL v0x = (REAL)RND(dstag_##SUF(P1, X, Z, x, z, 1, 0, 0)) / dx;             \
                    mx[i] = FMA((REAL)bxh[x], mx[i], (REAL)axh[x] * v0x);                              \
                    v1x[i] = (v0x / (REAL)Kxh[x] + mx[i]) / (REAL)rho_hx[i];                           \
                    const REAL v0z = (REAL)RND(dstag_##SUF(P1, X, Z, x, z, 0, 1, 0)) / dz;             \
                    mz[i] = FMA((REAL)bzh[z], mz[i], (REAL)azh[z] * v0z);                              \
                    v1z[i] = (v0z / (REAL)Kzh[z] + mz[i]) / (REAL)rho_hz[i];                           \
                }                                                                                      \
                /* simulateFrame2 */                                                                   \
                _Pragma("omp parallel for schedule(static)") for (int z = 4; z < Z - 4; z++)           \
                for (int x = 4; x < X - 4; x++)                                                       \
                {                                                                                      \
                    const size_t i = (size_t)z * X + x;                                                \
                    const REAL vxx0 = (REAL)RND(dstag_##SUF(v1x, X, Z, x, z, 1, 0, 1)) / dx;           \
                    mxx[i] = FMA((REAL)bx[x], mxx[i], (REAL)ax[x] * vxx0);                             \
                    const REAL vxx1 = vxx0 / (REAL)Kx[x] + mxx[i];                                     \
                    const REAL vzz0 = (REAL)RND(dstag_##SUF(v1z, X, Z, x, z, 0, 1, 1)) / dz;           \
                    mzz[i] = FMA((REAL)bz[z], mzz[i], (REAL)az[z] * vzz0);                             \
                    const REAL vzz1 = vzz0 / (REAL)Kz[z] + mzz[i];                                     \
                    const REAL lap = vxx1 + vzz1;                                                      \
                    Pn[i] = FMA(lap * dt2, (REAL)kappa[i], FMA((REAL)2, P1[i], -P2[i]));               \
                }                                                                                      \
                /* somaFonte */                                                                        \
                for (int n = 0; n < ns; n++) {                                                         \
                    if (ppe == 1 && idx != -1 && idx != n)                                             \
                        continue;                                                                      \
                    const size_t i = (size_t)ps_z[n] * X + ps_x[n];                                    \
                    Pn[i] = FMA(qtpi * (REAL)cquad[i] * (REAL)src[(size_t)n * T + t], dt2, Pn[i]);     \
                }                                                                                      \
            }                                                                                          \
            for (int n = 0; n < nm; n++)                                                               \
                rec[(size_t)n * T + t] = Pn[(size_t)pm_z[n] * X + pm_x[n]];                            \
        }                                                                                              \
        free(P);                                                                                       \
        free(mx);                                                                                      \
        free(mz);                                                                                      \
        free(mxx);                                                                                     \
        free(mzz);                                                                                     \
        free(v1x);                                                                                     \
        free(v1z);                                                                                     \
        return 0;                                                                                      \
    }

#define RND_F(v) ((float)(v))
#define RND_D(v) (v)
CPML_BODY(float, f32, RND_F, fmaf)
CPML_BODY(double, f64, RND_D, fma)
