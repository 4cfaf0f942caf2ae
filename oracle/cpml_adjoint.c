/*
 * Exact discrete adjoint of the second-order CPML scheme, FP64 (CPU oracle).
 *
 * TEST INFRASTRUCTURE ONLY: the checker of the CPML gradient.
 *
 * The forward map is the f64 mode of cpml_oracle.c (regression_CPML.cu:
 * 49-231, 451-531). For a loss L with dL/drec = g [nm][T], this returns
 * dL/dkappa [Z][X] (kappa = rho c^2, the coefficient of the Laplacian; the
 * source term's c^2 is held fixed). It runs the forward keeping lap(t) of
 * every step, then the transposed steps backwards. Every transpose is the
 * literal scatter of the forward's gather (masked reads included), so no
 * identity between the staggered operators is assumed.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define AC0 1.196289e+00
#define AC1 7.975260e-02
#define AC2 9.570313e-03
#define AC3 6.975446e-04

/* taps of derivPMLdx(m, off, x): m[x + k - off] * W[k + 3], k = -3..4 */
static const double W[8] = {AC3, -AC2, AC1, -AC0, AC0, -AC1, AC2, -AC3};

static inline int inb(int X, int Z, int x, int z) { return x >= 4 && z >= 4 && x < X - 4 && z < Z - 4; }

/* out[i] = sum_k W[k+3] * in_masked[i + (k - off) * step] for inbounds i */
static void gather(const double *in, double *out, int X, int Z, int ddx, int ddz, int off, double scale)
{
    for (int z = 0; z < Z; z++)
        for (int x = 0; x < X; x++) {
            const size_t i = (size_t)z * X + x;
            if (!inb(X, Z, x, z)) {
                out[i] = 0.0;
                continue;
            }
            double s = 0.0;
            for (int k = -3; k <= 4; k++) {
                const int xx = x + (k - off) * ddx, zz = z + (k - off) * ddz;
                if (inb(X, Z, xx, zz))
                    s += W[k + 3] * in[(size_t)zz * X + xx];
            }
            out[i] = s * scale;
        }
}

/* transpose of gather: adj_in[j] += sum over inbounds i reading j */
static void scatter(const double *adj_out, double *adj_in, int X, int Z, int ddx, int ddz, int off, double scale)
{
    for (int z = 0; z < Z; z++)
        for (int x = 0; x < X; x++) {
            if (!inb(X, Z, x, z))
                continue;
            const double a = adj_out[(size_t)z * X + x] * scale;
            if (a == 0.0)
                continue;
            for (int k = -3; k <= 4; k++) {
                const int xx = x + (k - off) * ddx, zz = z + (k - off) * ddz;
                if (inb(X, Z, xx, zz))
                    adj_in[(size_t)zz * X + xx] += W[k + 3] * a;
            }
        }
}

int orc_cpml_adjoint_f64(int X, int Z, int T, int ns, int ppe, const int *ps_x, const int *ps_z, int nm,
                         const int *pm_x, const int *pm_z, float dx_, float dz_, float dt2_, float qtpi_,
                         const float *cquad, const float *kappa, const float *rho_hx, const float *rho_hz,
                         const float *Kx, const float *ax, const float *bx, const float *Kxh, const float *axh,
                         const float *bxh, const float *Kz, const float *az, const float *bz, const float *Kzh,
                         const float *azh, const float *bzh, const float *src, const float *init, int idx,
                         const double *g, double *grad_kappa, double *rec)
{
    const size_t XZ = (size_t)X * Z;
    const double dx = dx_, dz = dz_, dt2 = dt2_, qtpi = qtpi_;
    double *P = calloc(4 * XZ, sizeof(double));
    double *mx = calloc(XZ, sizeof(double)), *mz = calloc(XZ, sizeof(double));
    double *mxx = calloc(XZ, sizeof(double)), *mzz = calloc(XZ, sizeof(double));
    double *v0 = calloc(XZ, sizeof(double)), *v1x = calloc(XZ, sizeof(double)), *v1z = calloc(XZ, sizeof(double));
    double *w0 = calloc(XZ, sizeof(double));
    double *lap = calloc((size_t)T * XZ, sizeof(double));
    double *LA = calloc(XZ, sizeof(double)), *LB = calloc(XZ, sizeof(double)), *LC = calloc(XZ, sizeof(double));
    double *lmx = calloc(XZ, sizeof(double)), *lmz = calloc(XZ, sizeof(double));
    double *lmxx = calloc(XZ, sizeof(double)), *lmzz = calloc(XZ, sizeof(double));
    double *lv1x = calloc(XZ, sizeof(double)), *lv1z = calloc(XZ, sizeof(double));
    double *l0 = calloc(XZ, sizeof(double));
    if (!P || !mx || !mz || !mxx || !mzz || !v0 || !v1x || !v1z || !w0 || !lap || !LA || !LB || !LC || !lmx ||
        !lmz || !lmxx || !lmzz || !lv1x || !lv1z || !l0)
        return -1;
    for (size_t i = 0; i < 2 * XZ; i++)
        P[i] = init[i];
    /* forward, keeping lap(t) */
    for (int t = 0; t < T; t++) {
        double *Pn = P + (t % 4) * XZ;
        const double *P1 = P + ((t + 3) % 4) * XZ, *P2 = P + ((t + 2) % 4) * XZ;
        if (t > 1) {
            gather(P1, v0, X, Z, 1, 0, 0, 1.0 / dx);
            for (size_t i = 0; i < XZ; i++) {
                const int x = (int)(i % X), z = (int)(i / X);
                if (!inb(X, Z, x, z)) {
                    v1x[i] = 0.0;
                    continue;
                }
                mx[i] = bxh[x] * mx[i] + axh[x] * v0[i];
                v1x[i] = (v0[i] / Kxh[x] + mx[i]) / rho_hx[i];
            }
            gather(P1, v0, X, Z, 0, 1, 0, 1.0 / dz);
            for (size_t i = 0; i < XZ; i++) {
                const int x = (int)(i % X), z = (int)(i / X);
                if (!inb(X, Z, x, z)) {
                    v1z[i] = 0.0;
                    continue;
                }
                mz[i] = bzh[z] * mz[i] + azh[z] * v0[i];
                v1z[i] = (v0[i] / Kzh[z] + mz[i]) / rho_hz[i];
            }
            gather(v1x, v0, X, Z, 1, 0, 1, 1.0 / dx);
            gather(v1z, w0, X, Z, 0, 1, 1, 1.0 / dz);
            double *lt = lap + (size_t)t * XZ;
            for (size_t i = 0; i < XZ; i++) {
                const int x = (int)(i % X), z = (int)(i / X);
                if (!inb(X, Z, x, z))
                    continue;
                mxx[i] = bx[x] * mxx[i] + ax[x] * v0[i];
                mzz[i] = bz[z] * mzz[i] + az[z] * w0[i];
                lt[i] = (v0[i] / Kx[x] + mxx[i]) + (w0[i] / Kz[z] + mzz[i]);
                Pn[i] = 2.0 * P1[i] - P2[i] + lt[i] * dt2 * kappa[i];
            }
            for (int n = 0; n < ns; n++) {
                if (ppe == 1 && idx != -1 && idx != n)
                    continue;
                const size_t i = (size_t)ps_z[n] * X + ps_x[n];
                Pn[i] += qtpi * cquad[i] * src[(size_t)n * T + t] * dt2;
            }
        }
        for (int n = 0; n < nm; n++)
            rec[(size_t)n * T + t] = Pn[(size_t)pm_z[n] * X + pm_x[n]];
    }
    /* reverse: LA = adjoint of P(t), LB = adjoint of P(t-1) gathered so far */
    memset(grad_kappa, 0, XZ * sizeof(double));
    for (int t = T - 1; t >= 2; t--) {
        for (int n = 0; n < nm; n++) {
            const size_t i = (size_t)pm_z[n] * X + pm_x[n];
            if (inb(X, Z, pm_x[n], pm_z[n]))
                LA[i] += g[(size_t)n * T + t];
        }
        const double *lt = lap + (size_t)t * XZ;
        memset(LC, 0, XZ * sizeof(double));
        memset(lv1x, 0, XZ * sizeof(double));
        memset(lv1z, 0, XZ * sizeof(double));
        /* P(t) = 2 P1 - P2 + dt2 kappa lap,  lap = vxx1 + vzz1 */
        for (size_t i = 0; i < XZ; i++) {
            const int x = (int)(i % X), z = (int)(i / X);
            if (!inb(X, Z, x, z)) {
                v0[i] = w0[i] = 0.0;
                continue;
            }
            grad_kappa[i] += LA[i] * dt2 * lt[i];
            const double gl = dt2 * kappa[i] * LA[i];
            LB[i] += 2.0 * LA[i];
            LC[i] -= LA[i];
            /* vxx1 = vxx0 / Kx + mxx(t),  mxx(t) = bx mxx(t-1) + ax vxx0 */
            const double tx = lmxx[i] + gl;
            v0[i] = gl / Kx[x] + ax[x] * tx;  /* adjoint of vxx0 */
            lmxx[i] = bx[x] * tx;
            const double tz = lmzz[i] + gl;
            w0[i] = gl / Kz[z] + az[z] * tz;  /* adjoint of vzz0 */
            lmzz[i] = bz[z] * tz;
        }
        /* vxx0 = D(v1x, off 1) / dx */
        scatter(v0, lv1x, X, Z, 1, 0, 1, 1.0 / dx);
        scatter(w0, lv1z, X, Z, 0, 1, 1, 1.0 / dz);
        for (size_t i = 0; i < XZ; i++) {
            const int x = (int)(i % X), z = (int)(i / X);
            if (!inb(X, Z, x, z)) {
                l0[i] = v0[i] = 0.0;
                continue;
            }
            /* v1x = (v0x / Kxh + mx(t)) / rho_hx,  mx(t) = bxh mx(t-1) + axh v0x */
            const double tx = lmx[i] + lv1x[i] / rho_hx[i];
            l0[i] = lv1x[i] / (Kxh[x] * rho_hx[i]) + axh[x] * tx;  /* adjoint of v0x */
            lmx[i] = bxh[x] * tx;
            const double tz = lmz[i] + lv1z[i] / rho_hz[i];
            v0[i] = lv1z[i] / (Kzh[z] * rho_hz[i]) + azh[z] * tz;  /* adjoint of v0z */
            lmz[i] = bzh[z] * tz;
        }
        /* v0x = D(P1, off 0) / dx into the adjoint of P(t-1) */
        scatter(l0, LB, X, Z, 1, 0, 0, 1.0 / dx);
        scatter(v0, LB, X, Z, 0, 1, 0, 1.0 / dz);
        /* shift: P(t-1) becomes the current state */
        double *tmp = LA;
        LA = LB;
        LB = LC;
        LC = tmp;
    }
    free(P);
    free(mx);
    free(mz);
    free(mxx);
    free(mzz);
    free(v0);
    free(v1x);
    free(v1z);
    free(w0);
    free(lap);
    free(LA);
    free(LB);
    free(LC);
    free(lmx);
    free(lmz);
    free(lmxx);
    free(lmzz);
    free(lv1x);
    free(lv1z);
    free(l0);
    return 0;
}
