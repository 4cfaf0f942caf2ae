/*
 * Exact discrete adjoint of the split-field PML forward map, FP64.
 *
 * TEST INFRASTRUCTURE ONLY (checker for the CUDA adjoint and for finite
 * differences); the product never loads it.
 *
 * Forward map (one shot or all sources, restating regression_PML_single.cu:
 * 447-615 and 276-309 in FP64, M = update mask 4 <= x < X-4, 4 <= z < Z-4):
 *   Px_t = M (ax Px_{t-1} + q Dx- Ax_{t-1}) + I_t/2 d_src      (q = c2*dt/dx)
 *   Pz_t = M (az Pz_{t-1} + q Dz- Az_{t-1}) + I_t/2 d_src
 *   rec_t = (Px_t + Pz_t)[receivers]
 *   Ax_t = M (ax Ax_{t-1} + r Dx+ (Px_t + Pz_t)),  Az_t likewise  (r = dt/dx)
 * with a = 1 - d*dt at the reference's +1-shifted damping index. Given
 * g_t = dL/drec_t, the reverse step t -> t-1 is
 *   S     = r (Dx+^T (M lAx_t) + Dz+^T (M lAz_t)) + scatter(g_t)
 *   lPxT  = lPx_t + S,   lPzT = lPz_t + S
 *   lAx_{t-1} = ax M lAx_t + Dx-^T (q M lPxT),  lAz likewise
 *   lPx_{t-1} = ax M lPxT,  lPz likewise
 *   dL/dq += M lPxT * Dx- Ax_{t-1} + M lPzT * Dz- Az_{t-1}
 * Transposes are applied literally (scatter), so the result is the exact
 * transpose of the discrete operator. Returns dL/d(c^2) = (dt/dx) dL/dq.
 * Build: oracle/Makefile (into liborc.so).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

static const double A0 = 1.196289e+00, A1 = 7.975260e-02, A2 = 9.570313e-03, A3 = 6.975446e-04;

/* staggered weights: D-(offset 1) taps k = -4..3, D+(offset 0) taps k = -3..4 */
static void weights(int off, int *k0, double w[8])
{
    /* macro order K = 4..-3 with coefficients -c3,+c2,-c1,+c0,-c0,+c1,-c2,+c3 at m[x+K-off] */
    const double c[8] = {A3, -A2, A1, -A0, A0, -A1, A2, -A3}; /* for K = -3..4 */
    *k0 = -3 - off;
    for (int i = 0; i < 8; i++)
        w[i] = c[i];
}

static int inb(int x, int z, int X, int Z) { return x >= 4 && z >= 4 && x < X - 4 && z < Z - 4; }

/* out(x) = sum_i w_i f(x + k0 + i) along (ddx, ddz), f masked to the update region */
static double dapply(const double *f, int X, int Z, int x, int z, int ddx, int ddz, int off)
{
    int k0;
    double w[8], s = 0.0;
    weights(off, &k0, w);
    for (int i = 0; i < 8; i++) {
        const int xx = x + (k0 + i) * ddx, zz = z + (k0 + i) * ddz;
        if (inb(xx, zz, X, Z))
            s += w[i] * f[xx + zz * X];
    }
    return s;
}

/* out(y) += sum over x with y = x + k0 + i of w_i v(x): transpose of dapply,
 * scattering only into cells the forward reads (the update region) */
static void dtrans(const double *v, double *out, int X, int Z, int ddx, int ddz, int off)
{
    int k0;
    double w[8];
    weights(off, &k0, w);
    for (int z = 0; z < Z; z++)
        for (int x = 0; x < X; x++) {
            const double vv = v[x + z * X];
            if (vv == 0.0)
                continue;
            for (int i = 0; i < 8; i++) {
                const int xx = x + (k0 + i) * ddx, zz = z + (k0 + i) * ddz;
                if (inb(xx, zz, X, Z))
                    out[xx + zz * X] += w[i] * vv;
            }
        }
}

/*
 * dL/d(c^2) [Z*X] of L with dL/drec_t = g [nm][T] (column 0 unused), and the
 * traces rec [nm][T] of the forward run. Sources fire as in cuda_simulate
 * (idx_source = -1: all).
 */
int orc_exact_adjoint_f64(int X, int Z, int T, const float *cquad, const float *constvec,
                          const float *d_x, const float *d_z, int ns, const int *sx, const int *sz,
                          const float *src, int idx_source, int nm, const int *mx, const int *mz,
                          const double *g, double *grad_c2, double *rec)
{
    const size_t XZ = (size_t)X * Z;
    const double dx = constvec[0], dt = constvec[2], r = dt / dx;
    double *q = calloc(XZ, sizeof(double)), *ax = calloc(XZ, sizeof(double)), *az = calloc(XZ, sizeof(double));
    double *AxH = calloc(XZ * T, sizeof(double)), *AzH = calloc(XZ * T, sizeof(double));
    double *Px = calloc(XZ, sizeof(double)), *Pz = calloc(XZ, sizeof(double));
    double *Pt = calloc(XZ, sizeof(double)), *integ = calloc(ns > 0 ? ns : 1, sizeof(double));
    double *lPx = calloc(XZ, sizeof(double)), *lPz = calloc(XZ, sizeof(double));
    double *lAx = calloc(XZ, sizeof(double)), *lAz = calloc(XZ, sizeof(double));
    double *tx = calloc(XZ, sizeof(double)), *tz = calloc(XZ, sizeof(double));
    double *S = calloc(XZ, sizeof(double)), *gq = calloc(XZ, sizeof(double));
    if (!q || !AxH || !AzH || !gq)
        return -1;
    for (int z = 0; z < Z; z++)
        for (int x = 0; x < X; x++) {
            const size_t i = (size_t)x + (size_t)z * X;
            q[i] = (double)cquad[i] * dt / dx;
            ax[i] = i + 1 < XZ ? 1.0 - (double)d_x[i + 1] * dt : 1.0;
            az[i] = z + 1 < Z ? 1.0 - (double)d_z[i + X] * dt : 1.0;
        }
    memset(rec, 0, sizeof(double) * (size_t)nm * T);
    /* forward with the A history */
    for (int t = 1; t < T; t++) {
        const double *Axo = AxH + XZ * (t - 1), *Azo = AzH + XZ * (t - 1);
        double *Axn = AxH + XZ * t, *Azn = AzH + XZ * t;
        for (int z = 0; z < Z; z++)
            for (int x = 0; x < X; x++) {
                const size_t i = (size_t)x + (size_t)z * X;
                if (!inb(x, z, X, Z))
                    continue;
                Px[i] = ax[i] * Px[i] + q[i] * dapply(Axo, X, Z, x, z, 1, 0, 1);
                Pz[i] = az[i] * Pz[i] + q[i] * dapply(Azo, X, Z, x, z, 0, 1, 1);
            }
        for (int k = 0; k < ns; k++) {
            if (idx_source != -1 && idx_source != k)
                continue;
            integ[k] += (double)src[(size_t)k * T + t];
            const size_t i = (size_t)sx[k] + (size_t)sz[k] * X;
            Px[i] += integ[k] / 2;
            Pz[i] += integ[k] / 2;
        }
        for (size_t i = 0; i < XZ; i++)
            Pt[i] = Px[i] + Pz[i];
        for (int n = 0; n < nm; n++)
            rec[(size_t)n * T + t] = Pt[mx[n] + (size_t)mz[n] * X];
        for (int z = 0; z < Z; z++)
            for (int x = 0; x < X; x++) {
                const size_t i = (size_t)x + (size_t)z * X;
                if (!inb(x, z, X, Z))
                    continue;
                Axn[i] = ax[i] * Axo[i] + r * dapply(Pt, X, Z, x, z, 1, 0, 0);
                Azn[i] = az[i] * Azo[i] + r * dapply(Pt, X, Z, x, z, 0, 1, 0);
            }
    }
    /* reverse */
    for (int t = T - 1; t >= 1; t--) {
        const double *Axo = AxH + XZ * (t - 1), *Azo = AzH + XZ * (t - 1);
        memset(S, 0, sizeof(double) * XZ);
        for (size_t i = 0; i < XZ; i++) {
            tx[i] = r * lAx[i];
            tz[i] = r * lAz[i];
        }
        dtrans(tx, S, X, Z, 1, 0, 0);
        dtrans(tz, S, X, Z, 0, 1, 0);
        for (int n = 0; n < nm; n++)
            if (inb(mx[n], mz[n], X, Z))
                S[mx[n] + (size_t)mz[n] * X] += g[(size_t)n * T + t];
        for (size_t i = 0; i < XZ; i++) {
            lPx[i] += S[i];
            lPz[i] += S[i];
        }
        /* gradient and the A adjoints use lPxT / lPzT (masked) */
        for (int z = 0; z < Z; z++)
            for (int x = 0; x < X; x++) {
                const size_t i = (size_t)x + (size_t)z * X;
                if (!inb(x, z, X, Z)) {
                    lPx[i] = lPz[i] = 0.0;
                    continue;
                }
                gq[i] += lPx[i] * dapply(Axo, X, Z, x, z, 1, 0, 1) + lPz[i] * dapply(Azo, X, Z, x, z, 0, 1, 1);
            }
        for (size_t i = 0; i < XZ; i++) {
            tx[i] = q[i] * lPx[i];
            tz[i] = q[i] * lPz[i];
        }
        for (int z = 0; z < Z; z++)
            for (int x = 0; x < X; x++) {
                const size_t i = (size_t)x + (size_t)z * X;
                const int m = inb(x, z, X, Z);
                lAx[i] = m ? ax[i] * lAx[i] : 0.0;
                lAz[i] = m ? az[i] * lAz[i] : 0.0;
            }
        dtrans(tx, lAx, X, Z, 1, 0, 1);
        dtrans(tz, lAz, X, Z, 0, 1, 1);
        for (size_t i = 0; i < XZ; i++) {
            lPx[i] *= ax[i];
            lPz[i] *= az[i];
        }
    }
    for (size_t i = 0; i < XZ; i++)
        grad_c2[i] = gq[i] * dt / dx;
    free(q); free(ax); free(az); free(AxH); free(AzH); free(Px); free(Pz); free(Pt); free(integ);
    free(lPx); free(lPz); free(lAx); free(lAz); free(tx); free(tz); free(S); free(gq);
    return 0;
}

/* FP64 forward traces of the same map (for finite differences). */
int orc_forward_f64(int X, int Z, int T, const double *cquad, const float *constvec, const float *d_x,
                    const float *d_z, int ns, const int *sx, const int *sz, const float *src, int idx_source,
                    int nm, const int *mx, const int *mz, double *rec)
{
    const size_t XZ = (size_t)X * Z;
    const double dx = constvec[0], dt = constvec[2], r = dt / dx;
    double *q = calloc(XZ, sizeof(double)), *ax = calloc(XZ, sizeof(double)), *az = calloc(XZ, sizeof(double));
    double *Ax = calloc(XZ, sizeof(double)), *Az = calloc(XZ, sizeof(double));
    double *Ax2 = calloc(XZ, sizeof(double)), *Az2 = calloc(XZ, sizeof(double));
    double *Px = calloc(XZ, sizeof(double)), *Pz = calloc(XZ, sizeof(double));
    double *Pt = calloc(XZ, sizeof(double)), *integ = calloc(ns > 0 ? ns : 1, sizeof(double));
    if (!q || !Ax || !Pt)
        return -1;
    for (int z = 0; z < Z; z++)
        for (int x = 0; x < X; x++) {
            const size_t i = (size_t)x + (size_t)z * X;
            q[i] = cquad[i] * dt / dx;
            ax[i] = i + 1 < XZ ? 1.0 - (double)d_x[i + 1] * dt : 1.0;
            az[i] = z + 1 < Z ? 1.0 - (double)d_z[i + X] * dt : 1.0;
        }
    memset(rec, 0, sizeof(double) * (size_t)nm * T);
    for (int t = 1; t < T; t++) {
        for (int z = 0; z < Z; z++)
            for (int x = 0; x < X; x++) {
                const size_t i = (size_t)x + (size_t)z * X;
                if (!inb(x, z, X, Z))
                    continue;
                Px[i] = ax[i] * Px[i] + q[i] * dapply(Ax, X, Z, x, z, 1, 0, 1);
                Pz[i] = az[i] * Pz[i] + q[i] * dapply(Az, X, Z, x, z, 0, 1, 1);
            }
        for (int k = 0; k < ns; k++) {
            if (idx_source != -1 && idx_source != k)
                continue;
            integ[k] += (double)src[(size_t)k * T + t];
            const size_t i = (size_t)sx[k] + (size_t)sz[k] * X;
            Px[i] += integ[k] / 2;
            Pz[i] += integ[k] / 2;
        }
        for (size_t i = 0; i < XZ; i++)
            Pt[i] = Px[i] + Pz[i];
        for (int n = 0; n < nm; n++)
            rec[(size_t)n * T + t] = Pt[mx[n] + (size_t)mz[n] * X];
        for (int z = 0; z < Z; z++)
            for (int x = 0; x < X; x++) {
                const size_t i = (size_t)x + (size_t)z * X;
                if (!inb(x, z, X, Z)) {
                    Ax2[i] = Az2[i] = 0.0;
                    continue;
                }
                Ax2[i] = ax[i] * Ax[i] + r * dapply(Pt, X, Z, x, z, 1, 0, 0);
                Az2[i] = az[i] * Az[i] + r * dapply(Pt, X, Z, x, z, 0, 1, 0);
            }
        double *s1 = Ax; Ax = Ax2; Ax2 = s1;
        double *s2 = Az; Az = Az2; Az2 = s2;
    }
    free(q); free(ax); free(az); free(Ax); free(Az); free(Ax2); free(Az2); free(Px); free(Pz); free(Pt);
    free(integ);
    return 0;
}
