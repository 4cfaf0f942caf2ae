/*
 * Body of the CPU oracle, included twice by pml_oracle.c:
 *   ORC_REAL = float  -> "f32" mode: the reference's own mixed precision
 *                        (FP32 fields, FP64 8-tap staggered sums rounded to
 *                        FP32, FP32 updates with the fused multiply-adds the
 *                        reference's expressions contract to);
 *   ORC_REAL = double -> "f64" mode: the same algorithm carried in FP64.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker, never the product:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.
 *
 * Restated from the reference (paths relative to the Otfwi project root):
 *   simulator/src/regression_PML_single.cu:9-10    xzt / inbounds
 *   simulator/src/regression_PML_single.cu:447-528 simulateFrameP
 *   simulator/src/regression_PML_single.cu:531-615 simulateFrameA
 *   simulator/src/regression_PML_single.cu:276-292 somaFonteIntegral
 *   simulator/src/regression_PML_single.cu:295-309 gravaBufferSensores
 *   simulator/src/regression_PML_single.cu:260-273 setRec
 *   simulator/src/regression_PML_single.cu:312-327 somaFrames
 *   simulator/src/regression_PML_single.cu:390-445 calcGrad2
 *   simulator/src/regression_PML_single.cu:618-702 cuda_simulate
 *   simulator/src/regression_PML_single.cu:704-846 cuda_grad_ext
 *   simulator/src/deriv_macros.h:84-135            prec_deriv == 4 stencils
 */

#define ORC_CAT2(a, b) a##_##b
#define ORC_CAT(a, b) ORC_CAT2(a, b)
#define ORC_FN(name) ORC_CAT(name, ORC_SUF)

typedef struct {
    int X, Z, T;
    ORC_REAL *Px, *Pz, *Ax, *Az; /* [2][Z][X] (time slot = t % 2) */
} ORC_FN(orc_fields);

/* Masked load: cells outside inbounds(.,4) read as zero, exactly as the
 * reference's shared-memory tile loaders do (regression_PML_single.cu:488-498). */
static inline ORC_REAL ORC_FN(ld)(const ORC_REAL *f, int X, int Z, int x, int z)
{
    if (x >= 4 && z >= 4 && x < X - 4 && z < Z - 4)
        return f[x + z * X];
    return (ORC_REAL)0;
}

/* 8-tap staggered first derivative along x or z (deriv_macros.h:85-108),
 * summed in FP64 in the reference's operand order: the expression
 * "-c3*m[+4-o] + c2*m[+3-o] - c1*m[+2-o] + c0*m[+1-o] - c0*m[-o]
 *  + c1*m[-1-o] - c2*m[-2-o] + c3*m[-3-o]" contracts to one product (the
 * leading negated term, rounded) followed by seven fused multiply-adds. */
static inline double ORC_FN(dstag)(const ORC_REAL *f, int X, int Z, int x, int z,
                                   int ddx, int ddz, int off)
{
#define M(k) ((double)ORC_FN(ld)(f, X, Z, x + (k)*ddx, z + (k)*ddz))
    double s = -ORC_C3 * M(4 - off);
    s = fma(ORC_C2, M(3 - off), s);
    s = fma(-ORC_C1, M(2 - off), s);
    s = fma(ORC_C0, M(1 - off), s);
    s = fma(-ORC_C0, M(0 - off), s);
    s = fma(ORC_C1, M(-1 - off), s);
    s = fma(-ORC_C2, M(-2 - off), s);
    s = fma(ORC_C3, M(-3 - off), s);
#undef M
    return s;
}

#if ORC_IS_F32
#define ORC_RND(v) ((float)(v))
#define ORC_FMA(a, b, c) fmaf((a), (b), (c))
#else
#define ORC_RND(v) (v)
#define ORC_FMA(a, b, c) fma((a), (b), (c))
#endif

/* 9-point second derivative (deriv_macros.h:110-135), FP32 literals in the
 * reference: the leading "-9*m[+4]" product rounded, eight fused
 * multiply-adds, then an IEEE division by 5040. (Pinned bit-exactly against
 * the reference's gradients; fusing the leading product instead changes
 * about 1% of gradient cells by an ulp.) */
static inline ORC_REAL ORC_FN(d2)(const ORC_REAL *f, int X, int Z, int x, int z,
                                  int ddx, int ddz)
{
#define M(k) (ORC_FN(ld)(f, X, Z, x + (k)*ddx, z + (k)*ddz))
    ORC_REAL s = (ORC_REAL)-9 * M(4);
    s = ORC_FMA((ORC_REAL)128, M(3), s);
    s = ORC_FMA((ORC_REAL)-1008, M(2), s);
    s = ORC_FMA((ORC_REAL)8064, M(1), s);
    s = ORC_FMA((ORC_REAL)-14350, M(0), s);
    s = ORC_FMA((ORC_REAL)8064, M(-1), s);
    s = ORC_FMA((ORC_REAL)-1008, M(-2), s);
    s = ORC_FMA((ORC_REAL)128, M(-3), s);
    s = ORC_FMA((ORC_REAL)-9, M(-4), s);
#undef M
    return s / (ORC_REAL)5040;
}

/* simulateFrameP (regression_PML_single.cu:447-528): P(t) from P(t-1), A(t-1).
 * Damping is read at the +1-shifted index, d_x[z][x+1] and d_z[z+1][x]
 * (regression_PML_single.cu:505-506). */
static void ORC_FN(frame_p)(ORC_FN(orc_fields) * F, int t, const float *cq, const float *dxa,
                            const float *dza, const float *cv, int revert)
{
    const int X = F->X, Z = F->Z;
    const size_t XZ = (size_t)X * Z;
    const ORC_REAL *Axo = F->Ax + ((t - 1) % 2) * XZ, *Azo = F->Az + ((t - 1) % 2) * XZ;
    const ORC_REAL *Pxo = F->Px + ((t - 1) % 2) * XZ, *Pzo = F->Pz + ((t - 1) % 2) * XZ;
    ORC_REAL *Pxn = F->Px + (t % 2) * XZ, *Pzn = F->Pz + (t % 2) * XZ;
    const ORC_REAL ddx = (ORC_REAL)cv[0], dt = (ORC_REAL)cv[2];
#pragma omp parallel for schedule(static)
    for (int z = 4; z < Z - 4; z++) {
        for (int x = 4; x < X - 4; x++) {
            const size_t i = (size_t)x + (size_t)z * X;
            const ORC_REAL dAx = ORC_RND(ORC_FN(dstag)(Axo, X, Z, x, z, 1, 0, 1));
            const ORC_REAL dAz = ORC_RND(ORC_FN(dstag)(Azo, X, Z, x, z, 0, 1, 1));
            const ORC_REAL c2 = (ORC_REAL)cq[i];
            if (!revert) {
                const ORC_REAL dmx = ORC_FMA(-(ORC_REAL)dxa[i + 1], dt, (ORC_REAL)1);
                const ORC_REAL dmz = ORC_FMA(-(ORC_REAL)dza[i + X], dt, (ORC_REAL)1);
                const ORC_REAL q = (c2 * dt) / ddx;
                Pxn[i] = ORC_FMA(Pxo[i], dmx, q * dAx);
                Pzn[i] = ORC_FMA(Pzo[i], dmz, q * dAz);
            } else {
                const ORC_REAL q = c2 * (dt / ddx);
                Pxn[i] = ORC_FMA(-q, dAx, Pxo[i]);
                Pzn[i] = ORC_FMA(-q, dAz, Pzo[i]);
            }
        }
    }
}

/* simulateFrameA (regression_PML_single.cu:531-615): A(t) from P(t), A(t-1). */
static void ORC_FN(frame_a)(ORC_FN(orc_fields) * F, int t, const float *dxa, const float *dza,
                            const float *cv, int revert)
{
    const int X = F->X, Z = F->Z;
    const size_t XZ = (size_t)X * Z;
    const ORC_REAL *Pxn = F->Px + (t % 2) * XZ, *Pzn = F->Pz + (t % 2) * XZ;
    const ORC_REAL *Axo = F->Ax + ((t - 1) % 2) * XZ, *Azo = F->Az + ((t - 1) % 2) * XZ;
    ORC_REAL *Axn = F->Ax + (t % 2) * XZ, *Azn = F->Az + (t % 2) * XZ;
    const ORC_REAL ddx = (ORC_REAL)cv[0], dt = (ORC_REAL)cv[2];
    const ORC_REAL r = dt / ddx;
#pragma omp parallel for schedule(static)
    for (int z = 4; z < Z - 4; z++) {
        for (int x = 4; x < X - 4; x++) {
            const size_t i = (size_t)x + (size_t)z * X;
            const ORC_REAL dPxdx = ORC_RND(ORC_FN(dstag)(Pxn, X, Z, x, z, 1, 0, 0));
            const ORC_REAL dPxdz = ORC_RND(ORC_FN(dstag)(Pxn, X, Z, x, z, 0, 1, 0));
            const ORC_REAL dPzdx = ORC_RND(ORC_FN(dstag)(Pzn, X, Z, x, z, 1, 0, 0));
            const ORC_REAL dPzdz = ORC_RND(ORC_FN(dstag)(Pzn, X, Z, x, z, 0, 1, 0));
            const ORC_REAL sx = dPxdx + dPzdx;
            const ORC_REAL sz = dPxdz + dPzdz;
            if (!revert) {
                const ORC_REAL dmx = ORC_FMA(-(ORC_REAL)dxa[i + 1], dt, (ORC_REAL)1);
                const ORC_REAL dmz = ORC_FMA(-(ORC_REAL)dza[i + X], dt, (ORC_REAL)1);
                Axn[i] = ORC_FMA(Axo[i], dmx, r * sx);
                Azn[i] = ORC_FMA(Azo[i], dmz, r * sz);
            } else {
                Axn[i] = ORC_FMA(-r, sx, Axo[i]);
                Azn[i] = ORC_FMA(-r, sz, Azo[i]);
            }
        }
    }
}

/* somaFonteIntegral (regression_PML_single.cu:276-292). */
static void ORC_FN(inject)(ORC_FN(orc_fields) * F, int t, int n, const int *px, const int *pz,
                           const float *s, ORC_REAL *integ, int flip, int idx)
{
    const int X = F->X, T = F->T;
    const size_t XZ = (size_t)X * F->Z;
    for (int k = 0; k < n; k++) {
        if (idx != -1 && idx != k)
            continue;
        integ[k] += (ORC_REAL)(flip ? s[(size_t)k * T + T - 1 - t] : s[(size_t)k * T + t]);
        const size_t i = (size_t)px[k] + (size_t)pz[k] * X + (t % 2) * XZ;
        F->Px[i] += integ[k] / (ORC_REAL)2;
        F->Pz[i] += integ[k] / (ORC_REAL)2;
    }
}

/* Same injection with an adjoint source carried in ORC_REAL (f64 mode feeds
 * an FP64 adjoint source back in). */
static void ORC_FN(inject_r)(ORC_FN(orc_fields) * F, int t, int n, const int *px, const int *pz,
                             const ORC_REAL *s, ORC_REAL *integ)
{
    const int X = F->X, T = F->T;
    const size_t XZ = (size_t)X * F->Z;
    for (int k = 0; k < n; k++) {
        integ[k] += s[(size_t)k * T + T - 1 - t];
        const size_t i = (size_t)px[k] + (size_t)pz[k] * X + (t % 2) * XZ;
        F->Px[i] += integ[k] / (ORC_REAL)2;
        F->Pz[i] += integ[k] / (ORC_REAL)2;
    }
}

/* gravaBufferSensores (regression_PML_single.cu:295-309). */
static void ORC_FN(record)(const ORC_FN(orc_fields) * F, int t, int n, const int *px,
                           const int *pz, ORC_REAL *buf)
{
    const int X = F->X, T = F->T;
    const size_t XZ = (size_t)X * F->Z;
    for (int k = 0; k < n; k++) {
        const size_t i = (size_t)px[k] + (size_t)pz[k] * X + (t % 2) * XZ;
        buf[(size_t)k * T + t] = F->Px[i] + F->Pz[i];
    }
}

/* setRec (regression_PML_single.cu:260-273). */
static void ORC_FN(set_ring)(ORC_FN(orc_fields) * F, int t, int n, const int *px, const int *pz,
                             const ORC_REAL *ring)
{
    const int X = F->X, T = F->T;
    const size_t XZ = (size_t)X * F->Z;
    for (int k = 0; k < n; k++) {
        const size_t i = (size_t)px[k] + (size_t)pz[k] * X + (t % 2) * XZ;
        F->Px[i] = ring[(size_t)k * T + T - 1 - t] / (ORC_REAL)2;
        F->Pz[i] = ring[(size_t)k * T + T - 1 - t] / (ORC_REAL)2;
    }
}

static int ORC_FN(alloc_fields)(ORC_FN(orc_fields) * F, int X, int Z, int T)
{
    const size_t n = (size_t)2 * X * Z;
    F->X = X;
    F->Z = Z;
    F->T = T;
    F->Px = (ORC_REAL *)calloc(n, sizeof(ORC_REAL));
    F->Pz = (ORC_REAL *)calloc(n, sizeof(ORC_REAL));
    F->Ax = (ORC_REAL *)calloc(n, sizeof(ORC_REAL));
    F->Az = (ORC_REAL *)calloc(n, sizeof(ORC_REAL));
    return (F->Px && F->Pz && F->Ax && F->Az) ? 0 : -1;
}

static void ORC_FN(free_fields)(ORC_FN(orc_fields) * F)
{
    free(F->Px);
    free(F->Pz);
    free(F->Ax);
    free(F->Az);
}

/* cuda_simulate (regression_PML_single.cu:618-702): forward modelling of one
 * shot (idx_source >= 0) or all sources at once (idx_source == -1).
 * rec_out [n_sensor][T]; column t = 0 is written as zero. */
int ORC_FN(orc_simulate)(int X, int Z, int T, const float *cquad, const float *constvec,
                         const float *d_x, const float *d_z, int ns, const int *sx,
                         const int *sz, const float *src, int idx_source, int nm,
                         const int *mx, const int *mz, ORC_REAL *rec_out)
{
    ORC_FN(orc_fields) F;
    if (ORC_FN(alloc_fields)(&F, X, Z, T))
        return -1;
    ORC_REAL *integ = (ORC_REAL *)calloc(ns > 0 ? ns : 1, sizeof(ORC_REAL));
    memset(rec_out, 0, sizeof(ORC_REAL) * (size_t)nm * T);
    for (int t = 1; t < T; t++) {
        ORC_FN(frame_p)(&F, t, cquad, d_x, d_z, constvec, 0);
        ORC_FN(inject)(&F, t, ns, sx, sz, src, integ, 0, idx_source);
        ORC_FN(record)(&F, t, nm, mx, mz, rec_out);
        ORC_FN(frame_a)(&F, t, d_x, d_z, constvec, 0);
    }
    free(integ);
    ORC_FN(free_fields)(&F);
    return 0;
}

/* Adjoint-source callback: receives the recorded traces [n_sensor][T] and
 * writes the adjoint source [n_sensor][T] (the reference's adj_calc,
 * regression_PML_single.cu:779). */
typedef void (*ORC_FN(orc_adj_cb))(const ORC_REAL *sim, ORC_REAL *adj, void *user);

/* cuda_grad_ext (regression_PML_single.cu:704-846): forward with boundary
 * ring recording, adjoint source from the callback, then the damped adjoint
 * field and the time-reversed reconstruction stepped together while the
 * imaging condition grad += P_adj(t) * lap9(P_rec(T-1-t)) accumulates. */
int ORC_FN(orc_grad)(int X, int Z, int T, const float *cquad, const float *constvec,
                     const float *d_x, const float *d_z, int ns, const int *sx, const int *sz,
                     const float *src, int idx_source, int nm, const int *mx, const int *mz,
                     int nr, const int *rx, const int *rz, ORC_FN(orc_adj_cb) cb, void *user,
                     ORC_REAL *grad_out, ORC_REAL *rec_out)
{
    const size_t XZ = (size_t)X * Z;
    ORC_FN(orc_fields) F, Fa, Fb;
    if (ORC_FN(alloc_fields)(&F, X, Z, T) || ORC_FN(alloc_fields)(&Fa, X, Z, T) ||
        ORC_FN(alloc_fields)(&Fb, X, Z, T))
        return -1;
    ORC_REAL *integ = (ORC_REAL *)calloc(ns > 0 ? ns : 1, sizeof(ORC_REAL));
    ORC_REAL *integ_a = (ORC_REAL *)calloc(nm > 0 ? nm : 1, sizeof(ORC_REAL));
    ORC_REAL *ring = (ORC_REAL *)calloc((size_t)(nr > 0 ? nr : 1) * T, sizeof(ORC_REAL));
    ORC_REAL *adj = (ORC_REAL *)calloc((size_t)(nm > 0 ? nm : 1) * T, sizeof(ORC_REAL));
    ORC_REAL *Pa = (ORC_REAL *)calloc(XZ, sizeof(ORC_REAL));
    ORC_REAL *Pb = (ORC_REAL *)calloc(XZ, sizeof(ORC_REAL));
    memset(rec_out, 0, sizeof(ORC_REAL) * (size_t)nm * T);
    memset(grad_out, 0, sizeof(ORC_REAL) * XZ);

    /* phase 1: forward with ring and sensor recording */
    for (int t = 1; t < T; t++) {
        ORC_FN(frame_p)(&F, t, cquad, d_x, d_z, constvec, 0);
        ORC_FN(inject)(&F, t, ns, sx, sz, src, integ, 0, idx_source);
        ORC_FN(record)(&F, t, nr, rx, rz, ring);
        ORC_FN(record)(&F, t, nm, mx, mz, rec_out);
        ORC_FN(frame_a)(&F, t, d_x, d_z, constvec, 0);
    }
    /* phase 1A: adjoint source */
    cb(rec_out, adj, user);
    /* reconstruction start: P(T-1), A(T-2) into slot 0 (regression_PML_single.cu:787-790) */
    memcpy(Fb.Px, F.Px + ((T - 1) % 2) * XZ, XZ * sizeof(ORC_REAL));
    memcpy(Fb.Pz, F.Pz + ((T - 1) % 2) * XZ, XZ * sizeof(ORC_REAL));
    memcpy(Fb.Ax, F.Ax + ((T - 2) % 2) * XZ, XZ * sizeof(ORC_REAL));
    memcpy(Fb.Az, F.Az + ((T - 2) % 2) * XZ, XZ * sizeof(ORC_REAL));

    /* phase 2 */
    for (int t = 0; t < T; t++) {
        if (t > 0) {
            ORC_FN(frame_p)(&Fa, t, cquad, d_x, d_z, constvec, 0);
            ORC_FN(frame_p)(&Fb, t, cquad, d_x, d_z, constvec, 1);
            ORC_FN(inject_r)(&Fa, t, nm, mx, mz, adj, integ_a);
            ORC_FN(set_ring)(&Fb, t, nr, rx, rz, ring);
            ORC_FN(frame_a)(&Fa, t, d_x, d_z, constvec, 0);
            ORC_FN(frame_a)(&Fb, t, d_x, d_z, constvec, 1);
        }
        /* somaFrames x2 (regression_PML_single.cu:815-816) */
        const ORC_REAL *pxa = Fa.Px + (t % 2) * XZ, *pza = Fa.Pz + (t % 2) * XZ;
        const ORC_REAL *pxb = Fb.Px + (t % 2) * XZ, *pzb = Fb.Pz + (t % 2) * XZ;
        for (size_t i = 0; i < XZ; i++) {
            Pa[i] = pxa[i] + pza[i];
            Pb[i] = pxb[i] + pzb[i];
        }
        /* calcGrad2 (regression_PML_single.cu:390-445): every cell */
#pragma omp parallel for schedule(static)
        for (int z = 0; z < Z; z++) {
            for (int x = 0; x < X; x++) {
                const ORC_REAL lap = ORC_FN(d2)(Pb, X, Z, x, z, 1, 0) + ORC_FN(d2)(Pb, X, Z, x, z, 0, 1);
                const size_t i = (size_t)x + (size_t)z * X;
                grad_out[i] = ORC_FMA(Pa[i], lap, grad_out[i]);
            }
        }
    }
    free(integ);
    free(integ_a);
    free(ring);
    free(adj);
    free(Pa);
    free(Pb);
    ORC_FN(free_fields)(&F);
    ORC_FN(free_fields)(&Fa);
    ORC_FN(free_fields)(&Fb);
    return 0;
}

#undef ORC_RND
#undef ORC_FMA
