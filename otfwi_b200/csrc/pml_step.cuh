// Fused time-step kernels for the 2D acoustic split-field PML.
//
// One launch advances every shot of a batch by one time step. A CTA owns a
// TX x TZ tile of cells of one shot and does, in one pass over HBM:
//   P half-step  P(t) = damp * P(t-1) + q * D-[A(t-1)]   over the tile + 4-cell
//                halo (halo recomputed instead of exchanged), into shared memory
//   point work   source / adjoint-source injection, ring overwrite (reverse)
//   recording    receivers and the boundary ring at owned cells (forward)
//   A half-step  A(t) = damp * A(t-1) + r * D+[P(t)]     at owned cells
//   imaging      grad += P_adj(t) * lap9(P_rec(t))       (reverse kernel)
// The reference launches 4 (forward) or 9 (reverse) kernels per step with a
// device synchronisation after each (regression_PML_single.cu:661-677,
// 793-834); here it is one launch, no synchronisation, replayed from a CUDA
// graph.
//
// Arithmetic follows regression_PML_single.cu:447-615 operation by operation
// (see Faithful below); Fast replaces only the FP64 staggered sums by an FP32
// antisymmetric-pair form.
#pragma once
#include "otf_common.cuh"

namespace otf {

// deriv_macros.h:85-95 (prec_deriv == 4) staggered-derivative weights
constexpr double kC0 = 1.196289e+00;
constexpr double kC1 = 7.975260e-02;
constexpr double kC2 = 9.570313e-03;
constexpr double kC3 = 6.975446e-04;

// Staggered first derivative at 4 consecutive cells from an 11-value window:
// cell j uses u[i] = w[j + i], u[i] = m[x - 3 - off + i] (off = 1 for the P
// update's D-, 0 for the A update's D+).
struct Faithful {
    // FP64 sum in the reference's order: "-c3*u7 + c2*u6 - c1*u5 + c0*u4 -
    // c0*u3 + c1*u2 - c2*u1 + c3*u0" with double literals contracts to the
    // leading negated product, rounded, then seven fused multiply-adds
    // (deriv_macros.h:85-108).
    __device__ __forceinline__ static void dstag4(const float *w, float *out)
    {
        double d[11];
#pragma unroll
        for (int i = 0; i < 11; i++)
            d[i] = (double)w[i];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            double s = __dmul_rn(-kC3, d[j + 7]);
            s = __fma_rn(kC2, d[j + 6], s);
            s = __fma_rn(-kC1, d[j + 5], s);
            s = __fma_rn(kC0, d[j + 4], s);
            s = __fma_rn(-kC0, d[j + 3], s);
            s = __fma_rn(kC1, d[j + 2], s);
            s = __fma_rn(-kC2, d[j + 1], s);
            s = __fma_rn(kC3, d[j + 0], s);
            out[j] = __double2float_rn(s);
        }
    }
};

struct Fast {
    // FP32: c0*(u4-u3) - c1*(u5-u2) + c2*(u6-u1) - c3*(u7-u0), c0 carried as
    // a hi+lo pair so the dominant weight has no systematic rounding bias.
    __device__ __forceinline__ static void dstag4(const float *w, float *out)
    {
        constexpr float c0h = (float)kC0;
        constexpr float c0l = (float)(kC0 - (double)(float)kC0);
        constexpr float c1 = (float)kC1, c2 = (float)kC2, c3 = (float)kC3;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const float *u = w + j;
            const float d0 = __fsub_rn(u[4], u[3]);
            const float d1 = __fsub_rn(u[5], u[2]);
            const float d2 = __fsub_rn(u[6], u[1]);
            const float d3 = __fsub_rn(u[7], u[0]);
            float s = __fmul_rn(-c3, d3);
            s = __fmaf_rn(c2, d2, s);
            s = __fmaf_rn(-c1, d1, s);
            s = __fmaf_rn(c0l, d0, s);
            s = __fmaf_rn(c0h, d0, s);
            out[j] = s;
        }
    }
};

// 9-point 8th-order second derivative at 4 consecutive cells from a
// 12-value window (cell j uses w[j..j+8], centre w[j+4]); FP32 with the
// reference's contraction: the leading "-9*m[+4]" product rounded, eight
// fused multiply-adds, IEEE division by 5040 (deriv_macros.h:110-135).
__device__ __forceinline__ void lap9_4(const float *w, float *out)
{
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const float *m = w + j + 4;  // m[k] = value at offset k
        float s = __fmul_rn(-9.0f, m[4]);
        s = __fmaf_rn(128.0f, m[3], s);
        s = __fmaf_rn(-1008.0f, m[2], s);
        s = __fmaf_rn(8064.0f, m[1], s);
        s = __fmaf_rn(-14350.0f, m[0], s);
        s = __fmaf_rn(8064.0f, m[-1], s);
        s = __fmaf_rn(-1008.0f, m[-2], s);
        s = __fmaf_rn(128.0f, m[-3], s);
        s = __fmaf_rn(-9.0f, m[-4], s);
        out[j] = __fdiv_rn(s, 5040.0f);
    }
}

// One wavefield set (split pressure Px/Pz, particle velocity Ax/Az) in the
// padded layout, shot 0 base pointers of the slot read and the slot written.
struct Fields {
    const float *px_in, *pz_in, *ax_in, *az_in;
    float *px_out, *pz_out, *ax_out, *az_out;
};

struct StepParams {
    int X, Z, pitch, rows, T, ntx;
    int64_t shot_stride;  // floats between shots in every field / grad buffer
    int t;                // time index being computed
    float r;              // dt/dx of the A update
    const float *q0;      // padded P coefficient of set 0
    const float *q1;      // padded P coefficient of set 1 (reverse kernel)
    const float *dampx, *dampz;    // separable: padded 1D 1 - d*dt (index by padded col / row)
    const float *dampx2, *dampz2;  // general: padded 2D 1 - d*dt
    Fields f0, f1;
    // point injection (forward: sources into f0; reverse: adjoint sources into f1)
    const int *inj_ptr;  // [n_shots + 1]
    const int *inj_x, *inj_z, *inj_row;
    const float *inj_tab;  // [rows][T] running integral of the injected series
    // receivers owned by each tile (forward recording)
    const int *sen_ptr, *sen_cell, *sen_id;  // [ntiles + 1], owned-local cell, receiver id
    float *rec;                              // [n_shots][n_sen][T]
    int n_sen;
    // boundary ring: owned cells (forward record; ring id = CSR position)
    const int *ringo_ptr, *ringo_cell;
    // ring cells inside each tile's halo-extended region (reverse overwrite)
    const int *ringe_ptr, *ringe_cell, *ringe_id;
    float *ring;  // [n_shots][T][n_ring]
    int n_ring;
    float *grad;  // padded [n_shots][rows][pitch]
    // strip-split (fast) kernels: per-tile flag (1 = the tile's halo region
    // holds damped or never-updated cells), per-tile point lists over the
    // halo region, and the firing table of sources per shot
    const int *tile_edge;                     // [ntiles]
    const int *srce_ptr, *srce_cell, *srce_id;  // sources in each tile's region
    const int *fire_row;                      // [n_shots][n_src]: tab row, -1 = silent
    int n_src;
    const int *rcve_ptr, *rcve_cell, *rcve_id;  // injectable receivers in each region
};

template <int TX, int TZ>
struct TileGeom {
    static_assert(TX % 4 == 0 && TZ % 4 == 0, "tile must be a multiple of 4 cells");
    static constexpr int EX = TX + 8, EZ = TZ + 8;      // P(t) region (tile + 4-cell halo)
    static constexpr int AXW = TX + 16, AXH = TZ + 8;   // Ax(t-1) tile: x halo 8, z halo 4
    static constexpr int AZW = TX + 8, AZH = TZ + 16;   // Az(t-1) tile: x halo 4, z halo 8
    static constexpr int NAX = AXW * AXH, NAZ = AZW * AZH, NE = EX * EZ, NO = TX * TZ;
    // v1 layout (one tile, A staged by the CTA itself)
    static constexpr int SAX = 0, SAZ = NAX, SPX = SAZ + NAZ, SPZ = SPX + NE;
    static constexpr int SMEM_FLOATS = SPZ + NE;
    // v2 stage (all inputs of one field set staged by TMA): Ax | Az | Px(t-1) | Pz(t-1) | q
    static constexpr int STAGE_FLOATS = NAX + NAZ + 3 * NE;
    static constexpr int NBEX = EX / 4, NBE = NBEX * (EZ / 4);  // 4x4 blocks of the P region
    static constexpr int NBOX = TX / 4, NBO = NBOX * (TZ / 4);  // 4x4 blocks of the owned tile
    static constexpr int KO = (NBO + NT - 1) / NT;               // owned blocks per thread
};

__device__ __forceinline__ float4 ld4(const float *base, int64_t idx)
{
    return __ldg(reinterpret_cast<const float4 *>(base + idx));
}
__device__ __forceinline__ float4 lds4(const float *base, int idx)
{
    return *reinterpret_cast<const float4 *>(base + idx);
}
__device__ __forceinline__ void f4a(const float4 v, float *a)
{
    a[0] = v.x;
    a[1] = v.y;
    a[2] = v.z;
    a[3] = v.w;
}

// Stage A(t-1) tiles (with halo) from global into shared memory, coalesced
// 16-byte loads; outside the allocation reads as zero (v1 kernels).
template <int TX, int TZ>
__device__ __forceinline__ void load_a_tiles(const StepParams &p, float *sAx_, float *sAz_,
                                             const float *ax, const float *az, int x0, int z0)
{
    using G = TileGeom<TX, TZ>;
    float4 *sAx = reinterpret_cast<float4 *>(sAx_);
    float4 *sAz = reinterpret_cast<float4 *>(sAz_);
    constexpr int AXW4 = G::AXW / 4, AZW4 = G::AZW / 4;
    for (int i = threadIdx.x; i < AXW4 * G::AXH; i += NT) {
        const int rr = i / AXW4, cc = i - rr * AXW4;
        const int prow = z0 - 4 + PAD + rr, pcol = x0 - 8 + PAD + 4 * cc;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (prow < p.rows && pcol < p.pitch)
            v = ld4(ax, (int64_t)prow * p.pitch + pcol);
        sAx[i] = v;
    }
    for (int i = threadIdx.x; i < AZW4 * G::AZH; i += NT) {
        const int rr = i / AZW4, cc = i - rr * AZW4;
        const int prow = z0 - 8 + PAD + rr, pcol = x0 - 4 + PAD + 4 * cc;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (prow < p.rows && pcol < p.pitch)
            v = ld4(az, (int64_t)prow * p.pitch + pcol);
        sAz[i] = v;
    }
}

__device__ __forceinline__ bool inb(const StepParams &p, int x, int z)
{
    return x >= 4 && z >= 4 && x < p.X - 4 && z < p.Z - 4;
}

// P half-step over the halo-extended region (simulateFrameP,
// regression_PML_single.cu:503-519), into sPx / sPz.
// TILED: P(t-1) and q are read from shared-memory E tiles (row stride EX);
// otherwise from the padded global arrays.
template <int TX, int TZ, class Prec, bool SEP, bool REVERT, bool TILED>
__device__ __forceinline__ void p_phase(const StepParams &p, const float *sAx, const float *sAz,
                                        float *sPx, float *sPz, const float *px_in,
                                        const float *pz_in, const float *q, int x0, int z0)
{
    using G = TileGeom<TX, TZ>;
    for (int b = threadIdx.x; b < G::NBE; b += NT) {
        const int ex = 4 * (b % G::NBEX), ez = 4 * (b / G::NBEX);
        float dAx[4][4], dAz[4][4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            float w[12];
            const float *row = sAx + (ez + i) * G::AXW + ex;
            f4a(lds4(row, 0), w);
            f4a(lds4(row, 4), w + 4);
            f4a(lds4(row, 8), w + 8);
            Prec::dstag4(w, dAx[i]);
        }
        {
            float wz[4][11];
#pragma unroll
            for (int k = 0; k < 11; k++) {
                const float4 v = lds4(sAz, (ez + k) * G::AZW + ex);
                wz[0][k] = v.x;
                wz[1][k] = v.y;
                wz[2][k] = v.z;
                wz[3][k] = v.w;
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                float o[4];
                Prec::dstag4(wz[j], o);
#pragma unroll
                for (int i = 0; i < 4; i++)
                    dAz[i][j] = o[i];
            }
        }
        const int xg = x0 - 4 + ex;  // first grid x of this block
        const int pcol = xg + PAD;
        float dmx[4] = {1.f, 1.f, 1.f, 1.f};
        if (SEP && pcol < p.pitch)
            f4a(ld4(p.dampx, pcol), dmx);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int zg = z0 - 4 + ez + i;
            const int prow = zg + PAD;
            float po_x[4] = {0.f, 0.f, 0.f, 0.f}, po_z[4] = {0.f, 0.f, 0.f, 0.f};
            float qv[4] = {0.f, 0.f, 0.f, 0.f};
            float dx2[4] = {1.f, 1.f, 1.f, 1.f}, dz2[4] = {1.f, 1.f, 1.f, 1.f};
            float dmz = 1.f;
            const bool ok = prow < p.rows && pcol < p.pitch;
            if (TILED) {
                const int e = (ez + i) * G::EX + ex;
                f4a(lds4(px_in, e), po_x);
                f4a(lds4(pz_in, e), po_z);
                f4a(lds4(q, e), qv);
            } else if (ok) {
                const int64_t o = (int64_t)prow * p.pitch + pcol;
                f4a(ld4(px_in, o), po_x);
                f4a(ld4(pz_in, o), po_z);
                f4a(ld4(q, o), qv);
            }
            if (!REVERT && ok) {
                if (SEP) {
                    dmz = __ldg(p.dampz + prow);
                } else {
                    const int64_t o = (int64_t)prow * p.pitch + pcol;
                    f4a(ld4(p.dampx2, o), dx2);
                    f4a(ld4(p.dampz2, o), dz2);
                }
            }
            float nx[4], nz[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                float vx, vz;
                if (!REVERT) {
                    const float mx = SEP ? dmx[j] : dx2[j];
                    const float mz = SEP ? dmz : dz2[j];
                    vx = __fmaf_rn(po_x[j], mx, __fmul_rn(qv[j], dAx[i][j]));
                    vz = __fmaf_rn(po_z[j], mz, __fmul_rn(qv[j], dAz[i][j]));
                } else {
                    vx = __fmaf_rn(-qv[j], dAx[i][j], po_x[j]);
                    vz = __fmaf_rn(-qv[j], dAz[i][j], po_z[j]);
                }
                const bool in = inb(p, xg + j, zg);
                nx[j] = in ? vx : 0.f;
                nz[j] = in ? vz : 0.f;
            }
            *reinterpret_cast<float4 *>(sPx + (ez + i) * G::EX + ex) = make_float4(nx[0], nx[1], nx[2], nx[3]);
            *reinterpret_cast<float4 *>(sPz + (ez + i) * G::EX + ex) = make_float4(nz[0], nz[1], nz[2], nz[3]);
        }
    }
}

// Point injection into P(t) in shared memory (somaFonteIntegral,
// regression_PML_single.cu:285-291): P += I(t)/2 on both split components.
template <int TX, int TZ>
__device__ __forceinline__ void inject(const StepParams &p, float *sPx, float *sPz, int shot, int x0,
                                       int z0)
{
    using G = TileGeom<TX, TZ>;
    const int b = p.inj_ptr[shot], e = p.inj_ptr[shot + 1];
    for (int k = b + threadIdx.x; k < e; k += NT) {
        const int ex = p.inj_x[k] - (x0 - 4), ez = p.inj_z[k] - (z0 - 4);
        if (ex >= 0 && ex < G::EX && ez >= 0 && ez < G::EZ) {
            const float h = __fmul_rn(p.inj_tab[(int64_t)p.inj_row[k] * p.T + p.t], 0.5f);
            atomicAdd(sPx + ez * G::EX + ex, h);
            atomicAdd(sPz + ez * G::EX + ex, h);
        }
    }
}

// setRec (regression_PML_single.cu:269-270): ring cells of the E region <- ring(T-1-t)/2
template <int TX, int TZ>
__device__ __forceinline__ void ring_overwrite(const StepParams &p, float *sPx, float *sPz, int shot,
                                               int tile)
{
    const float *ring = p.ring + ((int64_t)shot * p.T + (p.T - 1 - p.t)) * p.n_ring;
    for (int e = p.ringe_ptr[tile] + threadIdx.x; e < p.ringe_ptr[tile + 1]; e += NT) {
        const float v = __fmul_rn(ring[p.ringe_id[e]], 0.5f);
        sPx[p.ringe_cell[e]] = v;
        sPz[p.ringe_cell[e]] = v;
    }
}

// Receivers (and with RING the boundary ring) at owned cells, after injection
// (gravaBufferSensores, regression_PML_single.cu:758-759).
template <int TX, int TZ, bool RING>
__device__ __forceinline__ void record(const StepParams &p, const float *sPx, const float *sPz,
                                       int shot, int tile)
{
    using G = TileGeom<TX, TZ>;
    for (int e = p.sen_ptr[tile] + threadIdx.x; e < p.sen_ptr[tile + 1]; e += NT) {
        const int c = p.sen_cell[e];
        const int oz = c / TX, ox = c - oz * TX;
        const int s = (oz + 4) * G::EX + ox + 4;
        p.rec[((int64_t)shot * p.n_sen + p.sen_id[e]) * p.T + p.t] = __fadd_rn(sPx[s], sPz[s]);
    }
    if (RING) {
        float *ring = p.ring + ((int64_t)shot * p.T + p.t) * p.n_ring;
        for (int e = p.ringo_ptr[tile] + threadIdx.x; e < p.ringo_ptr[tile + 1]; e += NT) {
            const int c = p.ringo_cell[e];
            const int oz = c / TX, ox = c - oz * TX;
            const int s = (oz + 4) * G::EX + ox + 4;
            ring[e] = __fadd_rn(sPx[s], sPz[s]);
        }
    }
}

// Write P(t) of the owned tile from shared memory to the output slot.
template <int TX, int TZ>
__device__ __forceinline__ void store_p(const StepParams &p, const float *sPx, const float *sPz,
                                        float *px_out, float *pz_out, int x0, int z0)
{
    using G = TileGeom<TX, TZ>;
    constexpr int W4 = TX / 4;
    for (int i = threadIdx.x; i < W4 * TZ; i += NT) {
        const int oz = i / W4, ox = 4 * (i - oz * W4);
        const int prow = z0 + oz + PAD, pcol = x0 + ox + PAD;
        if (prow < p.rows && pcol < p.pitch) {
            const int64_t o = (int64_t)prow * p.pitch + pcol;
            const int s = (oz + 4) * G::EX + ox + 4;
            *reinterpret_cast<float4 *>(px_out + o) = lds4(sPx, s);
            *reinterpret_cast<float4 *>(pz_out + o) = lds4(sPz, s);
        }
    }
}

// A half-step at owned cells (simulateFrameA, regression_PML_single.cu:587-608).
// TILED: A(t-1) at owned cells is read from the staged A tiles; otherwise
// from global. With LAP, also returns lap9(Px + Pz) at the owned cells
// (calcGrad2's operand, regression_PML_single.cu:442) in lap[k] for the k-th
// owned block this thread handles.
template <int TX, int TZ, class Prec, bool SEP, bool REVERT, bool LAP, bool TILED>
__device__ __forceinline__ void a_phase(const StepParams &p, const float *sAx, const float *sAz,
                                        const float *sPx, const float *sPz, const float *ax_in,
                                        const float *az_in, float *ax_out, float *az_out, int x0,
                                        int z0, float (*lap)[16])
{
    using G = TileGeom<TX, TZ>;
#pragma unroll
    for (int k = 0; k < G::KO; k++) {
        const int b = threadIdx.x + k * NT;
        if (b >= G::NBO)
            break;
        const int ox = 4 * (b % G::NBOX), oz = 4 * (b / G::NBOX);
        float sx[4][4], sz[4][4];
        // x-derivatives: E rows oz+4+i, window E cols ox+1 .. ox+11
#pragma unroll
        for (int i = 0; i < 4; i++) {
            float wx[12], wz[12], ox4[4], oz4[4];
            const int r = (oz + 4 + i) * G::EX + ox;
            f4a(lds4(sPx, r), wx);
            f4a(lds4(sPx, r + 4), wx + 4);
            f4a(lds4(sPx, r + 8), wx + 8);
            f4a(lds4(sPz, r), wz);
            f4a(lds4(sPz, r + 4), wz + 4);
            f4a(lds4(sPz, r + 8), wz + 8);
            Prec::dstag4(wx + 1, ox4);
            Prec::dstag4(wz + 1, oz4);
#pragma unroll
            for (int j = 0; j < 4; j++)
                sx[i][j] = __fadd_rn(ox4[j], oz4[j]);
            if (LAP) {
                float ws[12], l[4];
#pragma unroll
                for (int c = 0; c < 12; c++)
                    ws[c] = __fadd_rn(wx[c], wz[c]);
                lap9_4(ws, l);
#pragma unroll
                for (int j = 0; j < 4; j++)
                    lap[k][i * 4 + j] = l[j];
            }
        }
        // z-derivatives: E rows oz+1 .. oz+11 at E cols ox+4 .. ox+7
        {
            float vx[4][11], vz[4][11];
#pragma unroll
            for (int c = 0; c < 11; c++) {
                const float4 a = lds4(sPx, (oz + 1 + c) * G::EX + ox + 4);
                const float4 bq = lds4(sPz, (oz + 1 + c) * G::EX + ox + 4);
                vx[0][c] = a.x; vx[1][c] = a.y; vx[2][c] = a.z; vx[3][c] = a.w;
                vz[0][c] = bq.x; vz[1][c] = bq.y; vz[2][c] = bq.z; vz[3][c] = bq.w;
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                float o1[4], o2[4];
                Prec::dstag4(vx[j], o1);
                Prec::dstag4(vz[j], o2);
#pragma unroll
                for (int i = 0; i < 4; i++)
                    sz[i][j] = __fadd_rn(o1[i], o2[i]);
            }
        }
        if (LAP) {
            // z part of the Laplacian: E rows oz .. oz+11
            float vs[4][12];
#pragma unroll
            for (int c = 0; c < 12; c++) {
                const float4 a = lds4(sPx, (oz + c) * G::EX + ox + 4);
                const float4 bq = lds4(sPz, (oz + c) * G::EX + ox + 4);
                vs[0][c] = __fadd_rn(a.x, bq.x);
                vs[1][c] = __fadd_rn(a.y, bq.y);
                vs[2][c] = __fadd_rn(a.z, bq.z);
                vs[3][c] = __fadd_rn(a.w, bq.w);
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                float l[4];
                lap9_4(vs[j], l);
#pragma unroll
                for (int i = 0; i < 4; i++)
                    lap[k][i * 4 + j] = __fadd_rn(lap[k][i * 4 + j], l[i]);
            }
        }
        const int xg = x0 + ox, pcol = xg + PAD;
        float dmx[4] = {1.f, 1.f, 1.f, 1.f};
        if (SEP && !REVERT && pcol < p.pitch)
            f4a(ld4(p.dampx, pcol), dmx);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int zg = z0 + oz + i, prow = zg + PAD;
            if (prow >= p.rows || pcol >= p.pitch)
                continue;
            const int64_t o = (int64_t)prow * p.pitch + pcol;
            float ao_x[4], ao_z[4];
            if (TILED) {
                f4a(lds4(sAx, (oz + 4 + i) * G::AXW + ox + 8), ao_x);
                f4a(lds4(sAz, (oz + 8 + i) * G::AZW + ox + 4), ao_z);
            } else {
                f4a(ld4(ax_in, o), ao_x);
                f4a(ld4(az_in, o), ao_z);
            }
            float dx2[4] = {1.f, 1.f, 1.f, 1.f}, dz2[4] = {1.f, 1.f, 1.f, 1.f};
            float dmz = 1.f;
            if (!REVERT) {
                if (SEP) {
                    dmz = __ldg(p.dampz + prow);
                } else {
                    f4a(ld4(p.dampx2, o), dx2);
                    f4a(ld4(p.dampz2, o), dz2);
                }
            }
            float nx[4], nz[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                float vx, vz;
                if (!REVERT) {
                    const float mx = SEP ? dmx[j] : dx2[j];
                    const float mz = SEP ? dmz : dz2[j];
                    vx = __fmaf_rn(ao_x[j], mx, __fmul_rn(p.r, sx[i][j]));
                    vz = __fmaf_rn(ao_z[j], mz, __fmul_rn(p.r, sz[i][j]));
                } else {
                    vx = __fmaf_rn(-p.r, sx[i][j], ao_x[j]);
                    vz = __fmaf_rn(-p.r, sz[i][j], ao_z[j]);
                }
                const bool in = inb(p, xg + j, zg);
                nx[j] = in ? vx : 0.f;
                nz[j] = in ? vz : 0.f;
            }
            *reinterpret_cast<float4 *>(ax_out + o) = make_float4(nx[0], nx[1], nx[2], nx[3]);
            *reinterpret_cast<float4 *>(az_out + o) = make_float4(nz[0], nz[1], nz[2], nz[3]);
        }
    }
}

// Imaging condition at owned cells (calcGrad2, regression_PML_single.cu:442-443):
// grad += (Px + Pz)(t) * lap. g_in: shared tile (row stride TX) when TILED,
// else the global gradient itself.
template <int TX, int TZ, bool TILED>
__device__ __forceinline__ void image(const StepParams &p, const float *sPx, const float *sPz,
                                      const float *g_tile, float *grad, int x0, int z0,
                                      const float (*lap)[16])
{
    using G = TileGeom<TX, TZ>;
#pragma unroll
    for (int k = 0; k < G::KO; k++) {
        const int b = threadIdx.x + k * NT;
        if (b >= G::NBO)
            break;
        const int ox = 4 * (b % G::NBOX), oz = 4 * (b / G::NBOX);
        const int pcol = x0 + ox + PAD;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int prow = z0 + oz + i + PAD;
            if (prow >= p.rows || pcol >= p.pitch)
                continue;
            const int64_t o = (int64_t)prow * p.pitch + pcol;
            const float4 a = lds4(sPx, (oz + 4 + i) * G::EX + ox + 4);
            const float4 bq = lds4(sPz, (oz + 4 + i) * G::EX + ox + 4);
            float4 g = TILED ? lds4(g_tile, (oz + i) * TX + ox) : *reinterpret_cast<float4 *>(grad + o);
            g.x = __fmaf_rn(__fadd_rn(a.x, bq.x), lap[k][i * 4 + 0], g.x);
            g.y = __fmaf_rn(__fadd_rn(a.y, bq.y), lap[k][i * 4 + 1], g.y);
            g.z = __fmaf_rn(__fadd_rn(a.z, bq.z), lap[k][i * 4 + 2], g.z);
            g.w = __fmaf_rn(__fadd_rn(a.w, bq.w), lap[k][i * 4 + 3], g.w);
            *reinterpret_cast<float4 *>(grad + o) = g;
        }
    }
}

// ---------------------------------------------------------------------------
// v1 kernels: one launch per time step, one tile per CTA, A(t-1) staged by
// the CTA's own loads.

// Forward step: cuda_simulate / cuda_grad_ext phase 1 body
// (regression_PML_single.cu:661-677, 745-764): P update, source injection,
// receiver (and with RING, boundary-ring) recording, A update.
template <int TX, int TZ, class Prec, bool SEP, bool RING>
__global__ void __launch_bounds__(NT) k_forward_step(const StepParams p)
{
    extern __shared__ float4 smem4[];
    float *sm = reinterpret_cast<float *>(smem4);
    using G = TileGeom<TX, TZ>;
    float *sAx = sm + G::SAX, *sAz = sm + G::SAZ, *sPx = sm + G::SPX, *sPz = sm + G::SPZ;
    const int tile = blockIdx.x, shot = blockIdx.y;
    const int x0 = (tile % p.ntx) * TX, z0 = (tile / p.ntx) * TZ;
    const int64_t so = p.shot_stride * shot;
    const Fields &f = p.f0;

    load_a_tiles<TX, TZ>(p, sAx, sAz, f.ax_in + so, f.az_in + so, x0, z0);
    __syncthreads();
    p_phase<TX, TZ, Prec, SEP, false, false>(p, sAx, sAz, sPx, sPz, f.px_in + so, f.pz_in + so, p.q0,
                                             x0, z0);
    __syncthreads();
    inject<TX, TZ>(p, sPx, sPz, shot, x0, z0);
    __syncthreads();
    store_p<TX, TZ>(p, sPx, sPz, f.px_out + so, f.pz_out + so, x0, z0);
    record<TX, TZ, RING>(p, sPx, sPz, shot, tile);
    a_phase<TX, TZ, Prec, SEP, false, false, false>(p, sAx, sAz, sPx, sPz, f.ax_in + so, f.az_in + so,
                                                    f.ax_out + so, f.az_out + so, x0, z0, nullptr);
}

// Reverse step: cuda_grad_ext phase 2 body (regression_PML_single.cu:795-825)
// for one t: set 0 = time-reversed reconstruction of the forward field
// (undamped, ring overwrite), set 1 = damped adjoint field with the
// time-flipped adjoint source injected at the receivers, then
// grad += (Px1+Pz1)(t) * lap9(Px0+Pz0)(t).
template <int TX, int TZ, class Prec, bool SEP>
__global__ void __launch_bounds__(NT) k_reverse_step(const StepParams p)
{
    extern __shared__ float4 smem4[];
    float *sm = reinterpret_cast<float *>(smem4);
    using G = TileGeom<TX, TZ>;
    float *sAx = sm + G::SAX, *sAz = sm + G::SAZ, *sPx = sm + G::SPX, *sPz = sm + G::SPZ;
    const int tile = blockIdx.x, shot = blockIdx.y;
    const int x0 = (tile % p.ntx) * TX, z0 = (tile / p.ntx) * TZ;
    const int64_t so = p.shot_stride * shot;
    float lap[G::KO][16];

    // reconstruction
    load_a_tiles<TX, TZ>(p, sAx, sAz, p.f0.ax_in + so, p.f0.az_in + so, x0, z0);
    __syncthreads();
    p_phase<TX, TZ, Prec, SEP, true, false>(p, sAx, sAz, sPx, sPz, p.f0.px_in + so, p.f0.pz_in + so,
                                            p.q0, x0, z0);
    __syncthreads();
    ring_overwrite<TX, TZ>(p, sPx, sPz, shot, tile);
    __syncthreads();
    store_p<TX, TZ>(p, sPx, sPz, p.f0.px_out + so, p.f0.pz_out + so, x0, z0);
    a_phase<TX, TZ, Prec, SEP, true, true, false>(p, sAx, sAz, sPx, sPz, p.f0.ax_in + so,
                                                  p.f0.az_in + so, p.f0.ax_out + so, p.f0.az_out + so,
                                                  x0, z0, lap);
    __syncthreads();

    // adjoint
    load_a_tiles<TX, TZ>(p, sAx, sAz, p.f1.ax_in + so, p.f1.az_in + so, x0, z0);
    __syncthreads();
    p_phase<TX, TZ, Prec, SEP, false, false>(p, sAx, sAz, sPx, sPz, p.f1.px_in + so, p.f1.pz_in + so,
                                             p.q1, x0, z0);
    __syncthreads();
    inject<TX, TZ>(p, sPx, sPz, shot, x0, z0);
    __syncthreads();
    store_p<TX, TZ>(p, sPx, sPz, p.f1.px_out + so, p.f1.pz_out + so, x0, z0);
    a_phase<TX, TZ, Prec, SEP, false, false, false>(p, sAx, sAz, sPx, sPz, p.f1.ax_in + so,
                                                    p.f1.az_in + so, p.f1.ax_out + so,
                                                    p.f1.az_out + so, x0, z0, nullptr);
    image<TX, TZ, false>(p, sPx, sPz, nullptr, p.grad + so, x0, z0, lap);
}

}  // namespace otf
