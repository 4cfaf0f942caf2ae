// Strip-split step kernels for the fast numerics (FP32 staggered sums).
//
// The reference keeps both split components Px, Pz of the pressure on every
// cell (regression_PML_single.cu:512-513), although they differ only where
// the PML damps: with d = 0 both evolve as P += q*D-[A] and only their sum
// is ever read (receivers, ring, the A update, the imaging condition). Here
// a field set is (P, Q, Ax, Az) with P the total pressure on every cell and
// Q = Px only on damped ("strip") cells:
//   strip cell:   Q' = Q*dmx + q*D-xAx,  Pz' = (P - Q)*dmz + q*D-zAz,  P' = Q' + Pz'
//   other cells:  P' = P + q*(D-xAx + D-zAz)
//   A update:     A' = A*dm + r*D+[P']       (two staggered sums instead of four)
// Tiles whose halo region holds no damped or never-updated cell skip the
// strip logic, the damping and the bounds tests altogether and never touch
// Q, so interior tiles move 28 bytes per cell-step (P, Ax, Az read + write,
// q read). The time-reversed reconstruction is undamped everywhere and needs
// no Q at all. Injection happens inside the P half-step (per-tile point
// lists), which removes a block barrier per item.
//
// Same persistent, TMA-pipelined structure as pml_step_tma.cuh, with
// NTH threads per CTA and 4 x BH register blocks.
#pragma once
#include "pml_step_tma.cuh"

namespace otf {

template <int TX, int TZ, int BH, int NTH>
struct SplitGeom {
    static_assert(TX % 4 == 0 && TZ % BH == 0 && (TZ + 8) % BH == 0, "tile / block mismatch");
    static constexpr int EX = TX + 8, EZ = TZ + 8;
    static constexpr int AXW = TX + 16, AXH = TZ + 8;
    static constexpr int AZW = TX + 8, AZH = TZ + 16;
    static constexpr int NAX = AXW * AXH, NAZ = AZW * AZH, NE = EX * EZ, NO = TX * TZ;
    static constexpr int STAGE = NAX + NAZ + 3 * NE;  // Ax | Az | P | Q | q
    static constexpr int NBEX = EX / 4, NBE = NBEX * (EZ / BH), KE = (NBE + NTH - 1) / NTH;
    static constexpr int NBOX = TX / 4, NBO = NBOX * (TZ / BH), KO = (NBO + NTH - 1) / NTH;
    static constexpr int FWD_FLOATS = 2 * STAGE + NE;
    static constexpr int REV_FLOATS = 2 * STAGE + NO + NE;
    static constexpr size_t FWD_BYTES = sizeof(float) * FWD_FLOATS + 2 * sizeof(uint64_t);
    static constexpr size_t REV_BYTES = sizeof(float) * REV_FLOATS + 2 * sizeof(uint64_t);
};

// FP32 staggered first derivative at N consecutive cells from N+7 values
// (the Fast pair form of pml_step.cuh).
template <int N>
__device__ __forceinline__ void dstag_n(const float *w, float *out)
{
    constexpr float c0h = (float)kC0;
    constexpr float c0l = (float)(kC0 - (double)(float)kC0);
    constexpr float c1 = (float)kC1, c2 = (float)kC2, c3 = (float)kC3;
#pragma unroll
    for (int j = 0; j < N; j++) {
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

// 9-point second-derivative tap sums (the weights times 5040) at N
// consecutive cells from N+8 values; lap_combine turns the x and z sums into
// the Laplacian with one rounded scaling instead of a division per axis.
template <int N>
__device__ __forceinline__ void lap_n(const float *w, float *out)
{
#pragma unroll
    for (int j = 0; j < N; j++) {
        const float *m = w + j + 4;
        float s = __fmul_rn(-9.0f, m[4]);
        s = __fmaf_rn(128.0f, m[3], s);
        s = __fmaf_rn(-1008.0f, m[2], s);
        s = __fmaf_rn(8064.0f, m[1], s);
        s = __fmaf_rn(-14350.0f, m[0], s);
        s = __fmaf_rn(8064.0f, m[-1], s);
        s = __fmaf_rn(-1008.0f, m[-2], s);
        s = __fmaf_rn(128.0f, m[-3], s);
        s = __fmaf_rn(-9.0f, m[-4], s);
        out[j] = s;
    }
}

__device__ __forceinline__ float lap_combine(float sx, float sz)
{
    constexpr float inv = (float)(1.0 / 5040.0);
    return __fmul_rn(__fadd_rn(sx, sz), inv);
}

enum Inject : int { kInjNone = 0, kInjSources = 1, kInjReceivers = 2 };

// P half-step over the halo-extended region into sP. EDGE: the tile's region
// holds strip or never-updated cells (uniform per item). Owned Q(t) is
// written to q_out (damped steps of edge tiles).
template <int TX, int TZ, int BH, int NTH, bool EDGE, bool REVERT, int INJ>
__device__ __forceinline__ void p_split(const StepParams &p, const float *sAx, const float *sAz,
                                        const float *sPo, const float *sQo, const float *sq, float *sP,
                                        float *q_out, int x0, int z0, int shot, int tile)
{
    using G = SplitGeom<TX, TZ, BH, NTH>;
#pragma unroll
    for (int kb = 0; kb < G::KE; kb++) {
        const int b = threadIdx.x + kb * NTH;
        if (b >= G::NBE)
            break;
        const int ex = 4 * (b % G::NBEX), ez = BH * (b / G::NBEX);
        float dAx[BH][4], dAz[BH][4];
#pragma unroll
        for (int i = 0; i < BH; i++) {
            float w[12];
            const int r = (ez + i) * G::AXW + ex;
            f4a(lds4(sAx, r), w);
            f4a(lds4(sAx, r + 4), w + 4);
            f4a(lds4(sAx, r + 8), w + 8);
            dstag_n<4>(w, dAx[i]);
        }
        {
            float wz[4][BH + 7];
#pragma unroll
            for (int k = 0; k < BH + 7; k++) {
                const float4 v = lds4(sAz, (ez + k) * G::AZW + ex);
                wz[0][k] = v.x;
                wz[1][k] = v.y;
                wz[2][k] = v.z;
                wz[3][k] = v.w;
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                float o[BH];
                dstag_n<BH>(wz[j], o);
#pragma unroll
                for (int i = 0; i < BH; i++)
                    dAz[i][j] = o[i];
            }
        }
        const int xg = x0 - 4 + ex, zg0 = z0 - 4 + ez;
        float dmx[4] = {1.f, 1.f, 1.f, 1.f};
        if (EDGE && !REVERT && xg + PAD < p.pitch)
            f4a(ld4(p.dampx, xg + PAD), dmx);
        float pn[BH][4], qn[BH][4];
        bool strip[BH][4];
#pragma unroll
        for (int i = 0; i < BH; i++) {
            const int e = (ez + i) * G::EX + ex;
            float po[4], qv[4];
            f4a(lds4(sPo, e), po);
            f4a(lds4(sq, e), qv);
            const int zg = zg0 + i;
            float dmz = 1.f;
            if (EDGE && !REVERT && zg + PAD < p.rows)
                dmz = __ldg(p.dampz + zg + PAD);
            float qo[4] = {0.f, 0.f, 0.f, 0.f};
            if (EDGE && !REVERT)
                f4a(lds4(sQo, e), qo);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const float s = __fadd_rn(dAx[i][j], dAz[i][j]);
                strip[i][j] = false;
                qn[i][j] = 0.f;
                if (REVERT) {
                    pn[i][j] = __fmaf_rn(-qv[j], s, po[j]);
                } else if (!EDGE) {
                    pn[i][j] = __fmaf_rn(qv[j], s, po[j]);
                } else if (dmx[j] != 1.f || dmz != 1.f) {
                    strip[i][j] = true;
                    const float q1 = __fmaf_rn(qo[j], dmx[j], __fmul_rn(qv[j], dAx[i][j]));
                    const float z1 = __fmaf_rn(__fsub_rn(po[j], qo[j]), dmz, __fmul_rn(qv[j], dAz[i][j]));
                    qn[i][j] = q1;
                    pn[i][j] = __fadd_rn(q1, z1);
                } else {
                    pn[i][j] = __fmaf_rn(qv[j], s, po[j]);
                }
                if (EDGE && !inb(p, xg + j, zg)) {
                    pn[i][j] = 0.f;
                    qn[i][j] = 0.f;
                }
            }
        }
        // point injection: P += I(t) (= I/2 on each split component), Q += I/2 on strip cells
        if (INJ != kInjNone) {
            const int *ptr = INJ == kInjSources ? p.srce_ptr : p.rcve_ptr;
            const int *cell = INJ == kInjSources ? p.srce_cell : p.rcve_cell;
            const int *id = INJ == kInjSources ? p.srce_id : p.rcve_id;
            for (int e = ptr[tile]; e < ptr[tile + 1]; e++) {
                const int c = cell[e];
                const int cz = c / G::EX - ez, cx = c - (c / G::EX) * G::EX - ex;
                if (cx < 0 || cx >= 4 || cz < 0 || cz >= BH)
                    continue;
                const int row = INJ == kInjSources ? p.fire_row[shot * p.n_src + id[e]]
                                                   : shot * p.n_sen + id[e];
                if (row < 0)
                    continue;
                const float I = p.inj_tab[(int64_t)row * p.T + p.t];
#pragma unroll
                for (int i = 0; i < BH; i++)
#pragma unroll
                    for (int j = 0; j < 4; j++)
                        if (i == cz && j == cx) {
                            pn[i][j] = __fadd_rn(pn[i][j], I);
                            if (strip[i][j])
                                qn[i][j] = __fadd_rn(qn[i][j], __fmul_rn(I, 0.5f));
                        }
            }
        }
#pragma unroll
        for (int i = 0; i < BH; i++)
            *reinterpret_cast<float4 *>(sP + (ez + i) * G::EX + ex) =
                make_float4(pn[i][0], pn[i][1], pn[i][2], pn[i][3]);
        // Q(t) of owned blocks (a 4 x BH block lies wholly in the halo or wholly owned)
        if (EDGE && !REVERT && ex >= 4 && ex < TX + 4 && ez >= 4 && ez < TZ + 4) {
#pragma unroll
            for (int i = 0; i < BH; i++) {
                const int prow = zg0 + i + PAD, pcol = xg + PAD;
                if (prow < p.rows && pcol < p.pitch)
                    *reinterpret_cast<float4 *>(q_out + (int64_t)prow * p.pitch + pcol) =
                        make_float4(qn[i][0], qn[i][1], qn[i][2], qn[i][3]);
            }
        }
    }
}

// A half-step at owned cells from the total pressure; with LAP also the
// 9-point Laplacian of P at owned cells into lap[k][i*4+j].
template <int TX, int TZ, int BH, int NTH, bool EDGE, bool REVERT, bool LAP>
__device__ __forceinline__ void a_split(const StepParams &p, const float *sAx, const float *sAz,
                                        const float *sP, float *ax_out, float *az_out, int x0, int z0,
                                        float (*lap)[4 * BH])
{
    using G = SplitGeom<TX, TZ, BH, NTH>;
#pragma unroll
    for (int kb = 0; kb < G::KO; kb++) {
        const int b = threadIdx.x + kb * NTH;
        if (b >= G::NBO)
            break;
        const int ox = 4 * (b % G::NBOX), oz = BH * (b / G::NBOX);
        float dx[BH][4], dz[BH][4];
#pragma unroll
        for (int i = 0; i < BH; i++) {
            float w[12];
            const int r = (oz + 4 + i) * G::EX + ox;
            f4a(lds4(sP, r), w);
            f4a(lds4(sP, r + 4), w + 4);
            f4a(lds4(sP, r + 8), w + 8);
            dstag_n<4>(w + 1, dx[i]);
            if (LAP)
                lap_n<4>(w, lap[kb] + 4 * i);
        }
        {
            float v[4][BH + 8];
#pragma unroll
            for (int c = 0; c < BH + 8; c++) {
                const float4 a = lds4(sP, (oz + c) * G::EX + ox + 4);
                v[0][c] = a.x;
                v[1][c] = a.y;
                v[2][c] = a.z;
                v[3][c] = a.w;
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                float o[BH];
                dstag_n<BH>(v[j] + 1, o);
#pragma unroll
                for (int i = 0; i < BH; i++)
                    dz[i][j] = o[i];
                if (LAP) {
                    float l[BH];
                    lap_n<BH>(v[j], l);
#pragma unroll
                    for (int i = 0; i < BH; i++)
                        lap[kb][4 * i + j] = lap_combine(lap[kb][4 * i + j], l[i]);
                }
            }
        }
        const int xg = x0 + ox, pcol = xg + PAD;
        float dmx[4] = {1.f, 1.f, 1.f, 1.f};
        if (EDGE && !REVERT && pcol < p.pitch)
            f4a(ld4(p.dampx, pcol), dmx);
#pragma unroll
        for (int i = 0; i < BH; i++) {
            const int zg = z0 + oz + i, prow = zg + PAD;
            if (prow >= p.rows || pcol >= p.pitch)
                continue;
            float ax[4], az[4];
            f4a(lds4(sAx, (oz + 4 + i) * G::AXW + ox + 8), ax);
            f4a(lds4(sAz, (oz + 8 + i) * G::AZW + ox + 4), az);
            const float dmz = (EDGE && !REVERT) ? __ldg(p.dampz + prow) : 1.f;
            float nx[4], nz[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (REVERT) {
                    nx[j] = __fmaf_rn(-p.r, dx[i][j], ax[j]);
                    nz[j] = __fmaf_rn(-p.r, dz[i][j], az[j]);
                } else if (!EDGE) {
                    nx[j] = __fmaf_rn(p.r, dx[i][j], ax[j]);
                    nz[j] = __fmaf_rn(p.r, dz[i][j], az[j]);
                } else {
                    nx[j] = __fmaf_rn(ax[j], dmx[j], __fmul_rn(p.r, dx[i][j]));
                    nz[j] = __fmaf_rn(az[j], dmz, __fmul_rn(p.r, dz[i][j]));
                }
                if (EDGE && !inb(p, xg + j, zg)) {
                    nx[j] = 0.f;
                    nz[j] = 0.f;
                }
            }
            const int64_t o = (int64_t)prow * p.pitch + pcol;
            *reinterpret_cast<float4 *>(ax_out + o) = make_float4(nx[0], nx[1], nx[2], nx[3]);
            *reinterpret_cast<float4 *>(az_out + o) = make_float4(nz[0], nz[1], nz[2], nz[3]);
        }
    }
}

template <int TX, int TZ>
__device__ __forceinline__ void store_p1(const StepParams &p, const float *sP, float *p_out, int x0, int z0,
                                         int nth)
{
    constexpr int EX = TX + 8, W4 = TX / 4;
    for (int i = threadIdx.x; i < W4 * TZ; i += nth) {
        const int oz = i / W4, ox = 4 * (i - oz * W4);
        const int prow = z0 + oz + PAD, pcol = x0 + ox + PAD;
        if (prow < p.rows && pcol < p.pitch)
            *reinterpret_cast<float4 *>(p_out + (int64_t)prow * p.pitch + pcol) =
                lds4(sP, (oz + 4) * EX + ox + 4);
    }
}

template <int TX, int TZ, bool RING>
__device__ __forceinline__ void record1(const StepParams &p, const float *sP, int shot, int tile, int nth)
{
    constexpr int EX = TX + 8;
    for (int e = p.sen_ptr[tile] + threadIdx.x; e < p.sen_ptr[tile + 1]; e += nth) {
        const int c = p.sen_cell[e];
        const int oz = c / TX, ox = c - oz * TX;
        p.rec[((int64_t)shot * p.n_sen + p.sen_id[e]) * p.T + p.t] = sP[(oz + 4) * EX + ox + 4];
    }
    if (RING) {
        float *ring = p.ring + ((int64_t)shot * p.T + p.t) * p.n_ring;
        for (int e = p.ringo_ptr[tile] + threadIdx.x; e < p.ringo_ptr[tile + 1]; e += nth) {
            const int c = p.ringo_cell[e];
            const int oz = c / TX, ox = c - oz * TX;
            ring[e] = sP[(oz + 4) * EX + ox + 4];
        }
    }
}

// setRec on the total pressure: P = ring(T-1-t) (= ring/2 + ring/2)
__device__ __forceinline__ void ring_overwrite1(const StepParams &p, float *sP, int shot, int tile, int nth)
{
    const float *ring = p.ring + ((int64_t)shot * p.T + (p.T - 1 - p.t)) * p.n_ring;
    for (int e = p.ringe_ptr[tile] + threadIdx.x; e < p.ringe_ptr[tile + 1]; e += nth)
        sP[p.ringe_cell[e]] = ring[p.ringe_id[e]];
}

template <int TX, int TZ, int BH, int NTH>
__device__ __forceinline__ void image1(const StepParams &p, const float *sP, const float *gt, float *grad,
                                       int x0, int z0, const float (*lap)[4 * BH])
{
    using G = SplitGeom<TX, TZ, BH, NTH>;
#pragma unroll
    for (int kb = 0; kb < G::KO; kb++) {
        const int b = threadIdx.x + kb * NTH;
        if (b >= G::NBO)
            break;
        const int ox = 4 * (b % G::NBOX), oz = BH * (b / G::NBOX);
        const int pcol = x0 + ox + PAD;
#pragma unroll
        for (int i = 0; i < BH; i++) {
            const int prow = z0 + oz + i + PAD;
            if (prow >= p.rows || pcol >= p.pitch)
                continue;
            const float4 a = lds4(sP, (oz + 4 + i) * G::EX + ox + 4);
            float4 g = lds4(gt, (oz + i) * TX + ox);
            g.x = __fmaf_rn(a.x, lap[kb][4 * i + 0], g.x);
            g.y = __fmaf_rn(a.y, lap[kb][4 * i + 1], g.y);
            g.z = __fmaf_rn(a.z, lap[kb][4 * i + 2], g.z);
            g.w = __fmaf_rn(a.w, lap[kb][4 * i + 3], g.w);
            *reinterpret_cast<float4 *>(grad + (int64_t)prow * p.pitch + pcol) = g;
        }
    }
}

// Copies of one field set's inputs for one item: Ax, Az, P and q always, Q
// only when WITH_Q (damped step of an edge tile), the gradient tile when gt.
template <int TX, int TZ, int BH, int NTH>
__device__ __forceinline__ void issue_split(const TmaParams &P, const SetMaps &m, int pin, int ain,
                                            const CUtensorMap *q, float *stage, uint64_t *bar, int item,
                                            bool with_q, float *gt)
{
    using G = SplitGeom<TX, TZ, BH, NTH>;
    int shot, tile, x0, z0;
    item_origin(P, item, TX, TZ, shot, tile, x0, z0);
    const uint32_t bytes = sizeof(float) * (G::NAX + G::NAZ + (with_q ? 3 : 2) * G::NE) +
                           (gt ? (uint32_t)(sizeof(float) * G::NO) : 0u);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_arrive_expect_tx(bar, bytes);
    tma_load_3d(stage, &m.ax[ain], x0 - 8 + PAD, z0 - 4 + PAD, shot, bar);
    tma_load_3d(stage + G::NAX, &m.az[ain], x0 - 4 + PAD, z0 - 8 + PAD, shot, bar);
    tma_load_3d(stage + G::NAX + G::NAZ, &m.px[pin], x0 - 4 + PAD, z0 - 4 + PAD, shot, bar);
    if (with_q)
        tma_load_3d(stage + G::NAX + G::NAZ + G::NE, &m.pz[pin], x0 - 4 + PAD, z0 - 4 + PAD, shot, bar);
    tma_load_3d(stage + G::NAX + G::NAZ + 2 * G::NE, q, x0 - 4 + PAD, z0 - 4 + PAD, 0, bar);
    if (gt)
        tma_load_3d(gt, &P.grad, x0 + PAD, z0 + PAD, shot, bar);
}

__device__ __forceinline__ int item_edge(const TmaParams &P, int item)
{
    return P.p.tile_edge[item % P.n_tiles];
}

template <int TX, int TZ, int BH, int NTH, bool RING, int MINB>
__global__ void __launch_bounds__(NTH, MINB) k_forward_split(const __grid_constant__ TmaParams P)
{
    using G = SplitGeom<TX, TZ, BH, NTH>;
    extern __shared__ __align__(128) float smf[];
    const StepParams &p = P.p;
    float *stage0 = smf, *stage1 = smf + G::STAGE;
    float *sP = smf + 2 * G::STAGE;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sP + G::NE);
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_barrier_init();
    }
    __syncthreads();
    int item = blockIdx.x;
    if (threadIdx.x == 0 && item < P.n_items)
        issue_split<TX, TZ, BH, NTH>(P, P.s0, P.s0_p_in, P.s0_a_in, &P.qf, stage0, &bar[0], item,
                                     item_edge(P, item) != 0, nullptr);
    for (int k = 0; item < P.n_items; k++, item += gridDim.x) {
        const int st = k & 1;
        float *S = st ? stage1 : stage0;
        const int next = item + gridDim.x;
        if (threadIdx.x == 0 && next < P.n_items)
            issue_split<TX, TZ, BH, NTH>(P, P.s0, P.s0_p_in, P.s0_a_in, &P.qf, st ? stage0 : stage1,
                                         &bar[st ^ 1], next, item_edge(P, next) != 0, nullptr);
        const bool ok = mbar_wait(&bar[st], (k >> 1) & 1, P.err);
        if (__syncthreads_or(!ok)) {
            drain(&bar[st], (k >> 1) & 1, next < P.n_items ? &bar[st ^ 1] : nullptr, ((k + 1) >> 1) & 1);
            return;
        }
        int shot, tile, x0, z0;
        item_origin(P, item, TX, TZ, shot, tile, x0, z0);
        const int64_t so = p.shot_stride * shot;
        const float *sAx = S, *sAz = S + G::NAX, *sPo = S + G::NAX + G::NAZ;
        const float *sQo = sPo + G::NE, *sq = sPo + 2 * G::NE;
        const bool edge = p.tile_edge[tile] != 0;
        if (edge)
            p_split<TX, TZ, BH, NTH, true, false, kInjSources>(p, sAx, sAz, sPo, sQo, sq, sP,
                                                               p.f0.pz_out + so, x0, z0, shot, tile);
        else
            p_split<TX, TZ, BH, NTH, false, false, kInjSources>(p, sAx, sAz, sPo, sQo, sq, sP, nullptr,
                                                                x0, z0, shot, tile);
        __syncthreads();
        store_p1<TX, TZ>(p, sP, p.f0.px_out + so, x0, z0, NTH);
        record1<TX, TZ, RING>(p, sP, shot, tile, NTH);
        if (edge)
            a_split<TX, TZ, BH, NTH, true, false, false>(p, sAx, sAz, sP, p.f0.ax_out + so,
                                                         p.f0.az_out + so, x0, z0, nullptr);
        else
            a_split<TX, TZ, BH, NTH, false, false, false>(p, sAx, sAz, sP, p.f0.ax_out + so,
                                                          p.f0.az_out + so, x0, z0, nullptr);
        __syncthreads();
    }
}

template <int TX, int TZ, int BH, int NTH, int MINB>
__global__ void __launch_bounds__(NTH, MINB) k_reverse_split(const __grid_constant__ TmaParams P)
{
    using G = SplitGeom<TX, TZ, BH, NTH>;
    extern __shared__ __align__(128) float smf[];
    const StepParams &p = P.p;
    float *bufR = smf, *bufA = smf + G::STAGE;
    float *gt = bufA + G::STAGE;
    float *sP = gt + G::NO;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sP + G::NE);
    float lap[G::KO][4 * BH];
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_barrier_init();
    }
    __syncthreads();
    int item = blockIdx.x;
    if (threadIdx.x == 0 && item < P.n_items) {
        issue_split<TX, TZ, BH, NTH>(P, P.s0, P.s0_p_in, P.s0_a_in, &P.qr, bufR, &bar[0], item, false,
                                     nullptr);
        issue_split<TX, TZ, BH, NTH>(P, P.s1, P.s1_in, P.s1_in, &P.qf, bufA, &bar[1], item,
                                     item_edge(P, item) != 0, gt);
    }
    for (int k = 0; item < P.n_items; k++, item += gridDim.x) {
        const uint32_t par = k & 1;
        const int next = item + gridDim.x;
        int shot, tile, x0, z0;
        item_origin(P, item, TX, TZ, shot, tile, x0, z0);
        const int64_t so = p.shot_stride * shot;
        const bool edge = p.tile_edge[tile] != 0;

        // reconstruction half: undamped everywhere, no Q
        bool ok = mbar_wait(&bar[0], par, P.err);
        if (__syncthreads_or(!ok)) {
            drain(&bar[0], par, &bar[1], par);
            return;
        }
        {
            const float *sAx = bufR, *sAz = bufR + G::NAX, *sPo = bufR + G::NAX + G::NAZ;
            const float *sq = sPo + 2 * G::NE;
            if (edge)
                p_split<TX, TZ, BH, NTH, true, true, kInjNone>(p, sAx, sAz, sPo, nullptr, sq, sP, nullptr,
                                                               x0, z0, shot, tile);
            else
                p_split<TX, TZ, BH, NTH, false, true, kInjNone>(p, sAx, sAz, sPo, nullptr, sq, sP,
                                                                nullptr, x0, z0, shot, tile);
            __syncthreads();
            if (p.ringe_ptr[tile + 1] > p.ringe_ptr[tile]) {  // uniform per item
                ring_overwrite1(p, sP, shot, tile, NTH);
                __syncthreads();
            }
            store_p1<TX, TZ>(p, sP, p.f0.px_out + so, x0, z0, NTH);
            if (edge)
                a_split<TX, TZ, BH, NTH, true, true, true>(p, sAx, sAz, sP, p.f0.ax_out + so,
                                                           p.f0.az_out + so, x0, z0, lap);
            else
                a_split<TX, TZ, BH, NTH, false, true, true>(p, sAx, sAz, sP, p.f0.ax_out + so,
                                                            p.f0.az_out + so, x0, z0, lap);
        }
        __syncthreads();
        if (threadIdx.x == 0 && next < P.n_items)
            issue_split<TX, TZ, BH, NTH>(P, P.s0, P.s0_p_in, P.s0_a_in, &P.qr, bufR, &bar[0], next, false,
                                         nullptr);

        // adjoint half and imaging condition
        ok = mbar_wait(&bar[1], par, P.err);
        if (__syncthreads_or(!ok)) {
            drain(&bar[1], par, next < P.n_items ? &bar[0] : nullptr, par ^ 1u);
            return;
        }
        {
            const float *sAx = bufA, *sAz = bufA + G::NAX, *sPo = bufA + G::NAX + G::NAZ;
            const float *sQo = sPo + G::NE, *sq = sPo + 2 * G::NE;
            if (edge)
                p_split<TX, TZ, BH, NTH, true, false, kInjReceivers>(p, sAx, sAz, sPo, sQo, sq, sP,
                                                                     p.f1.pz_out + so, x0, z0, shot, tile);
            else
                p_split<TX, TZ, BH, NTH, false, false, kInjReceivers>(p, sAx, sAz, sPo, sQo, sq, sP,
                                                                      nullptr, x0, z0, shot, tile);
            __syncthreads();
            store_p1<TX, TZ>(p, sP, p.f1.px_out + so, x0, z0, NTH);
            if (edge)
                a_split<TX, TZ, BH, NTH, true, false, false>(p, sAx, sAz, sP, p.f1.ax_out + so,
                                                             p.f1.az_out + so, x0, z0, nullptr);
            else
                a_split<TX, TZ, BH, NTH, false, false, false>(p, sAx, sAz, sP, p.f1.ax_out + so,
                                                              p.f1.az_out + so, x0, z0, nullptr);
            image1<TX, TZ, BH, NTH>(p, sP, gt, p.grad + so, x0, z0, lap);
        }
        __syncthreads();
        if (threadIdx.x == 0 && next < P.n_items)
            issue_split<TX, TZ, BH, NTH>(P, P.s1, P.s1_in, P.s1_in, &P.qf, bufA, &bar[1], next,
                                         item_edge(P, next) != 0, gt);
    }
}

}  // namespace otf
