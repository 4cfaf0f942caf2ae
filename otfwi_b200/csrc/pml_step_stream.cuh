// Streaming step kernels (fast numerics, separable damping): a CTA owns a
// strip of SO = 120 columns and a segment of rows of one shot and marches
// down z one row per step, instead of staging 2D halo tiles.
//
// Thread i holds column xc = x0 - 4 + i (i < 128): the strip plus a 4-column
// halo on each side, whose P(t) is recomputed because A(t) and the Laplacian
// need P(t) at x-3 .. x+4. Rows of the inputs of row r -- Ax(t-1) with an
// 8-column halo, Az(t-1) of row r+3, P(t-1), q and (edge rows / strips) Q --
// arrive in shared memory by 1D bulk copies (cp.async.bulk, mbarrier
// completion, no multicast) NSTG rows ahead. z-derivatives come from
// register windows: Az(t-1) rows r-4..r+3 for P(t) at row r, P(t) rows
// r-7..r for A(t) at row r-4 (r-8..r for the Laplacian); x-derivatives from
// the shared row buffers. One block barrier per row. A segment recomputes
// P(t) on 4 rows above and below it (the neighbour segments' rows), so no
// data is exchanged between CTAs within a step.
//
// The arithmetic is the strip-split form of pml_step_split.cuh (P total on
// every cell, Q = Px on damped cells) with the same operations per cell,
// except that every undamped cell takes the undamped A update form (the
// strip-split kernels use the damped form on all cells of an edge tile), so
// the two agree to FP32 rounding, not bit for bit.
#pragma once
#include "pml_step_split.cuh"

namespace otf {

constexpr int SO = 120;             // owned columns per strip
constexpr int SC = SO + 8;          // computed columns = threads per CTA
constexpr int SAXW = SC + 8;        // Ax row: computed columns + 4-column halo each side
constexpr int NSTG = 4;             // row stages in flight
constexpr int PRING = 6;            // P(t) rows kept for x-taps (A at r-4, written at r)
// stage layout (floats): Ax | Az(r+3) | P(t-1) | q | Q(t-1)
constexpr int SG_AX = 0, SG_AZ = SAXW, SG_P = SG_AZ + SC, SG_Q = SG_P + SC, SG_QQ = SG_Q + SC;
constexpr int SG_FLOATS = SG_QQ + SC;

// per (padded row, strip) point lists, key = (z + PAD) * n_strips + strip
struct StreamTabs {
    const int *src_ptr, *src_col, *src_id;     // sources (all computed columns)
    const int *rcv_ptr, *rcv_col, *rcv_id;     // adjoint-injected receivers (all computed columns)
    const int *sen_ptr, *sen_col, *sen_id;     // recorded receivers (owned columns)
    const int *ring_ptr, *ring_col;            // ring cells, owned columns (ring id = position)
    const int *ringe_ptr, *ringe_col, *ringe_id;  // ring cells, all computed columns (overwrite)
    const int *row_edge;                       // [rows]: damped or never-updated row
    const int *strip_edge;                     // [n_strips]: strip columns hold damped / never-updated cells
};

struct StreamParams {
    StepParams p;
    StreamTabs tb;
    int n_strips, seg_h, n_segs, n_items;  // items = strips x segments x shots
    int *err;
};

__device__ __forceinline__ void bulk_load_1d(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// First copied column (padded index) and float count of a row for strip x0:
// Ax rows [x0-8, x0+128), other rows [x0-4, x0+124), clipped at X+8 (the
// padded row holds x < X+8). Columns beyond the clip are never read by a
// cell whose result is kept.
__device__ __forceinline__ void row_span(int X, int x0, bool ax, int &col0, int &n)
{
    const int lo = ax ? x0 - 8 : x0 - 4, hi = min(ax ? x0 + SC : x0 + SC - 4, X + 8);
    col0 = lo + PAD;
    n = hi - lo;
}

// Issue the copies of row r of one field set into stage S (thread 0): Ax(t-1)
// row r, Az(t-1) row r+3, P(t-1) row r, coefficient q row r, Q(t-1) row r.
__device__ __forceinline__ void issue_row(const StepParams &p, const Fields &f, const float *qc, int64_t so,
                                          int x0, int r, bool with_q, float *S, uint64_t *bar)
{
    int ca, na, cc, nc;
    row_span(p.X, x0, true, ca, na);
    row_span(p.X, x0, false, cc, nc);
    const uint32_t bytes = 4u * (uint32_t)(na + (with_q ? 4 : 3) * nc);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_arrive_expect_tx(bar, bytes);
    const int64_t ro = (int64_t)(r + PAD) * p.pitch, ro3 = (int64_t)(r + 3 + PAD) * p.pitch;
    bulk_load_1d(S + SG_AX, f.ax_in + so + ro + ca, 4u * na, bar);
    bulk_load_1d(S + SG_AZ, f.az_in + so + ro3 + cc, 4u * nc, bar);
    bulk_load_1d(S + SG_P, f.px_in + so + ro + cc, 4u * nc, bar);
    bulk_load_1d(S + SG_Q, qc + ro + cc, 4u * nc, bar);
    if (with_q)
        bulk_load_1d(S + SG_QQ, f.pz_in + so + ro + cc, 4u * nc, bar);
}

__device__ __forceinline__ void stream_item(const StreamParams &P, int item, int &shot, int &strip, int &z0,
                                            int &z1)
{
    const int per_shot = P.n_strips * P.n_segs;
    shot = item / per_shot;
    const int k = item - shot * per_shot;
    const int seg = k / P.n_strips;
    strip = k - seg * P.n_strips;
    z0 = seg * P.seg_h;
    z1 = min(z0 + P.seg_h, P.p.Z);
}

// staggered derivative from 8 consecutive values w[0..7] (the pair form)
__device__ __forceinline__ float dstag8(const float *w)
{
    float o;
    dstag_n<1>(w, &o);
    return o;
}

// P(t) at one cell of the strip-split scheme. edge: this row or strip holds
// damped / never-updated cells; strip: the cell is damped.
__device__ __forceinline__ void p_cell(float dAx, float dAz, float po, float qv, float qo, float dmx, float dmz,
                                       bool edge, bool revert, float &pn, float &qn, bool &strip)
{
    strip = false;
    qn = 0.f;
    const float s = __fadd_rn(dAx, dAz);
    if (revert) {
        pn = __fmaf_rn(-qv, s, po);
    } else if (!edge) {
        pn = __fmaf_rn(qv, s, po);
    } else if (dmx != 1.f || dmz != 1.f) {
        strip = true;
        const float q1 = __fmaf_rn(qo, dmx, __fmul_rn(qv, dAx));
        const float z1 = __fmaf_rn(__fsub_rn(po, qo), dmz, __fmul_rn(qv, dAz));
        qn = q1;
        pn = __fadd_rn(q1, z1);
    } else {
        pn = __fmaf_rn(qv, s, po);
    }
}

// A(t) at one owned cell from its staggered P(t) derivatives: the damped
// form where the cell is damped, the undamped form elsewhere.
__device__ __forceinline__ void a_cell(float ax, float az, float dPx, float dPz, float r, float dmx, float dmz,
                                       bool revert, bool in_cell, float &nx, float &nz)
{
    if (revert) {
        nx = __fmaf_rn(-r, dPx, ax);
        nz = __fmaf_rn(-r, dPz, az);
    } else if (dmx != 1.f || dmz != 1.f) {
        nx = __fmaf_rn(ax, dmx, __fmul_rn(r, dPx));
        nz = __fmaf_rn(az, dmz, __fmul_rn(r, dPz));
    } else {
        nx = __fmaf_rn(r, dPx, ax);
        nz = __fmaf_rn(r, dPz, az);
    }
    if (!in_cell) {
        nx = 0.f;
        nz = 0.f;
    }
}

// Bounded drain of the copies still in flight after a failed wait (thread 0).
__device__ __forceinline__ void stream_drain(uint64_t *bar, int g_from, int g_to)
{
    for (int g = g_from; g < g_to; g++)
        mbar_wait(&bar[g % NSTG], (uint32_t)(g / NSTG) & 1u, nullptr);
}

// Forward step of every (strip, segment, shot) item, persistent CTAs. Stage
// use is round-robin over the CTA's whole run: global row step g uses stage
// g % NSTG at phase parity (g / NSTG) & 1.
template <bool RING>
__global__ void __launch_bounds__(SC, 4) k_forward_stream(const __grid_constant__ StreamParams P)
{
    __shared__ __align__(128) float stg[NSTG][SG_FLOATS];
    __shared__ __align__(16) float pring[PRING][SC];
    __shared__ uint64_t bar[NSTG];
    const StepParams &p = P.p;
    const int i = threadIdx.x;
    if (i == 0) {
        for (int s = 0; s < NSTG; s++)
            mbar_init(&bar[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    int g0 = 0;  // row steps done by this CTA before the current item
    for (int item = blockIdx.x; item < P.n_items; item += gridDim.x) {
        int shot, strip, z0, z1;
        stream_item(P, item, shot, strip, z0, z1);
        const int x0 = strip * SO, xc = x0 - 4 + i;
        const int64_t so = p.shot_stride * shot;
        const bool sedge = P.tb.strip_edge[strip] != 0;
        const bool col_ok = xc + PAD >= 0 && xc + PAD < p.pitch;
        const float dmx = (sedge && col_ok) ? __ldg(p.dampx + xc + PAD) : 1.f;
        const bool owned_col = i >= 4 && i < 4 + SO && xc < p.X;
        const bool in_x = xc >= 4 && xc < p.X - 4;
        const int r0 = z0 - 4, nsteps = (z1 - z0) + 8;
        if (i == 0)
            for (int k = 0; k < NSTG && k < nsteps; k++) {
                const int r = r0 + k, g = g0 + k;
                issue_row(p, p.f0, p.q0, so, x0, r, sedge || P.tb.row_edge[r + PAD], stg[g % NSTG],
                          &bar[g % NSTG]);
            }
        // Az(t-1) rows r-4..r+3 (prefilled with rows r0-4..r0+2), P(t) rows
        // r-7..r, Ax(t-1) rows r-4..r at this thread's column
        float azw[8], pw[8], axq[5];
        azw[0] = 0.f;
#pragma unroll
        for (int k = 1; k < 8; k++)
            azw[k] = col_ok ? __ldg(p.f0.az_in + so + (int64_t)(r0 - 5 + k + PAD) * p.pitch + xc + PAD) : 0.f;
#pragma unroll
        for (int k = 0; k < 8; k++)
            pw[k] = 0.f;
#pragma unroll
        for (int k = 0; k < 5; k++)
            axq[k] = 0.f;
        for (int k = 0; k < nsteps; k++) {
            const int r = r0 + k, g = g0 + k, st = g % NSTG;
            const bool ok = mbar_wait(&bar[st], (uint32_t)(g / NSTG) & 1u, P.err);
            if (__syncthreads_or(!ok)) {
                if (i == 0)
                    stream_drain(bar, g + 1, g0 + min(k + NSTG, nsteps));
                return;
            }
            const float *S = stg[st];
            const bool edge = sedge || P.tb.row_edge[r + PAD] != 0;
#pragma unroll
            for (int k2 = 0; k2 < 7; k2++)
                azw[k2] = azw[k2 + 1];
            azw[7] = S[SG_AZ + i];
            float w[8];
#pragma unroll
            for (int j = 0; j < 8; j++)
                w[j] = S[SG_AX + i + j];
            const float dAx = dstag8(w);
            const float dAz = dstag8(azw);
            const float dmz = edge ? __ldg(p.dampz + r + PAD) : 1.f;
            float pn, qn;
            bool strip_cell;
            p_cell(dAx, dAz, S[SG_P + i], S[SG_Q + i], edge ? S[SG_QQ + i] : 0.f, dmx, dmz, edge, false, pn, qn,
                   strip_cell);
            if (edge && !(in_x && r >= 4 && r < p.Z - 4)) {
                pn = 0.f;
                qn = 0.f;
            }
            const int key = (r + PAD) * P.n_strips + strip;
            for (int e = P.tb.src_ptr[key]; e < P.tb.src_ptr[key + 1]; e++) {
                if (P.tb.src_col[e] != i)
                    continue;
                const int row = p.fire_row[shot * p.n_src + P.tb.src_id[e]];
                if (row < 0)
                    continue;
                const float I = p.inj_tab[(int64_t)row * p.T + p.t];
                pn = __fadd_rn(pn, I);
                if (strip_cell)
                    qn = __fadd_rn(qn, __fmul_rn(I, 0.5f));
            }
            pring[k % PRING][i] = pn;
#pragma unroll
            for (int k2 = 0; k2 < 7; k2++)
                pw[k2] = pw[k2 + 1];
            pw[7] = pn;
#pragma unroll
            for (int k2 = 0; k2 < 4; k2++)
                axq[k2] = axq[k2 + 1];
            axq[4] = S[SG_AX + i + 4];
            __syncthreads();
            // the stage is consumed: refill it with row r + NSTG
            if (i == 0 && k + NSTG < nsteps) {
                const int rn = r + NSTG;
                issue_row(p, p.f0, p.q0, so, x0, rn, sedge || P.tb.row_edge[rn + PAD], stg[st], &bar[st]);
            }
            if (r >= z0 && r < z1) {
                if (owned_col) {
                    const int64_t o = so + (int64_t)(r + PAD) * p.pitch + xc + PAD;
                    p.f0.px_out[o] = pn;
                    if (edge)
                        p.f0.pz_out[o] = qn;
                }
                for (int e = P.tb.sen_ptr[key] + i; e < P.tb.sen_ptr[key + 1]; e += SC)
                    p.rec[((int64_t)shot * p.n_sen + P.tb.sen_id[e]) * p.T + p.t] =
                        pring[k % PRING][P.tb.sen_col[e]];
                if (RING) {
                    float *ring = p.ring + ((int64_t)shot * p.T + p.t) * p.n_ring;
                    for (int e = P.tb.ring_ptr[key] + i; e < P.tb.ring_ptr[key + 1]; e += SC)
                        ring[e] = pring[k % PRING][P.tb.ring_col[e]];
                }
            }
            // A(t) at row a = r - 4
            if (k >= 8 && owned_col) {
                const int a = r - 4;
                const float *pr = pring[(k - 4) % PRING];
                float wp[8];
#pragma unroll
                for (int j = 0; j < 8; j++)
                    wp[j] = pr[i - 3 + j];
                const bool aedge = sedge || P.tb.row_edge[a + PAD] != 0;
                const float dmza = aedge ? __ldg(p.dampz + a + PAD) : 1.f;
                float nx, nz;
                a_cell(axq[0], azw[0], dstag8(wp), dstag8(pw), p.r, dmx, dmza, false,
                       !aedge || (in_x && a >= 4 && a < p.Z - 4), nx, nz);
                const int64_t o = so + (int64_t)(a + PAD) * p.pitch + xc + PAD;
                p.f0.ax_out[o] = nx;
                p.f0.az_out[o] = nz;
            }
        }
        g0 += nsteps;
        __syncthreads();  // every thread is done with the shared rows of this item
    }
}

// Reverse-step stage: reconstruction set (Ax | Az | P | q) then adjoint set
// (Ax | Az | P | q | Q) then the gradient row r-4.
constexpr int RS_A = SG_QQ;                       // adjoint set offset (reconstruction has no Q)
constexpr int RS_G = RS_A + SG_FLOATS;            // gradient row
constexpr int RS_FLOATS = RS_G + SC;

__device__ __forceinline__ void issue_rev_row(const StepParams &p, int64_t so, int x0, int r, bool with_q,
                                              float *S, uint64_t *bar)
{
    int ca, na, cc, nc;
    row_span(p.X, x0, true, ca, na);
    row_span(p.X, x0, false, cc, nc);
    // reconstruction: Ax, Az, P, q; adjoint: Ax, Az, P, q (+ Q); gradient row
    const uint32_t bytes = 4u * (uint32_t)(2 * na + (with_q ? 8 : 7) * nc);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_arrive_expect_tx(bar, bytes);
    const int64_t ro = (int64_t)(r + PAD) * p.pitch, ro3 = (int64_t)(r + 3 + PAD) * p.pitch;
    const int64_t rg = (int64_t)(r - 4 + PAD) * p.pitch;
    bulk_load_1d(S + SG_AX, p.f0.ax_in + so + ro + ca, 4u * na, bar);
    bulk_load_1d(S + SG_AZ, p.f0.az_in + so + ro3 + cc, 4u * nc, bar);
    bulk_load_1d(S + SG_P, p.f0.px_in + so + ro + cc, 4u * nc, bar);
    bulk_load_1d(S + SG_Q, p.q0 + ro + cc, 4u * nc, bar);
    float *A = S + RS_A;
    bulk_load_1d(A + SG_AX, p.f1.ax_in + so + ro + ca, 4u * na, bar);
    bulk_load_1d(A + SG_AZ, p.f1.az_in + so + ro3 + cc, 4u * nc, bar);
    bulk_load_1d(A + SG_P, p.f1.px_in + so + ro + cc, 4u * nc, bar);
    bulk_load_1d(A + SG_Q, p.q1 + ro + cc, 4u * nc, bar);
    if (with_q)
        bulk_load_1d(A + SG_QQ, p.f1.pz_in + so + ro + cc, 4u * nc, bar);
    bulk_load_1d(S + RS_G, p.grad + so + rg + cc, 4u * nc, bar);
}

// Reverse step: time-reversed reconstruction (undamped, ring overwrite),
// damped adjoint with adjoint-source injection, and the imaging condition
// grad += P_adj * lap9(P_rec), per (strip, segment, shot) item.
template <int MINB>
__global__ void __launch_bounds__(SC, MINB) k_reverse_stream(const __grid_constant__ StreamParams P)
{
    __shared__ __align__(128) float stg[NSTG][RS_FLOATS];
    __shared__ __align__(16) float pr_r[PRING][SC];
    __shared__ __align__(16) float pr_a[PRING][SC];
    __shared__ uint64_t bar[NSTG];
    const StepParams &p = P.p;
    const int i = threadIdx.x;
    if (i == 0) {
        for (int s = 0; s < NSTG; s++)
            mbar_init(&bar[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    int g0 = 0;
    for (int item = blockIdx.x; item < P.n_items; item += gridDim.x) {
        int shot, strip, z0, z1;
        stream_item(P, item, shot, strip, z0, z1);
        const int x0 = strip * SO, xc = x0 - 4 + i;
        const int64_t so = p.shot_stride * shot;
        const bool sedge = P.tb.strip_edge[strip] != 0;
        const bool col_ok = xc + PAD >= 0 && xc + PAD < p.pitch;
        const float dmx = (sedge && col_ok) ? __ldg(p.dampx + xc + PAD) : 1.f;
        const bool owned_col = i >= 4 && i < 4 + SO && xc < p.X;
        const bool in_x = xc >= 4 && xc < p.X - 4;
        const int r0 = z0 - 4, nsteps = (z1 - z0) + 8;
        const float *ring_t = p.ring + ((int64_t)shot * p.T + (p.T - 1 - p.t)) * p.n_ring;
        if (i == 0)
            for (int k = 0; k < NSTG && k < nsteps; k++) {
                const int r = r0 + k, g = g0 + k;
                issue_rev_row(p, so, x0, r, sedge || P.tb.row_edge[r + PAD], stg[g % NSTG], &bar[g % NSTG]);
            }
        // windows: reconstruction Az rows r-4..r+3, P rows r-8..r, Ax rows r-4..r;
        // adjoint Az rows r-4..r+3, P rows r-7..r, Ax rows r-4..r
        float azr[8], pwr[9], axr[5], aza[8], pwa[8], axa[5];
        azr[0] = aza[0] = 0.f;
#pragma unroll
        for (int k = 1; k < 8; k++) {
            const int64_t o = so + (int64_t)(r0 - 5 + k + PAD) * p.pitch + xc + PAD;
            azr[k] = col_ok ? __ldg(p.f0.az_in + o) : 0.f;
            aza[k] = col_ok ? __ldg(p.f1.az_in + o) : 0.f;
        }
#pragma unroll
        for (int k = 0; k < 9; k++)
            pwr[k] = 0.f;
#pragma unroll
        for (int k = 0; k < 8; k++)
            pwa[k] = 0.f;
#pragma unroll
        for (int k = 0; k < 5; k++)
            axr[k] = axa[k] = 0.f;
        for (int k = 0; k < nsteps; k++) {
            const int r = r0 + k, g = g0 + k, st = g % NSTG;
            const bool ok = mbar_wait(&bar[st], (uint32_t)(g / NSTG) & 1u, P.err);
            if (__syncthreads_or(!ok)) {
                if (i == 0)
                    stream_drain(bar, g + 1, g0 + min(k + NSTG, nsteps));
                return;
            }
            const float *S = stg[st], *SA = S + RS_A;
            const bool edge = sedge || P.tb.row_edge[r + PAD] != 0;
            const bool in_cell = !edge || (in_x && r >= 4 && r < p.Z - 4);
            const int key = (r + PAD) * P.n_strips + strip;
            // reconstruction P(t) at row r (undamped, reversed)
#pragma unroll
            for (int k2 = 0; k2 < 7; k2++) {
                azr[k2] = azr[k2 + 1];
                aza[k2] = aza[k2 + 1];
            }
            azr[7] = S[SG_AZ + i];
            aza[7] = SA[SG_AZ + i];
            float w[8];
#pragma unroll
            for (int j = 0; j < 8; j++)
                w[j] = S[SG_AX + i + j];
            float prn, qdum;
            bool sdum;
            p_cell(dstag8(w), dstag8(azr), S[SG_P + i], S[SG_Q + i], 0.f, 1.f, 1.f, edge, true, prn, qdum, sdum);
            if (!in_cell)
                prn = 0.f;
            pr_r[k % PRING][i] = prn;
            // adjoint P(t) at row r (damped) with adjoint-source injection
#pragma unroll
            for (int j = 0; j < 8; j++)
                w[j] = SA[SG_AX + i + j];
            const float dmz = edge ? __ldg(p.dampz + r + PAD) : 1.f;
            float pan, qan;
            bool strip_cell;
            p_cell(dstag8(w), dstag8(aza), SA[SG_P + i], SA[SG_Q + i], edge ? SA[SG_QQ + i] : 0.f, dmx, dmz, edge,
                   false, pan, qan, strip_cell);
            if (!in_cell) {
                pan = 0.f;
                qan = 0.f;
            }
            for (int e = P.tb.rcv_ptr[key]; e < P.tb.rcv_ptr[key + 1]; e++) {
                if (P.tb.rcv_col[e] != i)
                    continue;
                const float I = p.inj_tab[((int64_t)shot * p.n_sen + P.tb.rcv_id[e]) * p.T + p.t];
                pan = __fadd_rn(pan, I);
                if (strip_cell)
                    qan = __fadd_rn(qan, __fmul_rn(I, 0.5f));
            }
            pr_a[k % PRING][i] = pan;
#pragma unroll
            for (int k2 = 0; k2 < 7; k2++)
                pwa[k2] = pwa[k2 + 1];
            pwa[7] = pan;
#pragma unroll
            for (int k2 = 0; k2 < 4; k2++) {
                axr[k2] = axr[k2 + 1];
                axa[k2] = axa[k2 + 1];
            }
            axr[4] = S[SG_AX + i + 4];
            axa[4] = SA[SG_AX + i + 4];
            const float gold = S[RS_G + i];
            // ring overwrite of the reconstruction (setRec): P = ring(T-1-t)
            const int rb = P.tb.ringe_ptr[key], re = P.tb.ringe_ptr[key + 1];
            if (rb < re) {
                __syncthreads();
                for (int e = rb + i; e < re; e += SC)
                    pr_r[k % PRING][P.tb.ringe_col[e]] = ring_t[P.tb.ringe_id[e]];
                __syncthreads();
                prn = pr_r[k % PRING][i];
            } else {
                __syncthreads();
            }
#pragma unroll
            for (int k2 = 0; k2 < 8; k2++)
                pwr[k2] = pwr[k2 + 1];
            pwr[8] = prn;
            if (i == 0 && k + NSTG < nsteps) {
                const int rn = r + NSTG;
                issue_rev_row(p, so, x0, rn, sedge || P.tb.row_edge[rn + PAD], stg[st], &bar[st]);
            }
            if (r >= z0 && r < z1 && owned_col) {
                const int64_t o = so + (int64_t)(r + PAD) * p.pitch + xc + PAD;
                p.f0.px_out[o] = prn;
                p.f1.px_out[o] = pan;
                if (edge)
                    p.f1.pz_out[o] = qan;
            }
            if (k >= 8 && owned_col) {
                const int a = r - 4;
                const bool aedge = sedge || P.tb.row_edge[a + PAD] != 0;
                const bool a_in = !aedge || (in_x && a >= 4 && a < p.Z - 4);
                const float dmza = aedge ? __ldg(p.dampz + a + PAD) : 1.f;
                const float *rr = pr_r[(k - 4) % PRING], *ra = pr_a[(k - 4) % PRING];
                float wp[8];
#pragma unroll
                for (int j = 0; j < 8; j++)
                    wp[j] = rr[i - 3 + j];
                float nx, nz;
                a_cell(axr[0], azr[0], dstag8(wp), dstag8(pwr + 1), p.r, 1.f, 1.f, true, a_in, nx, nz);
                const int64_t o = so + (int64_t)(a + PAD) * p.pitch + xc + PAD;
                p.f0.ax_out[o] = nx;
                p.f0.az_out[o] = nz;
                // imaging condition with the 9-point Laplacian of the reconstruction
                float lx, lz;
                lap_n<1>(rr + i - 4, &lx);
                lap_n<1>(pwr, &lz);
                p.grad[o] = __fmaf_rn(pwa[3], lap_combine(lx, lz), gold);
#pragma unroll
                for (int j = 0; j < 8; j++)
                    wp[j] = ra[i - 3 + j];
                a_cell(axa[0], aza[0], dstag8(wp), dstag8(pwa), p.r, dmx, dmza, false, a_in, nx, nz);
                p.f1.ax_out[o] = nx;
                p.f1.az_out[o] = nz;
            }
        }
        g0 += nsteps;
        __syncthreads();
    }
}

}  // namespace otf
