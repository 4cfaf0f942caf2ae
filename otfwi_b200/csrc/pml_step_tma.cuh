// Persistent, TMA-pipelined versions of the fused step kernels.
//
// A time step is one launch of a grid sized to the GPU (one or two CTAs per
// SM). Each CTA walks the (shot, tile) work items of the step round-robin and
// keeps the Tensor Memory Accelerator one item ahead: while it computes item
// i from shared memory, cp.async.bulk.tensor copies the halo tiles of item
// i+1 (A(t-1) with an 8-cell halo, P(t-1) and the P coefficient with a
// 4-cell halo, and for the reverse step the gradient tile) into the other
// half of a double buffer, completion signalled on an mbarrier. Global loads
// therefore never sit on the compute path; the arithmetic is the same device
// code as the per-tile kernels, so results are bit-identical to them.
//
// The reverse step pipelines at half-item granularity: the reconstruction
// half of item i overlaps the copies for the adjoint half of item i, and the
// adjoint half overlaps the copies for the reconstruction half of item i+1.
#pragma once
#include "pml_step.cuh"
#include "tma.cuh"

namespace otf {

struct SetMaps {  // one wavefield set, one map per slot
    CUtensorMap ax[2];  // box (TX+16) x (TZ+8)
    CUtensorMap az[2];  // box (TX+8) x (TZ+16)
    CUtensorMap px[2];  // box (TX+8) x (TZ+8)
    CUtensorMap pz[2];
};

struct TmaParams {
    SetMaps s0, s1;
    CUtensorMap qf, qr;  // P coefficient boxes (TX+8) x (TZ+8)
    CUtensorMap grad;    // owned box TX x TZ of the per-shot gradients
    StepParams p;
    int s0_p_in, s0_a_in;  // slots read by set 0 (P and A may differ: reconstruction)
    int s1_in;             // slot read by set 1
    int n_tiles, n_items;
    int *err;              // device error flag (set on a wait that timed out)
};

template <int TX, int TZ>
struct TmaGeom {
    using G = TileGeom<TX, TZ>;
    static constexpr int FWD_FLOATS = 2 * G::STAGE_FLOATS + 2 * G::NE;
    static constexpr int REV_FLOATS = 2 * G::STAGE_FLOATS + G::NO + 2 * G::NE;
    static constexpr size_t FWD_BYTES = sizeof(float) * FWD_FLOATS + 2 * sizeof(uint64_t);
    static constexpr size_t REV_BYTES = sizeof(float) * REV_FLOATS + 2 * sizeof(uint64_t);
    static constexpr uint32_t STAGE_BYTES = sizeof(float) * G::STAGE_FLOATS;
    static constexpr uint32_t GRAD_BYTES = sizeof(float) * G::NO;
};

__device__ __forceinline__ void item_origin(const TmaParams &P, int item, int tx_, int tz_, int &shot,
                                            int &tile, int &x0, int &z0)
{
    shot = item / P.n_tiles;
    tile = item - shot * P.n_tiles;
    x0 = (tile % P.p.ntx) * tx_;
    z0 = (tile / P.p.ntx) * tz_;
}

// Issue the copies of one field set's inputs for one item into a stage.
// Padded coordinates: Ax box starts at (x0-8, z0-4), Az at (x0-4, z0-8),
// P(t-1) / q at (x0-4, z0-4), the gradient tile at (x0, z0); +PAD each.
// Every x start is a multiple of 4 floats (16 bytes).
template <int TX, int TZ>
__device__ __forceinline__ void issue_set(const TmaParams &P, const SetMaps &m, int pin, int ain,
                                          const CUtensorMap *q, float *stage, uint64_t *bar, int item,
                                          float *gtile)
{
    using G = TileGeom<TX, TZ>;
    using M = TmaGeom<TX, TZ>;
    int shot, tile, x0, z0;
    item_origin(P, item, TX, TZ, shot, tile, x0, z0);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_arrive_expect_tx(bar, M::STAGE_BYTES + (gtile ? M::GRAD_BYTES : 0u));
    tma_load_3d(stage, &m.ax[ain], x0 - 8 + PAD, z0 - 4 + PAD, shot, bar);
    tma_load_3d(stage + G::NAX, &m.az[ain], x0 - 4 + PAD, z0 - 8 + PAD, shot, bar);
    tma_load_3d(stage + G::NAX + G::NAZ, &m.px[pin], x0 - 4 + PAD, z0 - 4 + PAD, shot, bar);
    tma_load_3d(stage + G::NAX + G::NAZ + G::NE, &m.pz[pin], x0 - 4 + PAD, z0 - 4 + PAD, shot, bar);
    tma_load_3d(stage + G::NAX + G::NAZ + 2 * G::NE, q, x0 - 4 + PAD, z0 - 4 + PAD, 0, bar);
    if (gtile)
        tma_load_3d(gtile, &P.grad, x0 + PAD, z0 + PAD, shot, bar);
}

// After a wait timed out: give the copies still in flight into this CTA's
// shared memory (up to two barriers, b1 optional) a bounded chance to land
// before the CTA exits.
__device__ __forceinline__ void drain(uint64_t *b0, uint32_t p0, uint64_t *b1, uint32_t p1)
{
    if (threadIdx.x == 0) {
        mbar_wait(b0, p0, nullptr);
        if (b1)
            mbar_wait(b1, p1, nullptr);
    }
    __syncthreads();
}

template <int TX, int TZ, class Prec, bool SEP, bool RING, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_forward_tma(const __grid_constant__ TmaParams P)
{
    using G = TileGeom<TX, TZ>;
    extern __shared__ __align__(128) float smf[];
    const StepParams &p = P.p;
    float *stage0 = smf, *stage1 = smf + G::STAGE_FLOATS;
    float *sPx = smf + 2 * G::STAGE_FLOATS, *sPz = sPx + G::NE;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sPz + G::NE);
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_barrier_init();
    }
    __syncthreads();
    int item = blockIdx.x;
    if (threadIdx.x == 0 && item < P.n_items)
        issue_set<TX, TZ>(P, P.s0, P.s0_p_in, P.s0_a_in, &P.qf, stage0, &bar[0], item, nullptr);
    for (int k = 0; item < P.n_items; k++, item += gridDim.x) {
        const int st = k & 1;
        float *S = st ? stage1 : stage0;
        const int next = item + gridDim.x;
        if (threadIdx.x == 0 && next < P.n_items)
            issue_set<TX, TZ>(P, P.s0, P.s0_p_in, P.s0_a_in, &P.qf, st ? stage0 : stage1, &bar[st ^ 1],
                              next, nullptr);
        const bool ok = mbar_wait(&bar[st], (k >> 1) & 1, P.err);
        if (__syncthreads_or(!ok)) {
            drain(&bar[st], (k >> 1) & 1, next < P.n_items ? &bar[st ^ 1] : nullptr, ((k + 1) >> 1) & 1);
            return;
        }
        int shot, tile, x0, z0;
        item_origin(P, item, TX, TZ, shot, tile, x0, z0);
        const int64_t so = p.shot_stride * shot;
        const float *sAx = S, *sAz = S + G::NAX;
        p_phase<TX, TZ, Prec, SEP, false, true>(p, sAx, sAz, sPx, sPz, S + G::NAX + G::NAZ,
                                                S + G::NAX + G::NAZ + G::NE,
                                                S + G::NAX + G::NAZ + 2 * G::NE, x0, z0);
        __syncthreads();
        inject<TX, TZ>(p, sPx, sPz, shot, x0, z0);
        __syncthreads();
        store_p<TX, TZ>(p, sPx, sPz, p.f0.px_out + so, p.f0.pz_out + so, x0, z0);
        record<TX, TZ, RING>(p, sPx, sPz, shot, tile);
        a_phase<TX, TZ, Prec, SEP, false, false, true>(p, sAx, sAz, sPx, sPz, nullptr, nullptr,
                                                       p.f0.ax_out + so, p.f0.az_out + so, x0, z0,
                                                       nullptr);
        __syncthreads();
    }
}

template <int TX, int TZ, class Prec, bool SEP, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_reverse_tma(const __grid_constant__ TmaParams P)
{
    using G = TileGeom<TX, TZ>;
    extern __shared__ __align__(128) float smf[];
    const StepParams &p = P.p;
    float *bufR = smf, *bufA = smf + G::STAGE_FLOATS;
    float *gt = bufA + G::STAGE_FLOATS;
    float *sPx = gt + G::NO, *sPz = sPx + G::NE;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sPz + G::NE);
    float lap[G::KO][16];
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_barrier_init();
    }
    __syncthreads();
    int item = blockIdx.x;
    if (threadIdx.x == 0 && item < P.n_items) {
        issue_set<TX, TZ>(P, P.s0, P.s0_p_in, P.s0_a_in, &P.qr, bufR, &bar[0], item, nullptr);
        issue_set<TX, TZ>(P, P.s1, P.s1_in, P.s1_in, &P.qf, bufA, &bar[1], item, gt);
    }
    for (int k = 0; item < P.n_items; k++, item += gridDim.x) {
        const uint32_t par = k & 1;
        const int next = item + gridDim.x;
        int shot, tile, x0, z0;
        item_origin(P, item, TX, TZ, shot, tile, x0, z0);
        const int64_t so = p.shot_stride * shot;

        // reconstruction half
        bool ok = mbar_wait(&bar[0], par, P.err);
        if (__syncthreads_or(!ok)) {
            drain(&bar[0], par, &bar[1], par);
            return;
        }
        p_phase<TX, TZ, Prec, SEP, true, true>(p, bufR, bufR + G::NAX, sPx, sPz,
                                               bufR + G::NAX + G::NAZ, bufR + G::NAX + G::NAZ + G::NE,
                                               bufR + G::NAX + G::NAZ + 2 * G::NE, x0, z0);
        __syncthreads();
        ring_overwrite<TX, TZ>(p, sPx, sPz, shot, tile);
        __syncthreads();
        store_p<TX, TZ>(p, sPx, sPz, p.f0.px_out + so, p.f0.pz_out + so, x0, z0);
        a_phase<TX, TZ, Prec, SEP, true, true, true>(p, bufR, bufR + G::NAX, sPx, sPz, nullptr, nullptr,
                                                     p.f0.ax_out + so, p.f0.az_out + so, x0, z0, lap);
        __syncthreads();
        if (threadIdx.x == 0 && next < P.n_items)
            issue_set<TX, TZ>(P, P.s0, P.s0_p_in, P.s0_a_in, &P.qr, bufR, &bar[0], next, nullptr);

        // adjoint half and imaging condition
        ok = mbar_wait(&bar[1], par, P.err);
        if (__syncthreads_or(!ok)) {
            drain(&bar[1], par, next < P.n_items ? &bar[0] : nullptr, par ^ 1u);
            return;
        }
        p_phase<TX, TZ, Prec, SEP, false, true>(p, bufA, bufA + G::NAX, sPx, sPz,
                                                bufA + G::NAX + G::NAZ, bufA + G::NAX + G::NAZ + G::NE,
                                                bufA + G::NAX + G::NAZ + 2 * G::NE, x0, z0);
        __syncthreads();
        inject<TX, TZ>(p, sPx, sPz, shot, x0, z0);
        __syncthreads();
        store_p<TX, TZ>(p, sPx, sPz, p.f1.px_out + so, p.f1.pz_out + so, x0, z0);
        a_phase<TX, TZ, Prec, SEP, false, false, true>(p, bufA, bufA + G::NAX, sPx, sPz, nullptr, nullptr,
                                                       p.f1.ax_out + so, p.f1.az_out + so, x0, z0,
                                                       nullptr);
        image<TX, TZ, true>(p, sPx, sPz, gt, p.grad + so, x0, z0, lap);
        __syncthreads();
        if (threadIdx.x == 0 && next < P.n_items)
            issue_set<TX, TZ>(P, P.s1, P.s1_in, P.s1_in, &P.qf, bufA, &bar[1], next, gt);
    }
}

}  // namespace otf
