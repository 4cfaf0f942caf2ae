// Unfused streaming step kernels for the fast numerics (variant 4).
//
// The fused kernels (pml_step_split.cuh, pml_step_stream.cuh) compute P(t)
// and A(t) of a tile in one pass, recomputing P on a 4-cell halo and
// synchronising the CTA between the two half-steps; measured, they run
// latency- and barrier-bound near half of the HBM bandwidth. Here each
// half-step is its own launch over the whole batch, every cell is computed
// once, and nothing waits on anything but its own loads:
//
//   forward step:  P kernel  P(t), Q(t) from P, Q, Ax, Az (t-1); then each
//                            CTA injects the shot's sources in its cells
//                  A kernel  Ax, Az (t) from P(t); extra CTAs record the
//                            receivers and the boundary ring
//   reverse step:  P kernel  both field sets: reconstruction (undamped,
//                            reverted; then P_rec(t) = ring(T-1-t) on the
//                            CTA's ring cells) and adjoint (damped; then the
//                            adjoint sources at the CTA's receivers)
//                  A kernel  one CTA per field set: the reconstruction's A
//                            update, the 9-point Laplacian of P_rec(t) and
//                            grad += P_adj(t) * lap; the adjoint's damped A
//                            update (k_unfused_a_rev_sets; both sets in one
//                            CTA: k_unfused_a_rev)
//
// Within a time loop the engine may split the shots into lanes, each its own
// chain of these launches (grid z = the lane's shots, UnfusedParams::shot0
// its first): the lanes run concurrently and fill each other's launch tails.
//
// A thread owns 4 adjacent columns (16-byte loads and stores) of a
// 128-column block and marches down kURows rows: z-derivatives come from a
// sliding register window per column, x-derivatives from three 16-byte row
// loads (columns x-4 .. x+7) that L1 shares between neighbouring threads.
// One warp per CTA, no shared memory, no barrier. Bytes per cell: 40 for a
// forward step (P kernel 20 + Q on damped cells, A kernel 20), 92 for a
// reverse step (P 40, A 52), against 28 and 64 for the fused kernels, at
// 70-80% of the bandwidth instead of under 50%.
//
// Shot order alternates between consecutive launches: CTAs are dispatched in
// grid order, the P kernels walk the shots upwards and the A kernels
// downwards, so each launch begins on the shots its predecessor finished
// with, whose fields may still be in the L2 (P(t) and Ax, Az (t-1) for the A
// kernel; P(t) and Ax, Az (t) for the next P kernel). The order of CTAs
// changes no result: every cell and every shot's gradient is written by one
// thread. Measured on one B200 (64 shots, 512^2): forward step 0.119 ms
// against 0.123 in launch order, reverse step unchanged (0.27 ms).
//
// The cell arithmetic is that of the strip-split kernels: the same pair-form
// staggered sums, P and Q updates, injection (after the cell's update, in
// source order) and Laplacian; the damped
// A update fma(A, dm, r*D) is used exactly on damped cells (the strip-split
// kernels use it on every cell of a tile that holds a damped cell, so the
// two agree bit for bit when dt/dx = 1 and within rounding otherwise).
#pragma once
#include "pml_step.cuh"
#include "pml_step_split.cuh"

namespace otf {

constexpr int kUThreads = 32;             // threads per CTA
constexpr int kUCols = 4 * kUThreads;     // columns per CTA
constexpr int kURows = 8;                 // rows marched by a thread (4 / 8 / 16 measured: 8 fastest)
constexpr int kUTailPer = 8;              // receiver / ring cells recorded per thread

struct UnfusedParams {
    StepParams p;
    int ncb, nseg;  // column blocks, row segments per shot
    // injection cells (CSR): padded offset of each distinct cell holding a
    // source / an injectable receiver, and its source / receiver indices in
    // increasing order; cells grouped by the P-kernel CTA that owns them
    // (src_cta / rcv_cta [ncb * nseg + 1] index the cell arrays)
    const int *src_ptr, *src_off, *src_id, *src_cta;
    int n_src_cells;
    const int *rcv_ptr, *rcv_off, *rcv_id, *rcv_cta;
    int n_rcv_cells;
    // ring cells grouped by owning CTA: ring_cta [ncb * nseg + 1] indexes
    // ring_cta_off (padded offset) and ring_cta_k (ring index)
    const int *ring_cta, *ring_cta_off, *ring_cta_k;
    // padded offsets (within a shot) of the receivers and of the ring cells
    // (ring id = the caller's ring index)
    const int *rec_off, *ring_off;
    int record_ring;  // forward: also record the boundary ring
    unsigned *ledger;  // launches of this time loop: the first CTA of each launch counts it
    int shot0;         // first shot of this launch (a lane of the batch: grid z covers its shots)
};

// Count this launch (thread 0 of the first CTA), after pdl_enter: a launch
// that never ran leaves the count short, which the loop's check turns into
// an error of the call.
__device__ __forceinline__ void count_launch(const UnfusedParams &U)
{
    if ((blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.x) == 0u)
        atomicAdd(U.ledger, 1u);
}

// Programmatic dependent launch: the engine launches these kernels with
// programmatic stream serialization, so a kernel's CTAs may be scheduled
// while its predecessor's last CTAs still run (hiding the launch gap and the
// predecessor's tail). Every kernel waits here, before touching memory,
// until the predecessor grid has completed and its writes are visible, then
// allows its own successor to start launching. Without the launch attribute
// both calls return at once.
__device__ __forceinline__ void pdl_enter()
{
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 900
    cudaGridDependencySynchronize();
    cudaTriggerProgrammaticLaunchCompletion();
#endif
}

__device__ __forceinline__ float4 uld4(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
// P(t) as the A half-step reads it: through the read-only path when another
// launch wrote it (unfused kernels), from L2 (ld.global.cg, coherent) when
// P items of the same launch wrote it (paired kernels, pml_step_paired.cuh)
template <bool COHERENT>
__device__ __forceinline__ float4 pld4(const float *p)
{
    if (COHERENT)
        return __ldcg(reinterpret_cast<const float4 *>(p));
    return __ldg(reinterpret_cast<const float4 *>(p));
}
__device__ __forceinline__ float4 uld4c(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void ust4(float *p, const float *v)
{
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}

// One 4-column segment of a P half-step. REVERT: time-reversed
// reconstruction (undamped, no Q); otherwise damped with the strip
// component Q. The CTA's point work follows in the calling kernel.
template <bool REVERT>
__device__ __forceinline__ void p_segment(const UnfusedParams &U, const Fields &f, const float *__restrict__ q,
                                          int shot, int x, int z0)
{
    const StepParams &p = U.p;
    const int64_t so = p.shot_stride * shot;
    const float *__restrict__ AX = f.ax_in + so;
    const float *__restrict__ AZ = f.az_in + so;
    const float *__restrict__ PI = f.px_in + so;
    const float *__restrict__ QI = f.pz_in + so;
    float *__restrict__ PO = f.px_out + so;
    float *__restrict__ QO = f.pz_out + so;
    const int64_t col = x + PAD, pitch = p.pitch;
    float w[4][8];
#pragma unroll
    for (int k = 0; k < 7; k++) {
        const float4 v = uld4(AZ + (int64_t)(z0 - 4 + k + PAD) * pitch + col);
        w[0][k] = v.x;
        w[1][k] = v.y;
        w[2][k] = v.z;
        w[3][k] = v.w;
    }
    const int nz = min(kURows, p.Z - z0);
#pragma unroll 1
    for (int r = 0; r < nz; r++) {
        const int z = z0 + r;
        const int64_t o = (int64_t)(z + PAD) * pitch + col;
        {
            const float4 v = uld4(AZ + o + 3 * pitch);
            w[0][7] = v.x;
            w[1][7] = v.y;
            w[2][7] = v.z;
            w[3][7] = v.w;
        }
        float u[12], po[4], qv[4];
        f4a(uld4(AX + o - 4), u);
        f4a(uld4(AX + o), u + 4);
        f4a(uld4(AX + o + 4), u + 8);
        f4a(uld4(PI + o), po);
        f4a(uld4(q + o), qv);
        float dmx[4] = {1.f, 1.f, 1.f, 1.f};
        if (!REVERT)
            f4a(uld4(p.dampx + col), dmx);  // L1-resident, reloaded per row
        const float dmz = REVERT ? 1.f : __ldg(p.dampz + z + PAD);
        const bool damp = !REVERT && (dmx[0] != 1.f || dmx[1] != 1.f || dmx[2] != 1.f || dmx[3] != 1.f ||
                                      dmz != 1.f);
        float qo[4] = {0.f, 0.f, 0.f, 0.f};
        if (damp)
            f4a(uld4(QI + o), qo);
        const bool zin = z >= 4 && z < p.Z - 4;
        float pn[4], qn[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            float dAx, dAz;
            dstag_n<1>(u + j, &dAx);
            dstag_n<1>(w[j], &dAz);
            const float s = __fadd_rn(dAx, dAz);
            qn[j] = 0.f;
            if (REVERT) {
                pn[j] = __fmaf_rn(-qv[j], s, po[j]);
            } else if (dmx[j] != 1.f || dmz != 1.f) {
                const float q1 = __fmaf_rn(qo[j], dmx[j], __fmul_rn(qv[j], dAx));
                const float z1 = __fmaf_rn(__fsub_rn(po[j], qo[j]), dmz, __fmul_rn(qv[j], dAz));
                qn[j] = q1;
                pn[j] = __fadd_rn(q1, z1);
            } else {
                pn[j] = __fmaf_rn(qv[j], s, po[j]);
            }
            if (x + j < 4 || x + j >= p.X - 4 || !zin) {
                pn[j] = 0.f;
                qn[j] = 0.f;
            }
        }
        ust4(PO + o, pn);
        if (damp)
            ust4(QO + o, qn);
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int k = 0; k < 7; k++)
                w[j][k] = w[j][k + 1];
    }
}

// Injection at one cell after its P update: the sources fired by the shot
// (or the adjoint sources at a receiver), P += I (both split components get
// I/2) and Q += I/2 on strip cells, in source order, exactly as the fused
// kernels inject.
__device__ __forceinline__ void inject_cell(const StepParams &p, const Fields &f, int shot, int off, const int *ids,
                                            int e0, int e1, bool sources)
{
    const int64_t o = p.shot_stride * shot + off;
    const int z = off / p.pitch - PAD, x = off - (z + PAD) * p.pitch - PAD;
    const bool strip = __ldg(p.dampx + x + PAD) != 1.f || __ldg(p.dampz + z + PAD) != 1.f;
    float pn = f.px_out[o], qn = strip ? f.pz_out[o] : 0.f;
    for (int e = e0; e < e1; e++) {
        const int row = sources ? p.fire_row[shot * p.n_src + ids[e]] : shot * p.n_sen + ids[e];
        if (row < 0)
            continue;
        const float I = p.inj_tab[(int64_t)row * p.T + p.t];
        pn = __fadd_rn(pn, I);
        if (strip)
            qn = __fadd_rn(qn, __fmul_rn(I, 0.5f));
    }
    f.px_out[o] = pn;
    if (strip)
        f.pz_out[o] = qn;
}

// The point work of a P-kernel CTA, after its lanes wrote P(t) (and Q(t))
// of its cells: lanes take distinct cells, so nothing races; __syncwarp
// orders the lanes' writes before these reads.
__device__ __forceinline__ void cta_inject(const StepParams &p, const Fields &f, int shot, const int *cta_idx,
                                           const int *off, const int *ptr, const int *ids, int cta, bool sources)
{
    for (int c = cta_idx[cta] + (int)threadIdx.x; c < cta_idx[cta + 1]; c += kUThreads)
        inject_cell(p, f, shot, off[c], ids, ptr[c], ptr[c + 1], sources);
}

// Resident CTAs each kernel is compiled for (a register cap), from
// measurements: 24 (80 registers) for the reverse P kernel, 28 (72) for the
// forward P and A kernels, 20 (96) for the reverse A kernel. The row loops of
// the P half-step and of the reverse adjoint A half-step are not unrolled
// (measured 2-3% faster than unrolled by 2 on the reverse step).
constexpr int kUPMinBlocks = 24;
constexpr int kUPFwdMinBlocks = 28;  // the forward P kernel fits 72 registers without spilling
constexpr int kUAMinBlocks = 28;

// Forward P half-step and the sources: grid (ncb, nseg, shots of the
// launch), shots upwards.
__global__ void __launch_bounds__(kUThreads, kUPFwdMinBlocks) k_unfused_p_fwd(const __grid_constant__ UnfusedParams U)
{
    pdl_enter();
    count_launch(U);
    const int x = blockIdx.x * kUCols + 4 * threadIdx.x;
    const int cta = blockIdx.x + U.ncb * blockIdx.y;
    if (x < U.p.X)
        p_segment<false>(U, U.p.f0, U.p.q0, U.shot0 + (int)blockIdx.z, x, blockIdx.y * kURows);
    __syncwarp();
    cta_inject(U.p, U.p.f0, U.shot0 + (int)blockIdx.z, U.src_cta, U.src_off, U.src_ptr, U.src_id, cta, true);
}

// Reverse P half-steps of both sets: grid (ncb, nseg, 2 * n_shots), shot
// z / 2 upwards; even z: reconstruction (set 0, q0) then the ring
// overwrite, odd z: adjoint (set 1, q1) then the adjoint sources.
__global__ void __launch_bounds__(kUThreads, kUPMinBlocks) k_unfused_p_rev(const __grid_constant__ UnfusedParams U)
{
    pdl_enter();
    count_launch(U);
    const StepParams &p = U.p;
    const int x = blockIdx.x * kUCols + 4 * threadIdx.x;
    const int cta = blockIdx.x + U.ncb * blockIdx.y;
    const bool rec_set = (blockIdx.z & 1u) == 0u;
    const int shot = U.shot0 + (int)(blockIdx.z >> 1);
    if (x < p.X) {
        if (rec_set)
            p_segment<true>(U, p.f0, p.q0, shot, x, blockIdx.y * kURows);
        else
            p_segment<false>(U, p.f1, p.q1, shot, x, blockIdx.y * kURows);
    }
    __syncwarp();
    if (rec_set) {
        // setRec: P_rec(t) = ring(T-1-t) on the ring cells of this CTA
        const float *ring = p.ring + ((int64_t)shot * p.T + (p.T - 1 - p.t)) * p.n_ring;
        for (int c = U.ring_cta[cta] + (int)threadIdx.x; c < U.ring_cta[cta + 1]; c += kUThreads)
            p.f0.px_out[p.shot_stride * shot + U.ring_cta_off[c]] = ring[U.ring_cta_k[c]];
    } else {
        cta_inject(p, p.f1, shot, U.rcv_cta, U.rcv_off, U.rcv_ptr, U.rcv_id, cta, false);
    }
}

// A update of one cell from the staggered derivatives of P(t): reverted,
// damped, or undamped with a single rounding.
__device__ __forceinline__ void a_update(const StepParams &p, bool revert, float dmx, float dmz, float dx, float dz,
                                         float ax, float az, bool in, float &nx, float &nz)
{
    if (revert) {
        nx = __fmaf_rn(-p.r, dx, ax);
        nz = __fmaf_rn(-p.r, dz, az);
    } else if (dmx != 1.f || dmz != 1.f) {
        nx = __fmaf_rn(ax, dmx, __fmul_rn(p.r, dx));
        nz = __fmaf_rn(az, dmz, __fmul_rn(p.r, dz));
    } else {
        nx = __fmaf_rn(p.r, dx, ax);
        nz = __fmaf_rn(p.r, dz, az);
    }
    if (!in) {
        nx = 0.f;
        nz = 0.f;
    }
}

// Forward A half-step of one 4-column segment of rows z0 .. z0+7 of a shot:
// Ax, Az (t) from P(t) (pld4<COHERENT>) and Ax, Az (t-1).
template <bool COHERENT>
__device__ __forceinline__ void a_fwd_segment(const UnfusedParams &U, int shot, int x, int z0)
{
    const StepParams &p = U.p;
    const int64_t so = p.shot_stride * shot;
    const float *__restrict__ P = p.f0.px_out + so;
    const float *__restrict__ AXI = p.f0.ax_in + so;
    const float *__restrict__ AZI = p.f0.az_in + so;
    float *__restrict__ AXO = p.f0.ax_out + so;
    float *__restrict__ AZO = p.f0.az_out + so;
    const int64_t col = x + PAD, pitch = p.pitch;
    float dmx[4];
    f4a(uld4(p.dampx + col), dmx);
    float w[4][8];
#pragma unroll
    for (int k = 0; k < 7; k++) {
        const float4 v = pld4<COHERENT>(P + (int64_t)(z0 - 3 + k + PAD) * pitch + col);
        w[0][k] = v.x;
        w[1][k] = v.y;
        w[2][k] = v.z;
        w[3][k] = v.w;
    }
    const int nz = min(kURows, p.Z - z0);
#pragma unroll 2
    for (int r = 0; r < nz; r++) {
        const int z = z0 + r;
        const int64_t o = (int64_t)(z + PAD) * pitch + col;
        {
            const float4 v = pld4<COHERENT>(P + o + 4 * pitch);
            w[0][7] = v.x;
            w[1][7] = v.y;
            w[2][7] = v.z;
            w[3][7] = v.w;
        }
        float u[12], ax[4], az[4], nx[4], nzv[4];
        f4a(pld4<COHERENT>(P + o - 4), u);
        f4a(pld4<COHERENT>(P + o), u + 4);
        f4a(pld4<COHERENT>(P + o + 4), u + 8);
        f4a(uld4(AXI + o), ax);
        f4a(uld4(AZI + o), az);
        const float dmz = __ldg(p.dampz + z + PAD);
        const bool zin = z >= 4 && z < p.Z - 4;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            float dx, dz;
            dstag_n<1>(u + j + 1, &dx);
            dstag_n<1>(w[j], &dz);
            a_update(p, false, dmx[j], dmz, dx, dz, ax[j], az[j], zin && x + j >= 4 && x + j < p.X - 4, nx[j],
                     nzv[j]);
        }
        ust4(AXO + o, nx);
        ust4(AZO + o, nzv);
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int k = 0; k < 7; k++)
                w[j][k] = w[j][k + 1];
    }
}

// Forward A half-step: grid (ncb, n_tail + nseg, n_shots), shots downwards;
// the first n_tail rows of CTAs record the receivers (and the ring) of their
// shot: first, so that these latency-bound CTAs run beside the stencil CTAs,
// not after them.
__global__ void __launch_bounds__(kUThreads, kUAMinBlocks) k_unfused_a_fwd(const __grid_constant__ UnfusedParams U)
{
    pdl_enter();
    count_launch(U);
    const StepParams &p = U.p;
    const int shot = U.shot0 + (int)(gridDim.z - 1u - blockIdx.z);
    const int64_t so = p.shot_stride * shot;
    const float *__restrict__ P = p.f0.px_out + so;
    const int n_tail = gridDim.y - U.nseg;
    if ((int)blockIdx.y < n_tail) {
        // recording CTAs: each thread records up to kUTailPer cells, strided
        const int n = p.n_sen + (U.record_ring ? p.n_ring : 0);
        const int stride = n_tail * U.ncb * kUThreads;
        for (int i = (blockIdx.y * U.ncb + blockIdx.x) * kUThreads + threadIdx.x; i < n; i += stride) {
            if (i < p.n_sen) {
                p.rec[((int64_t)shot * p.n_sen + i) * p.T + p.t] = P[U.rec_off[i]];
            } else {
                const int k = i - p.n_sen;
                p.ring[((int64_t)shot * p.T + p.t) * p.n_ring + k] = P[U.ring_off[k]];
            }
        }
        return;
    }
    const int x = blockIdx.x * kUCols + 4 * threadIdx.x;
    if (x >= p.X)
        return;
    a_fwd_segment<false>(U, shot, x, (blockIdx.y - n_tail) * kURows);
}

// Reverse A half-steps of both sets and the imaging condition on one
// 4-column segment of rows z0 .. z0+7 of a shot (P(t) of both sets read with
// pld4<COHERENT>).
template <bool COHERENT>
__device__ __forceinline__ void a_rev_segment(const UnfusedParams &U, int shot, int x, int z0)
{
    const StepParams &p = U.p;
    const int64_t so = p.shot_stride * shot;
    const float *__restrict__ PR = p.f0.px_out + so;
    const float *__restrict__ PA = p.f1.px_out + so;
    const int64_t col = x + PAD, pitch = p.pitch;
    float dmx[4];
    f4a(uld4(p.dampx + col), dmx);
    bool xin[4];
#pragma unroll
    for (int j = 0; j < 4; j++)
        xin[j] = x + j >= 4 && x + j < p.X - 4;
    float wr[4][9], wa[4][8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const float4 v = pld4<COHERENT>(PR + (int64_t)(z0 - 4 + k + PAD) * pitch + col);
        wr[0][k] = v.x;
        wr[1][k] = v.y;
        wr[2][k] = v.z;
        wr[3][k] = v.w;
    }
#pragma unroll
    for (int k = 0; k < 7; k++) {
        const float4 v = pld4<COHERENT>(PA + (int64_t)(z0 - 3 + k + PAD) * pitch + col);
        wa[0][k] = v.x;
        wa[1][k] = v.y;
        wa[2][k] = v.z;
        wa[3][k] = v.w;
    }
    const int nz = min(kURows, p.Z - z0);
    for (int r = 0; r < nz; r++) {
        const int z = z0 + r;
        const int64_t o = (int64_t)(z + PAD) * pitch + col;
        const bool zin = z >= 4 && z < p.Z - 4;
        {
            const float4 v = pld4<COHERENT>(PR + o + 4 * pitch);
            wr[0][8] = v.x;
            wr[1][8] = v.y;
            wr[2][8] = v.z;
            wr[3][8] = v.w;
            const float4 a = pld4<COHERENT>(PA + o + 4 * pitch);
            wa[0][7] = a.x;
            wa[1][7] = a.y;
            wa[2][7] = a.z;
            wa[3][7] = a.w;
        }
        float lap[4];
        {
            // reconstruction: reverted A update and the Laplacian of P_rec(t)
            float u[12], ax[4], az[4], nx[4], nzv[4];
            f4a(pld4<COHERENT>(PR + o - 4), u);
            f4a(pld4<COHERENT>(PR + o), u + 4);
            f4a(pld4<COHERENT>(PR + o + 4), u + 8);
            f4a(uld4(p.f0.ax_in + so + o), ax);
            f4a(uld4(p.f0.az_in + so + o), az);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                float dx, dz, lx, lz;
                dstag_n<1>(u + j + 1, &dx);
                dstag_n<1>(wr[j] + 1, &dz);
                lap_n<1>(u + j, &lx);
                lap_n<1>(wr[j], &lz);
                lap[j] = lap_combine(lx, lz);
                a_update(p, true, 1.f, 1.f, dx, dz, ax[j], az[j], xin[j] && zin, nx[j], nzv[j]);
            }
            ust4(p.f0.ax_out + so + o, nx);
            ust4(p.f0.az_out + so + o, nzv);
        }
        {
            // adjoint: damped A update and the imaging condition
            float u[12], ax[4], az[4], nx[4], nzv[4], g[4];
            f4a(pld4<COHERENT>(PA + o - 4), u);
            f4a(pld4<COHERENT>(PA + o), u + 4);
            f4a(pld4<COHERENT>(PA + o + 4), u + 8);
            f4a(uld4(p.f1.ax_in + so + o), ax);
            f4a(uld4(p.f1.az_in + so + o), az);
            f4a(uld4c(p.grad + so + o), g);
            const float dmz = __ldg(p.dampz + z + PAD);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                float dx, dz;
                dstag_n<1>(u + j + 1, &dx);
                dstag_n<1>(wa[j], &dz);
                a_update(p, false, dmx[j], dmz, dx, dz, ax[j], az[j], xin[j] && zin, nx[j], nzv[j]);
                g[j] = __fmaf_rn(u[4 + j], lap[j], g[j]);
            }
            ust4(p.f1.ax_out + so + o, nx);
            ust4(p.f1.az_out + so + o, nzv);
            ust4(p.grad + so + o, g);
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
#pragma unroll
            for (int k = 0; k < 8; k++)
                wr[j][k] = wr[j][k + 1];
#pragma unroll
            for (int k = 0; k < 7; k++)
                wa[j][k] = wa[j][k + 1];
        }
    }
}

// The reverse A half-step split by field set, for twice the CTAs at a lower
// register count than a_rev_segment (the same arithmetic, bit for bit):
// the reconstruction set with the Laplacian of P_rec(t) and the imaging
// condition (P_adj(t) read on the CTA's own cells) ...
__device__ __forceinline__ void a_rev_rec_segment(const UnfusedParams &U, int shot, int x, int z0)
{
    const StepParams &p = U.p;
    const int64_t so = p.shot_stride * shot;
    const float *__restrict__ PR = p.f0.px_out + so;
    const float *__restrict__ PA = p.f1.px_out + so;
    const int64_t col = x + PAD, pitch = p.pitch;
    bool xin[4];
#pragma unroll
    for (int j = 0; j < 4; j++)
        xin[j] = x + j >= 4 && x + j < p.X - 4;
    float wr[4][9];
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const float4 v = uld4(PR + (int64_t)(z0 - 4 + k + PAD) * pitch + col);
        wr[0][k] = v.x;
        wr[1][k] = v.y;
        wr[2][k] = v.z;
        wr[3][k] = v.w;
    }
    const int nz = min(kURows, p.Z - z0);
    for (int r = 0; r < nz; r++) {
        const int z = z0 + r;
        const int64_t o = (int64_t)(z + PAD) * pitch + col;
        const bool zin = z >= 4 && z < p.Z - 4;
        {
            const float4 v = uld4(PR + o + 4 * pitch);
            wr[0][8] = v.x;
            wr[1][8] = v.y;
            wr[2][8] = v.z;
            wr[3][8] = v.w;
        }
        float u[12], ax[4], az[4], nx[4], nzv[4], lap[4], pa[4], g[4];
        f4a(uld4(PR + o - 4), u);
        f4a(uld4(PR + o), u + 4);
        f4a(uld4(PR + o + 4), u + 8);
        f4a(uld4(p.f0.ax_in + so + o), ax);
        f4a(uld4(p.f0.az_in + so + o), az);
        f4a(uld4(PA + o), pa);
        f4a(uld4c(p.grad + so + o), g);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            float dx, dz, lx, lz;
            dstag_n<1>(u + j + 1, &dx);
            dstag_n<1>(wr[j] + 1, &dz);
            lap_n<1>(u + j, &lx);
            lap_n<1>(wr[j], &lz);
            lap[j] = lap_combine(lx, lz);
            a_update(p, true, 1.f, 1.f, dx, dz, ax[j], az[j], xin[j] && zin, nx[j], nzv[j]);
            g[j] = __fmaf_rn(pa[j], lap[j], g[j]);
        }
        ust4(p.f0.ax_out + so + o, nx);
        ust4(p.f0.az_out + so + o, nzv);
        ust4(p.grad + so + o, g);
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int k = 0; k < 8; k++)
                wr[j][k] = wr[j][k + 1];
    }
}

// ... and the adjoint set (damped A update).
__device__ __forceinline__ void a_rev_adj_segment(const UnfusedParams &U, int shot, int x, int z0)
{
    const StepParams &p = U.p;
    const int64_t so = p.shot_stride * shot;
    const float *__restrict__ PA = p.f1.px_out + so;
    const int64_t col = x + PAD, pitch = p.pitch;
    float dmx[4];
    f4a(uld4(p.dampx + col), dmx);
    bool xin[4];
#pragma unroll
    for (int j = 0; j < 4; j++)
        xin[j] = x + j >= 4 && x + j < p.X - 4;
    float wa[4][8];
#pragma unroll
    for (int k = 0; k < 7; k++) {
        const float4 v = uld4(PA + (int64_t)(z0 - 3 + k + PAD) * pitch + col);
        wa[0][k] = v.x;
        wa[1][k] = v.y;
        wa[2][k] = v.z;
        wa[3][k] = v.w;
    }
    const int nz = min(kURows, p.Z - z0);
#pragma unroll 1
    for (int r = 0; r < nz; r++) {
        const int z = z0 + r;
        const int64_t o = (int64_t)(z + PAD) * pitch + col;
        const bool zin = z >= 4 && z < p.Z - 4;
        {
            const float4 a = uld4(PA + o + 4 * pitch);
            wa[0][7] = a.x;
            wa[1][7] = a.y;
            wa[2][7] = a.z;
            wa[3][7] = a.w;
        }
        float u[12], ax[4], az[4], nx[4], nzv[4];
        f4a(uld4(PA + o - 4), u);
        f4a(uld4(PA + o), u + 4);
        f4a(uld4(PA + o + 4), u + 8);
        f4a(uld4(p.f1.ax_in + so + o), ax);
        f4a(uld4(p.f1.az_in + so + o), az);
        const float dmz = __ldg(p.dampz + z + PAD);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            float dx, dz;
            dstag_n<1>(u + j + 1, &dx);
            dstag_n<1>(wa[j], &dz);
            a_update(p, false, dmx[j], dmz, dx, dz, ax[j], az[j], xin[j] && zin, nx[j], nzv[j]);
        }
        ust4(p.f1.ax_out + so + o, nx);
        ust4(p.f1.az_out + so + o, nzv);
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int k = 0; k < 7; k++)
                wa[j][k] = wa[j][k + 1];
    }
}

// Reverse A half-steps split by set: grid (ncb, nseg, 2 * n_shots), shot
// (z / 2) downwards; even z: reconstruction + imaging, odd z: adjoint.
// Register cap from a sweep (16 / 20 / 24 resident CTAs: 115 / 96 / 80
// registers, the last spilling): 20 is the fastest.
constexpr int kUARevMinBlocks = 20;
template <int MINB>
__global__ void __launch_bounds__(kUThreads, MINB) k_unfused_a_rev_sets(const __grid_constant__ UnfusedParams U)
{
    pdl_enter();
    count_launch(U);
    const int x = blockIdx.x * kUCols + 4 * threadIdx.x;
    if (x >= U.p.X)
        return;
    const int shot = U.shot0 + (int)(gridDim.z / 2u - 1u - (blockIdx.z >> 1));
    if ((blockIdx.z & 1u) == 0u)
        a_rev_rec_segment(U, shot, x, blockIdx.y * kURows);
    else
        a_rev_adj_segment(U, shot, x, blockIdx.y * kURows);
}

// Reverse A half-steps of both sets and the imaging condition: grid (ncb,
// nseg, n_shots), shots downwards.
__global__ void __launch_bounds__(kUThreads) k_unfused_a_rev(const __grid_constant__ UnfusedParams U)
{
    pdl_enter();
    count_launch(U);
    const int x = blockIdx.x * kUCols + 4 * threadIdx.x;
    if (x >= U.p.X)
        return;
    a_rev_segment<false>(U, U.shot0 + (int)(gridDim.z - 1u - blockIdx.z), x, blockIdx.y * kURows);
}

}  // namespace otf
