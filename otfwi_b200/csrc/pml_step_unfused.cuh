// Unfused streaming step kernels for the fast numerics (variant 4).
//
// The fused kernels (pml_step_split.cuh, pml_step_stream.cuh) compute P(t)
// and A(t) of a tile in one pass, recomputing P on a 4-cell halo and
// synchronising the CTA between the two half-steps. Here each half-step is
// its own launch over the whole batch and every cell is computed once:
//
//   forward step:  P kernel  P(t), Q(t) from P, Q, Ax, Az (t-1), sources
//                  A kernel  Ax, Az (t) from P(t); extra CTAs record the
//                            receivers and the boundary ring
//   reverse step:  P kernel  both field sets: reconstruction (undamped,
//                            reverted) and adjoint (damped, receivers)
//                  ring      P_rec(t) = ring(T-1-t) on the ring cells
//                  A kernel  both A updates, the 9-point Laplacian of
//                            P_rec(t) and grad += P_adj(t) * lap
//
// A thread owns one column of a 128-column block and marches down R rows:
// z-derivatives come from a sliding register window of the column, the
// x-derivatives from eight neighbouring columns read through L1. No shared
// memory, no block barrier, about 32 registers: the SMs hold up to 16 CTAs
// and the loads of many rows are in flight. The cell arithmetic is that of
// the strip-split kernels (same pair-form staggered sums, same update and
// injection order), with the damped A update used exactly on damped cells.
// This moves 40 bytes per forward cell-step and 92 per reverse cell-step
// instead of 28 and 64, and trades them for full-rate streaming.
#pragma once
#include "pml_step.cuh"
#include "pml_step_split.cuh"

namespace otf {

constexpr int kUCols = 128;  // columns (threads) per CTA

struct UnfusedParams {
    StepParams p;
    int ncb, nseg;  // column blocks, row segments per shot
    // injection points per stencil CTA (cb + ncb * seg), in source / receiver
    // order: local column | local row << 8, and the source / receiver index
    const int *src_ptr, *src_pos, *src_id;
    const int *rcv_ptr, *rcv_pos, *rcv_id;
    // padded offsets of the receivers and of the ring cells (ring order)
    const int64_t *rec_off, *ring_off;
    int record_ring;  // forward: also record the boundary ring
};

__device__ __forceinline__ float ustag(const float *u)
{
    float o;
    dstag_n<1>(u, &o);
    return o;
}

// Injection points of this thread's column within the CTA's segment: the
// first two are kept in registers; more (never seen in practice) switch the
// thread to a scan of the CTA's list per row.
struct ColumnPoints {
    int r0 = -1, id0 = 0, r1 = -1, id1 = 0;
    int e_begin = 0, e_end = 0;
    bool scan = false;
};

__device__ __forceinline__ ColumnPoints column_points(const int *ptr, const int *pos, const int *id, int cta)
{
    ColumnPoints c;
    c.e_begin = ptr[cta];
    c.e_end = ptr[cta + 1];
    int n = 0;
    for (int e = c.e_begin; e < c.e_end; e++) {
        const int v = pos[e];
        if ((v & 0xff) != (int)threadIdx.x)
            continue;
        if (n == 0) {
            c.r0 = v >> 8;
            c.id0 = id[e];
        } else if (n == 1) {
            c.r1 = v >> 8;
            c.id1 = id[e];
        }
        n++;
    }
    c.scan = n > 2;
    return c;
}

// P += I (both split components get I/2), Q += I/2 on strip cells
template <bool SOURCES>
__device__ __forceinline__ void inject_one(const StepParams &p, int shot, int id, bool strip, float &pn, float &qn)
{
    const int row = SOURCES ? p.fire_row[shot * p.n_src + id] : shot * p.n_sen + id;
    if (row < 0)
        return;
    const float I = p.inj_tab[(int64_t)row * p.T + p.t];
    pn = __fadd_rn(pn, I);
    if (strip)
        qn = __fadd_rn(qn, __fmul_rn(I, 0.5f));
}

// One column segment of a P half-step. REVERT: time-reversed reconstruction
// (undamped, no Q, no injection); otherwise damped with the strip component
// Q and point injection (SOURCES: the shot's firing sources, else the
// adjoint sources at the receivers).
template <int R, bool REVERT, bool SOURCES>
__device__ __forceinline__ void p_column(const UnfusedParams &U, const Fields &f, const float *__restrict__ q,
                                         int shot, int x, int z0, int cta)
{
    const StepParams &p = U.p;
    const int64_t so = p.shot_stride * shot;
    const float *__restrict__ AX = f.ax_in + so;
    const float *__restrict__ AZ = f.az_in + so;
    const float *__restrict__ PI = f.px_in + so;
    const float *__restrict__ QI = f.pz_in + so;
    float *__restrict__ PO = f.px_out + so;
    float *__restrict__ QO = f.pz_out + so;
    const int64_t col = x + PAD;
    const int64_t pitch = p.pitch;
    ColumnPoints pts;
    if (!REVERT)
        pts = SOURCES ? column_points(U.src_ptr, U.src_pos, U.src_id, cta)
                      : column_points(U.rcv_ptr, U.rcv_pos, U.rcv_id, cta);
    const float dmx = REVERT ? 1.f : __ldg(p.dampx + col);
    const bool xin = x >= 4 && x < p.X - 4;
    float w[8];
#pragma unroll
    for (int k = 0; k < 7; k++)
        w[k] = __ldg(AZ + (int64_t)(z0 - 4 + k + PAD) * pitch + col);
    const int nz = min(R, p.Z - z0);
#pragma unroll 4
    for (int r = 0; r < nz; r++) {
        const int z = z0 + r;
        const int64_t o = (int64_t)(z + PAD) * pitch + col;
        w[7] = __ldg(AZ + o + 3 * pitch);
        float u[8];
#pragma unroll
        for (int k = 0; k < 8; k++)
            u[k] = __ldg(AX + o - 4 + k);
        const float dAx = ustag(u), dAz = ustag(w);
        const float po = __ldg(PI + o), qv = __ldg(q + o);
        const float s = __fadd_rn(dAx, dAz);
        float pn, qn = 0.f;
        bool strip = false;
        if (REVERT) {
            pn = __fmaf_rn(-qv, s, po);
        } else {
            const float dmz = __ldg(p.dampz + z + PAD);
            if (dmx != 1.f || dmz != 1.f) {
                strip = true;
                const float qo = __ldg(QI + o);
                const float q1 = __fmaf_rn(qo, dmx, __fmul_rn(qv, dAx));
                const float z1 = __fmaf_rn(__fsub_rn(po, qo), dmz, __fmul_rn(qv, dAz));
                qn = q1;
                pn = __fadd_rn(q1, z1);
            } else {
                pn = __fmaf_rn(qv, s, po);
            }
        }
        if (!xin || z < 4 || z >= p.Z - 4) {
            pn = 0.f;
            qn = 0.f;
        }
        if (!REVERT) {
            if (pts.scan) {
                for (int e = pts.e_begin; e < pts.e_end; e++) {
                    const int v = SOURCES ? U.src_pos[e] : U.rcv_pos[e];
                    if ((v & 0xff) == (int)threadIdx.x && (v >> 8) == r)
                        inject_one<SOURCES>(p, shot, SOURCES ? U.src_id[e] : U.rcv_id[e], strip, pn, qn);
                }
            } else {
                if (pts.r0 == r)
                    inject_one<SOURCES>(p, shot, pts.id0, strip, pn, qn);
                if (pts.r1 == r)
                    inject_one<SOURCES>(p, shot, pts.id1, strip, pn, qn);
            }
        }
        PO[o] = pn;
        if (strip)
            QO[o] = qn;
#pragma unroll
        for (int k = 0; k < 7; k++)
            w[k] = w[k + 1];
    }
}

// Forward P half-step: grid (ncb, nseg, n_shots).
template <int R>
__global__ void __launch_bounds__(kUCols) k_unfused_p_fwd(const __grid_constant__ UnfusedParams U)
{
    const int x = blockIdx.x * kUCols + threadIdx.x;
    if (x >= U.p.X)
        return;
    p_column<R, false, true>(U, U.p.f0, U.p.q0, blockIdx.z, x, blockIdx.y * R, blockIdx.x + U.ncb * blockIdx.y);
}

// Reverse P half-steps of both sets: grid (ncb, nseg, 2 * n_shots); z <
// n_shots: reconstruction (set 0, q0), else adjoint (set 1, q1).
template <int R>
__global__ void __launch_bounds__(kUCols) k_unfused_p_rev(const __grid_constant__ UnfusedParams U, int n_shots)
{
    const int x = blockIdx.x * kUCols + threadIdx.x;
    if (x >= U.p.X)
        return;
    const int cta = blockIdx.x + U.ncb * blockIdx.y;
    if ((int)blockIdx.z < n_shots)
        p_column<R, true, false>(U, U.p.f0, U.p.q0, blockIdx.z, x, blockIdx.y * R, cta);
    else
        p_column<R, false, false>(U, U.p.f1, U.p.q1, blockIdx.z - n_shots, x, blockIdx.y * R, cta);
}

// A update of one cell from the staggered derivatives of P(t): reverted,
// undamped (single rounding) or damped.
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

// Forward A half-step: grid (ncb, nseg + n_tail, n_shots); rows of CTAs
// past nseg record the receivers (and the ring) of their shot.
template <int R>
__global__ void __launch_bounds__(kUCols) k_unfused_a_fwd(const __grid_constant__ UnfusedParams U)
{
    const StepParams &p = U.p;
    const int shot = blockIdx.z;
    const int64_t so = p.shot_stride * shot;
    const float *__restrict__ P = p.f0.px_out + so;
    if ((int)blockIdx.y >= U.nseg) {
        const int i = ((blockIdx.y - U.nseg) * U.ncb + blockIdx.x) * kUCols + threadIdx.x;
        if (i < p.n_sen) {
            p.rec[((int64_t)shot * p.n_sen + i) * p.T + p.t] = P[U.rec_off[i]];
        } else if (U.record_ring && i - p.n_sen < p.n_ring) {
            const int k = i - p.n_sen;
            p.ring[((int64_t)shot * p.T + p.t) * p.n_ring + k] = P[U.ring_off[k]];
        }
        return;
    }
    const int x = blockIdx.x * kUCols + threadIdx.x;
    if (x >= p.X)
        return;
    const int z0 = blockIdx.y * R;
    const float *__restrict__ AXI = p.f0.ax_in + so;
    const float *__restrict__ AZI = p.f0.az_in + so;
    float *__restrict__ AXO = p.f0.ax_out + so;
    float *__restrict__ AZO = p.f0.az_out + so;
    const int64_t col = x + PAD, pitch = p.pitch;
    const float dmx = __ldg(p.dampx + col);
    const bool xin = x >= 4 && x < p.X - 4;
    float w[8];
#pragma unroll
    for (int k = 0; k < 7; k++)
        w[k] = P[(int64_t)(z0 - 3 + k + PAD) * pitch + col];
    const int nz = min(R, p.Z - z0);
#pragma unroll 4
    for (int r = 0; r < nz; r++) {
        const int z = z0 + r;
        const int64_t o = (int64_t)(z + PAD) * pitch + col;
        w[7] = P[o + 4 * pitch];
        float u[8];
#pragma unroll
        for (int k = 0; k < 8; k++)
            u[k] = P[o - 3 + k];
        float nx, nz_;
        a_update(p, false, dmx, __ldg(p.dampz + z + PAD), ustag(u), ustag(w), AXI[o], AZI[o],
                 xin && z >= 4 && z < p.Z - 4, nx, nz_);
        AXO[o] = nx;
        AZO[o] = nz_;
#pragma unroll
        for (int k = 0; k < 7; k++)
            w[k] = w[k + 1];
    }
}

// Reverse A half-steps of both sets and the imaging condition: grid (ncb,
// nseg, n_shots).
template <int R>
__global__ void __launch_bounds__(kUCols) k_unfused_a_rev(const __grid_constant__ UnfusedParams U)
{
    const StepParams &p = U.p;
    const int x = blockIdx.x * kUCols + threadIdx.x;
    if (x >= p.X)
        return;
    const int shot = blockIdx.z, z0 = blockIdx.y * R;
    const int64_t so = p.shot_stride * shot;
    const float *__restrict__ PR = p.f0.px_out + so;
    const float *__restrict__ PA = p.f1.px_out + so;
    const int64_t col = x + PAD, pitch = p.pitch;
    const float dmx = __ldg(p.dampx + col);
    const bool xin = x >= 4 && x < p.X - 4;
    float wr[9], wa[8];
#pragma unroll
    for (int k = 0; k < 8; k++)
        wr[k] = PR[(int64_t)(z0 - 4 + k + PAD) * pitch + col];
#pragma unroll
    for (int k = 0; k < 7; k++)
        wa[k] = PA[(int64_t)(z0 - 3 + k + PAD) * pitch + col];
    const int nz = min(R, p.Z - z0);
#pragma unroll 2
    for (int r = 0; r < nz; r++) {
        const int z = z0 + r;
        const int64_t o = (int64_t)(z + PAD) * pitch + col;
        const bool in = xin && z >= 4 && z < p.Z - 4;
        wr[8] = PR[o + 4 * pitch];
        wa[7] = PA[o + 4 * pitch];
        // reconstruction: reverted A update and the Laplacian of P_rec(t)
        float u[9];
#pragma unroll
        for (int k = 0; k < 9; k++)
            u[k] = PR[o - 4 + k];
        float lx, lz;
        lap_n<1>(u, &lx);
        lap_n<1>(wr, &lz);
        float nx, nz_;
        a_update(p, true, 1.f, 1.f, ustag(u + 1), ustag(wr + 1), p.f0.ax_in[so + o], p.f0.az_in[so + o], in, nx,
                 nz_);
        p.f0.ax_out[so + o] = nx;
        p.f0.az_out[so + o] = nz_;
        // adjoint: damped A update and the imaging condition
        float v[8];
#pragma unroll
        for (int k = 0; k < 8; k++)
            v[k] = PA[o - 3 + k];
        a_update(p, false, dmx, __ldg(p.dampz + z + PAD), ustag(v), ustag(wa), p.f1.ax_in[so + o],
                 p.f1.az_in[so + o], in, nx, nz_);
        p.f1.ax_out[so + o] = nx;
        p.f1.az_out[so + o] = nz_;
        p.grad[so + o] = __fmaf_rn(v[3], lap_combine(lx, lz), p.grad[so + o]);
#pragma unroll
        for (int k = 0; k < 8; k++)
            wr[k] = wr[k + 1];
#pragma unroll
        for (int k = 0; k < 7; k++)
            wa[k] = wa[k + 1];
    }
}

// Reverse: P_rec(t) = ring(T-1-t) on the ring cells: grid (ceil(n_ring /
// 256), n_shots).
__global__ void k_unfused_ring(const __grid_constant__ UnfusedParams U)
{
    const StepParams &p = U.p;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= p.n_ring)
        return;
    const int shot = blockIdx.y;
    p.f0.px_out[p.shot_stride * shot + U.ring_off[k]] =
        p.ring[((int64_t)shot * p.T + (p.T - 1 - p.t)) * p.n_ring + k];
}

}  // namespace otf
