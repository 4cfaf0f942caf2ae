// Row-lag fused step kernels for the fast numerics (variant 6): both
// half-steps of a time step in one pass over the fields, with no dependency
// between CTAs.
//
// The unfused kernels (pml_step_unfused.cuh) run the P and the A half-steps as
// separate launches, so the A launch re-reads from DRAM the P(t) the P launch
// has just written and the A(t-1) it has just read: about 81 bytes per cell of
// a reverse step move where 56 are compulsory. Here one warp owns a strip of
// columns of one shot and marches down a chunk of rows. At row r it computes
// P(t) of row r (then the sources, receivers, ring cells of that row), keeps
// it in a register window of the last nine P(t) rows, and computes the A
// half-step of row r - 4 from that window: the z taps from the window, the x
// taps from the neighbouring lanes' windows by warp shuffles. Every field is
// read and written once per step (inputs of the first and last 4 rows of a
// chunk twice).
//
// The x taps reach 4 columns beyond a lane's 4: a warp computes P(t) on 128
// columns and the A half-step on the middle 120 (lanes 1 .. 30); lanes 0 and
// 31 compute the 4 halo columns on either side, which the neighbouring warp
// owns and writes. Likewise a chunk computes P(t) on 4 halo rows above and
// below its own rows. Sources, adjoint sources and the ring overwrite are
// applied on halo cells too (the A taps see them); P, Q, A, receivers and the
// ring are written only by the owner.
//
// Reverse step: a CTA of two warps on the same columns and rows, warp 0 the
// time-reversed reconstruction (undamped), warp 1 the adjoint (damped); warp 0
// hands the 9-point Laplacian of P_rec(t) of each row to warp 1 through shared
// memory (double-buffered, one named barrier of the two warps per row), and
// warp 1 adds P_adj(t) * lap to the gradient.
//
// The cell arithmetic is that of the unfused kernels operation for operation
// (the same device functions, the same order of the injections), so the
// results are bit-identical to them.
#pragma once
#include "pml_step_unfused.cuh"

namespace otf {

constexpr int kFLanes = 32;            // one warp per set
constexpr int kFCols = 4 * kFLanes;    // columns a warp computes P(t) on
constexpr int kFInner = kFCols - 8;    // columns it owns (lanes 1 .. 30)

struct FusedParams {
    StepParams p;
    int nxb;            // column strips of kFInner owned columns
    int chunk;          // rows per chunk
    const int *ringmap;  // padded [rows][pitch]: ring index of the cell, or -1
    // point cells by row (CSR over the Z rows): column and the cell's point
    // range [ce[c], ce[c+1]) into id (increasing source / receiver indices)
    const int *src_rp, *src_cx, *src_ce, *src_id;  // sources (forward)
    const int *rcv_rp, *rcv_cx, *rcv_ce, *rcv_id;  // injectable receivers (adjoint sources)
    const int *rec_rp, *rec_cx, *rec_id;           // every receiver, one entry each (recording)
    int record_ring;
};

// Sources (forward) or adjoint sources (reverse, adjoint set) of row z on
// this lane's 4 columns, in point order as inject_cell adds them.
__device__ __forceinline__ void fused_inject(const StepParams &p, const int *rp, const int *cx, const int *ce,
                                             const int *id, bool sources, int shot, int z, int x, float *pn,
                                             float *qn, const bool *strip)
{
    for (int c = rp[z]; c < rp[z + 1]; c++) {
        const int j = cx[c] - x;
        if (j < 0 || j > 3)
            continue;
        for (int e = ce[c]; e < ce[c + 1]; e++) {
            const int row = sources ? p.fire_row[shot * p.n_src + id[e]] : shot * p.n_sen + id[e];
            if (row < 0)
                continue;
            const float I = p.inj_tab[(int64_t)row * p.T + p.t];
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (k == j) {
                    pn[k] = __fadd_rn(pn[k], I);
                    if (strip[k])
                        qn[k] = __fadd_rn(qn[k], __fmul_rn(I, 0.5f));
                }
        }
    }
}

// P half-step of row z on this lane's 4 columns (p_segment's arithmetic):
// inputs P, Q (t-1) of the row, Ax (t-1) of the row at columns x-4 .. x+7,
// the Az (t-1) window of rows z-4 .. z+3.
__device__ __forceinline__ void fused_p_row(const StepParams &p, const Fields &f, const float *q, int64_t so,
                                            bool revert, int x, int z, const float (*w)[8], float *pn, float *qn,
                                            bool *strip, bool &damp)
{
    const int64_t col = x + PAD, pitch = p.pitch;
    const int64_t o = (int64_t)(z + PAD) * pitch + col;
    float u[12], po[4], qv[4], qo[4] = {0.f, 0.f, 0.f, 0.f};
    float dmx[4] = {1.f, 1.f, 1.f, 1.f};
    float dmz = 1.f;
    f4a(uld4(f.ax_in + so + o - 4), u);
    f4a(uld4(f.ax_in + so + o), u + 4);
    f4a(uld4(f.ax_in + so + o + 4), u + 8);
    f4a(uld4(f.px_in + so + o), po);
    f4a(uld4(q + o), qv);
    if (!revert) {
        f4a(uld4(p.dampx + col), dmx);
        dmz = __ldg(p.dampz + z + PAD);
    }
    damp = !revert && (dmx[0] != 1.f || dmx[1] != 1.f || dmx[2] != 1.f || dmx[3] != 1.f || dmz != 1.f);
    if (damp)
        f4a(uld4(f.pz_in + so + o), qo);
    const bool zin = z >= 4 && z < p.Z - 4;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        float dAx, dAz;
        dstag_n<1>(u + j, &dAx);
        dstag_n<1>(w[j], &dAz);
        const float s = __fadd_rn(dAx, dAz);
        qn[j] = 0.f;
        strip[j] = !revert && (dmx[j] != 1.f || dmz != 1.f);
        if (revert) {
            pn[j] = __fmaf_rn(-qv[j], s, po[j]);
        } else if (strip[j]) {
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
}

// x taps of row values v (this lane's 4 columns) from the neighbouring
// lanes: u[0..3] = left lane's, u[4..7] = own, u[8..11] = right lane's.
__device__ __forceinline__ void fused_row_taps(const float *v, float *u)
{
#pragma unroll
    for (int k = 0; k < 4; k++) {
        u[k] = __shfl_up_sync(0xffffffffu, v[k], 1);
        u[4 + k] = v[k];
        u[8 + k] = __shfl_down_sync(0xffffffffu, v[k], 1);
    }
}

// Forward step: grid (nxb, ceil(Z / chunk), n_shots), one warp per CTA.
template <int MINB>
__global__ void __launch_bounds__(kFLanes, MINB) k_fused_fwd(const __grid_constant__ FusedParams F)
{
    pdl_enter();
    const StepParams &p = F.p;
    const int lane = threadIdx.x, shot = blockIdx.z;
    const int x = (int)blockIdx.x * kFInner - 4 + 4 * lane;
    const bool active = x < p.X;
    const bool own_x = active && lane >= 1 && lane <= 30;
    const int z0 = blockIdx.y * F.chunk, z1 = min(p.Z, z0 + F.chunk);
    const int64_t so = p.shot_stride * shot, col = x + PAD, pitch = p.pitch;
    const Fields &f = p.f0;
    float w[4][8], pw[4][9], dmx[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
#pragma unroll
        for (int k = 0; k < 9; k++)
            pw[j][k] = 0.f;
        dmx[j] = 1.f;
    }
    if (active) {
        f4a(uld4(p.dampx + col), dmx);
#pragma unroll
        for (int k = 0; k < 7; k++) {
            const float4 v = uld4(f.az_in + so + (int64_t)(z0 - 8 + k + PAD) * pitch + col);
            w[0][k] = v.x;
            w[1][k] = v.y;
            w[2][k] = v.z;
            w[3][k] = v.w;
        }
    }
    for (int r = z0 - 4; r < z1 + 4; r++) {
        float pn[4] = {0.f, 0.f, 0.f, 0.f}, qn[4] = {0.f, 0.f, 0.f, 0.f};
        if (active) {
            const float4 v = uld4(f.az_in + so + (int64_t)(r + 3 + PAD) * pitch + col);
            w[0][7] = v.x;
            w[1][7] = v.y;
            w[2][7] = v.z;
            w[3][7] = v.w;
            bool strip[4], damp;
            fused_p_row(p, f, p.q0, so, false, x, r, w, pn, qn, strip, damp);
            if (r >= 0 && r < p.Z) {
                fused_inject(p, F.src_rp, F.src_cx, F.src_ce, F.src_id, true, shot, r, x, pn, qn, strip);
                if (own_x && r >= z0 && r < z1) {
                    const int64_t o = (int64_t)(r + PAD) * pitch + col;
                    ust4(f.px_out + so + o, pn);
                    if (damp)
                        ust4(f.pz_out + so + o, qn);
                    for (int c = F.rec_rp[r]; c < F.rec_rp[r + 1]; c++) {
                        const int j = F.rec_cx[c] - x;
                        if (j >= 0 && j < 4)
                            p.rec[((int64_t)shot * p.n_sen + F.rec_id[c]) * p.T + p.t] = pn[j];
                    }
                    if (F.record_ring) {
                        const int4 km = *reinterpret_cast<const int4 *>(F.ringmap + o);
                        const int kk[4] = {km.x, km.y, km.z, km.w};
                        float *ring = p.ring + ((int64_t)shot * p.T + p.t) * p.n_ring;
#pragma unroll
                        for (int j = 0; j < 4; j++)
                            if (kk[j] >= 0)
                                ring[kk[j]] = pn[j];
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < 4; j++)
#pragma unroll
                for (int k = 0; k < 7; k++)
                    w[j][k] = w[j][k + 1];
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
#pragma unroll
            for (int k = 0; k < 8; k++)
                pw[j][k] = pw[j][k + 1];
            pw[j][8] = pn[j];
        }
        // A half-step of row z = r - 4 (pw rows z-4 .. z+4)
        const int z = r - 4;
        if (z < z0)
            continue;
        float own[4], u[12];
#pragma unroll
        for (int j = 0; j < 4; j++)
            own[j] = pw[j][4];
        fused_row_taps(own, u);
        if (!own_x)
            continue;
        const int64_t o = (int64_t)(z + PAD) * pitch + col;
        float ax[4], az[4], nx[4], nzv[4];
        f4a(uld4(f.ax_in + so + o), ax);
        f4a(uld4(f.az_in + so + o), az);
        const float dmz = __ldg(p.dampz + z + PAD);
        const bool zin = z >= 4 && z < p.Z - 4;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            float dx, dz;
            dstag_n<1>(u + j + 1, &dx);
            dstag_n<1>(pw[j] + 1, &dz);
            a_update(p, false, dmx[j], dmz, dx, dz, ax[j], az[j], zin && x + j >= 4 && x + j < p.X - 4, nx[j],
                     nzv[j]);
        }
        ust4(f.ax_out + so + o, nx);
        ust4(f.az_out + so + o, nzv);
    }
}

// Reverse step: grid (nxb, ceil(Z / chunk), n_shots), two warps per CTA
// (warp 0 reconstruction, warp 1 adjoint + imaging condition).
template <int MINB>
__global__ void __launch_bounds__(2 * kFLanes, MINB) k_fused_rev(const __grid_constant__ FusedParams F)
{
    pdl_enter();
    __shared__ float lapbuf[2][kFCols];
    const StepParams &p = F.p;
    const int lane = threadIdx.x & 31, set = threadIdx.x >> 5, shot = blockIdx.z;
    const bool revert = set == 0;
    const int x = (int)blockIdx.x * kFInner - 4 + 4 * lane;
    const bool active = x < p.X;
    const bool own_x = active && lane >= 1 && lane <= 30;
    const int z0 = blockIdx.y * F.chunk, z1 = min(p.Z, z0 + F.chunk);
    const int64_t so = p.shot_stride * shot, col = x + PAD, pitch = p.pitch;
    const Fields &f = revert ? p.f0 : p.f1;
    const float *q = revert ? p.q0 : p.q1;
    float w[4][8], pw[4][9], dmx[4];
    bool xin[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
#pragma unroll
        for (int k = 0; k < 9; k++)
            pw[j][k] = 0.f;
        dmx[j] = 1.f;
        xin[j] = x + j >= 4 && x + j < p.X - 4;
    }
    if (active) {
        f4a(uld4(p.dampx + col), dmx);
#pragma unroll
        for (int k = 0; k < 7; k++) {
            const float4 v = uld4(f.az_in + so + (int64_t)(z0 - 8 + k + PAD) * pitch + col);
            w[0][k] = v.x;
            w[1][k] = v.y;
            w[2][k] = v.z;
            w[3][k] = v.w;
        }
    }
    for (int r = z0 - 4; r < z1 + 4; r++) {
        float pn[4] = {0.f, 0.f, 0.f, 0.f}, qn[4] = {0.f, 0.f, 0.f, 0.f};
        if (active) {
            const float4 v = uld4(f.az_in + so + (int64_t)(r + 3 + PAD) * pitch + col);
            w[0][7] = v.x;
            w[1][7] = v.y;
            w[2][7] = v.z;
            w[3][7] = v.w;
            bool strip[4], damp;
            fused_p_row(p, f, q, so, revert, x, r, w, pn, qn, strip, damp);
            if (r >= 0 && r < p.Z) {
                const int64_t o = (int64_t)(r + PAD) * pitch + col;
                if (revert) {
                    // setRec: P_rec(t) = ring(T-1-t) on ring cells
                    const int4 km = *reinterpret_cast<const int4 *>(F.ringmap + o);
                    const int kk[4] = {km.x, km.y, km.z, km.w};
                    const float *ring = p.ring + ((int64_t)shot * p.T + (p.T - 1 - p.t)) * p.n_ring;
#pragma unroll
                    for (int j = 0; j < 4; j++)
                        if (kk[j] >= 0)
                            pn[j] = ring[kk[j]];
                } else {
                    fused_inject(p, F.rcv_rp, F.rcv_cx, F.rcv_ce, F.rcv_id, false, shot, r, x, pn, qn, strip);
                }
                if (own_x && r >= z0 && r < z1) {
                    ust4(f.px_out + so + o, pn);
                    if (damp)
                        ust4(f.pz_out + so + o, qn);
                }
            }
#pragma unroll
            for (int j = 0; j < 4; j++)
#pragma unroll
                for (int k = 0; k < 7; k++)
                    w[j][k] = w[j][k + 1];
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
#pragma unroll
            for (int k = 0; k < 8; k++)
                pw[j][k] = pw[j][k + 1];
            pw[j][8] = pn[j];
        }
        const int z = r - 4;
        if (z < z0)
            continue;
        // A half-step of row z (pw rows z-4 .. z+4); x taps by shuffles
        float own[4], u[12];
#pragma unroll
        for (int j = 0; j < 4; j++)
            own[j] = pw[j][4];
        fused_row_taps(own, u);
        const int64_t o = (int64_t)(z + PAD) * pitch + col;
        const bool zin = z >= 4 && z < p.Z - 4;
        float *lb = lapbuf[z & 1];
        if (own_x) {
            float ax[4], az[4], nx[4], nzv[4];
            f4a(uld4(f.ax_in + so + o), ax);
            f4a(uld4(f.az_in + so + o), az);
            const float dmz = revert ? 1.f : __ldg(p.dampz + z + PAD);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                float dx, dz;
                dstag_n<1>(u + j + 1, &dx);
                dstag_n<1>(pw[j] + 1, &dz);
                if (revert) {
                    float lx, lz;
                    lap_n<1>(u + j, &lx);
                    lap_n<1>(pw[j], &lz);
                    lb[4 * lane + j] = lap_combine(lx, lz);
                    a_update(p, true, 1.f, 1.f, dx, dz, ax[j], az[j], xin[j] && zin, nx[j], nzv[j]);
                } else {
                    a_update(p, false, dmx[j], dmz, dx, dz, ax[j], az[j], xin[j] && zin, nx[j], nzv[j]);
                }
            }
            ust4(f.ax_out + so + o, nx);
            ust4(f.az_out + so + o, nzv);
        }
        // the Laplacian of P_rec(t) row z from warp 0 to warp 1
        asm volatile("bar.sync 1, 64;" ::: "memory");
        if (!revert && own_x) {
            float g[4];
            f4a(uld4c(p.grad + so + o), g);
#pragma unroll
            for (int j = 0; j < 4; j++)
                g[j] = __fmaf_rn(u[4 + j], lb[4 * lane + j], g[j]);
            ust4(p.grad + so + o, g);
        }
    }
}

}  // namespace otf
