// Exact discrete adjoint step of the split-field PML scheme (FP32).
//
// Forward step t (regression_PML_single.cu:503-519, 587-602), M = update
// mask, a = 1 - d*dt, q = c^2 dt/dx, r = dt/dx:
//   Px_t = M (ax Px_{t-1} + q Dx- Ax_{t-1}) + src,   Pz_t likewise along z
//   rec_t = (Px_t + Pz_t)[receivers]
//   Ax_t = M (ax Ax_{t-1} + r Dx+ (Px_t + Pz_t)),    Az_t likewise
// Its transpose, with the staggered identities Dx+^T = -Dx-, Dx-^T = -Dx+
// (the weights are antisymmetric about the half cell), maps the adjoint
// state (Lx, Lz, Mx, Mz) of step t to that of step t-1:
//   S    = -r (Dx- Mx + Dz- Mz) + g_t at the receivers        (over the halo region)
//   LxT  = M (Lx + S),  LzT = M (Lz + S)
//   Mx'  = M (ax Mx - Dx+ (q LxT)),  Mz' = M (az Mz - Dz+ (q LzT))
//   Lx'  = ax LxT,  Lz' = az LzT
//   dL/dq += LxT Dx- Ax_{t-1} + LzT Dz- Az_{t-1}
// This is the gradient of the discrete forward map itself (checked against
// finite differences of the FP64 oracle), unlike the reference's
// cross-correlation of a reconstructed field (regression_PML_single.cu:
// 793-834), which is an approximation of it.
//
// One tile per CTA, 4 x BH register blocks, FP32 pair-form stencils.
#pragma once
#include "pml_step_split.cuh"

namespace otf {

struct AdjParams {
    int X, Z, pitch, rows, T, ntx, n_rec, t;
    int64_t shot_stride;
    float r;
    const float *q;                 // padded (c^2*dt)/dx
    const float *dampx, *dampz;     // separable 1 - d*dt (padded index)
    const float *lx_in, *lz_in, *mx_in, *mz_in;  // adjoint state at t
    float *lx_out, *lz_out, *mx_out, *mz_out;    // adjoint state at t-1
    const float *ax_prev, *az_prev;              // forward A(t-1)
    const float *g;                  // [n_shots][n_rec][T] dL/drec
    const int *rcve_ptr, *rcve_cell, *rcve_id;   // receivers in each tile's region (interior only)
    float *grad_q;                   // padded [n_shots][rows][pitch], accumulated
};

template <int TX, int TZ, int BH>
struct AdjGeom {
    static constexpr int EX = TX + 8, EZ = TZ + 8;
    static constexpr int AXW = TX + 16, AXH = TZ + 8, AZW = TX + 8, AZH = TZ + 16;
    static constexpr int NAX = AXW * AXH, NAZ = AZW * AZH, NE = EX * EZ;
    // smem: Mx tile | Mz tile | q*LxT (E) | q*LzT (E) | LxT (E) | LzT (E) | Ax(t-1) (E) | Az(t-1) (E)
    static constexpr int SMX = 0, SMZ = NAX, SQX = SMZ + NAZ, SQZ = SQX + NE, SLX = SQZ + NE,
                         SLZ = SLX + NE, SAX = SLZ + NE, SAZ = SAX + NE, FLOATS = SAZ + NE;
    static constexpr int NBEX = EX / 4, NBE = NBEX * (EZ / BH);
    static constexpr int NBOX = TX / 4, NBO = NBOX * (TZ / BH);
};

template <int TX, int TZ, int BH>
__global__ void __launch_bounds__(NT) k_adjoint_step(const AdjParams p)
{
    using G = AdjGeom<TX, TZ, BH>;
    extern __shared__ float4 sm4[];
    float *sm = reinterpret_cast<float *>(sm4);
    float *sMx = sm + G::SMX, *sMz = sm + G::SMZ, *sQx = sm + G::SQX, *sQz = sm + G::SQZ;
    float *sLx = sm + G::SLX, *sLz = sm + G::SLZ, *sAx = sm + G::SAX, *sAz = sm + G::SAZ;
    const int tile = blockIdx.x, shot = blockIdx.y;
    const int x0 = (tile % p.ntx) * TX, z0 = (tile / p.ntx) * TZ;
    const int64_t so = p.shot_stride * shot;
    auto inside = [&](int x, int z) { return x >= 4 && z >= 4 && x < p.X - 4 && z < p.Z - 4; };
    auto ldf4 = [&](const float *base, int prow, int pcol) {
        if (prow < p.rows && pcol < p.pitch)
            return __ldg(reinterpret_cast<const float4 *>(base + so + (int64_t)prow * p.pitch + pcol));
        return make_float4(0.f, 0.f, 0.f, 0.f);
    };
    // stage Mx (x halo 8, z halo 4), Mz (x halo 4, z halo 8), forward A(t-1) over E
    for (int i = threadIdx.x; i < G::NAX / 4; i += NT) {
        const int rr = i / (G::AXW / 4), cc = i - rr * (G::AXW / 4);
        reinterpret_cast<float4 *>(sMx)[i] = ldf4(p.mx_in, z0 - 4 + PAD + rr, x0 - 8 + PAD + 4 * cc);
    }
    for (int i = threadIdx.x; i < G::NAZ / 4; i += NT) {
        const int rr = i / (G::AZW / 4), cc = i - rr * (G::AZW / 4);
        reinterpret_cast<float4 *>(sMz)[i] = ldf4(p.mz_in, z0 - 8 + PAD + rr, x0 - 4 + PAD + 4 * cc);
    }
    for (int i = threadIdx.x; i < G::NE / 4; i += NT) {
        const int rr = i / (G::EX / 4), cc = i - rr * (G::EX / 4);
        reinterpret_cast<float4 *>(sAx)[i] = ldf4(p.ax_prev, z0 - 4 + PAD + rr, x0 - 4 + PAD + 4 * cc);
        reinterpret_cast<float4 *>(sAz)[i] = ldf4(p.az_prev, z0 - 4 + PAD + rr, x0 - 4 + PAD + 4 * cc);
    }
    __syncthreads();
    // S and the adjoints of P(t) after the receiver term, over E
    for (int b = threadIdx.x; b < G::NBE; b += NT) {
        const int ex = 4 * (b % G::NBEX), ez = BH * (b / G::NBEX);
        float dmx[BH][4], dmz[BH][4];
#pragma unroll
        for (int i = 0; i < BH; i++) {
            float w[12];
            const int r = (ez + i) * G::AXW + ex;
            f4a(lds4(sMx, r), w);
            f4a(lds4(sMx, r + 4), w + 4);
            f4a(lds4(sMx, r + 8), w + 8);
            dstag_n<4>(w, dmx[i]);
        }
        {
            float wz[4][BH + 7];
#pragma unroll
            for (int k = 0; k < BH + 7; k++) {
                const float4 v = lds4(sMz, (ez + k) * G::AZW + ex);
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
                    dmz[i][j] = o[i];
            }
        }
        float s[BH][4];
#pragma unroll
        for (int i = 0; i < BH; i++)
#pragma unroll
            for (int j = 0; j < 4; j++)
                s[i][j] = -p.r * (dmx[i][j] + dmz[i][j]);
        for (int e = p.rcve_ptr[tile]; e < p.rcve_ptr[tile + 1]; e++) {
            const int c = p.rcve_cell[e];
            const int cz = c / G::EX - ez, cx = c - (c / G::EX) * G::EX - ex;
            if (cx < 0 || cx >= 4 || cz < 0 || cz >= BH)
                continue;
            const float gv = p.g[((int64_t)shot * p.n_rec + p.rcve_id[e]) * p.T + p.t];
#pragma unroll
            for (int i = 0; i < BH; i++)
#pragma unroll
                for (int j = 0; j < 4; j++)
                    if (i == cz && j == cx)
                        s[i][j] += gv;
        }
#pragma unroll
        for (int i = 0; i < BH; i++) {
            const int zg = z0 - 4 + ez + i;
            float lx[4], lz[4], qv[4];
            const float4 a = ldf4(p.lx_in, zg + PAD, x0 - 4 + ex + PAD);
            const float4 bq = ldf4(p.lz_in, zg + PAD, x0 - 4 + ex + PAD);
            float4 qq = make_float4(0.f, 0.f, 0.f, 0.f);
            if (zg + PAD < p.rows && x0 - 4 + ex + PAD < p.pitch)
                qq = __ldg(reinterpret_cast<const float4 *>(p.q + (int64_t)(zg + PAD) * p.pitch + x0 - 4 + ex + PAD));
            f4a(a, lx);
            f4a(bq, lz);
            f4a(qq, qv);
            float tx[4], tz[4], ux[4], uz[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const bool in = inside(x0 - 4 + ex + j, zg);
                tx[j] = in ? lx[j] + s[i][j] : 0.f;
                tz[j] = in ? lz[j] + s[i][j] : 0.f;
                ux[j] = qv[j] * tx[j];
                uz[j] = qv[j] * tz[j];
            }
            const int o = (ez + i) * G::EX + ex;
            *reinterpret_cast<float4 *>(sLx + o) = make_float4(tx[0], tx[1], tx[2], tx[3]);
            *reinterpret_cast<float4 *>(sLz + o) = make_float4(tz[0], tz[1], tz[2], tz[3]);
            *reinterpret_cast<float4 *>(sQx + o) = make_float4(ux[0], ux[1], ux[2], ux[3]);
            *reinterpret_cast<float4 *>(sQz + o) = make_float4(uz[0], uz[1], uz[2], uz[3]);
        }
    }
    __syncthreads();
    // owned cells: new adjoint state and the gradient
    for (int b = threadIdx.x; b < G::NBO; b += NT) {
        const int ox = 4 * (b % G::NBOX), oz = BH * (b / G::NBOX);
        const int xg = x0 + ox, pcol = xg + PAD;
        float dqx[BH][4], dqz[BH][4], dax[BH][4], daz[BH][4];
#pragma unroll
        for (int i = 0; i < BH; i++) {
            float w[12], u[12];
            const int r = (oz + 4 + i) * G::EX + ox;
            f4a(lds4(sQx, r), w);
            f4a(lds4(sQx, r + 4), w + 4);
            f4a(lds4(sQx, r + 8), w + 8);
            dstag_n<4>(w + 1, dqx[i]);  // D+ at E cols ox+4.. (taps ox+1 ..)
            f4a(lds4(sAx, r), u);
            f4a(lds4(sAx, r + 4), u + 4);
            f4a(lds4(sAx, r + 8), u + 8);
            dstag_n<4>(u, dax[i]);      // D- at E cols ox+4.. (taps ox ..)
        }
        {
            float vq[4][BH + 8], va[4][BH + 8];
#pragma unroll
            for (int c = 0; c < BH + 8; c++) {
                const float4 a = lds4(sQz, (oz + c) * G::EX + ox + 4);
                const float4 bq = lds4(sAz, (oz + c) * G::EX + ox + 4);
                vq[0][c] = a.x; vq[1][c] = a.y; vq[2][c] = a.z; vq[3][c] = a.w;
                va[0][c] = bq.x; va[1][c] = bq.y; va[2][c] = bq.z; va[3][c] = bq.w;
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                float o1[BH], o2[BH];
                dstag_n<BH>(vq[j] + 1, o1);
                dstag_n<BH>(va[j], o2);
#pragma unroll
                for (int i = 0; i < BH; i++) {
                    dqz[i][j] = o1[i];
                    daz[i][j] = o2[i];
                }
            }
        }
        float dm[4] = {1.f, 1.f, 1.f, 1.f};
        if (pcol < p.pitch)
            f4a(__ldg(reinterpret_cast<const float4 *>(p.dampx + pcol)), dm);
#pragma unroll
        for (int i = 0; i < BH; i++) {
            const int zg = z0 + oz + i, prow = zg + PAD;
            if (prow >= p.rows || pcol >= p.pitch)
                continue;
            const float dz = __ldg(p.dampz + prow);
            const int e = (oz + 4 + i) * G::EX + ox + 4;
            float lx[4], lz[4], mx[4], mz[4];
            f4a(lds4(sLx, e), lx);
            f4a(lds4(sLz, e), lz);
            f4a(lds4(sMx, (oz + 4 + i) * G::AXW + ox + 8), mx);
            f4a(lds4(sMz, (oz + 8 + i) * G::AZW + ox + 4), mz);
            const int64_t o = so + (int64_t)prow * p.pitch + pcol;
            float4 g = *reinterpret_cast<const float4 *>(p.grad_q + o);
            float nlx[4], nlz[4], nmx[4], nmz[4], gg[4] = {g.x, g.y, g.z, g.w};
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const bool in = inside(xg + j, zg);
                nlx[j] = dm[j] * lx[j];
                nlz[j] = dz * lz[j];
                nmx[j] = in ? dm[j] * mx[j] - dqx[i][j] : 0.f;
                nmz[j] = in ? dz * mz[j] - dqz[i][j] : 0.f;
                gg[j] += lx[j] * dax[i][j] + lz[j] * daz[i][j];
            }
            *reinterpret_cast<float4 *>(p.lx_out + o) = make_float4(nlx[0], nlx[1], nlx[2], nlx[3]);
            *reinterpret_cast<float4 *>(p.lz_out + o) = make_float4(nlz[0], nlz[1], nlz[2], nlz[3]);
            *reinterpret_cast<float4 *>(p.mx_out + o) = make_float4(nmx[0], nmx[1], nmx[2], nmx[3]);
            *reinterpret_cast<float4 *>(p.mz_out + o) = make_float4(nmz[0], nmz[1], nmz[2], nmz[3]);
            *reinterpret_cast<float4 *>(p.grad_q + o) = make_float4(gg[0], gg[1], gg[2], gg[3]);
        }
    }
}

}  // namespace otf
