// Kernels of the learned gradient preconditioner: a U-Net over NHWC BF16
// activations with FP32 accumulation, trained on the GPU by these kernels.
// No reference counterpart (the reference's inversion is plain L-BFGS-B,
// regression.py:82-88).
//
// Layout: activations and activation gradients [N][H][W][C] BF16 with C a
// multiple of 16; conv weights [9][Cout][Cin] BF16 (tap = 3*dy + dx, Cin
// contiguous) for the forward pass and their flipped transpose
// [9][Cin][Cout] for the input gradient; FP32 master weights, gradients and
// Adam moments.
//
// 3x3 convolutions (zero padding) are implicit GEMMs on the tensor cores
// (mma.m16n8k16 BF16 -> FP32): M = pixels (a 16 x 8 tile per CTA), N = 32
// output channels, K = 9 taps x 16-channel chunks, the input halo tile and
// the weight slice of each chunk double-buffered in shared memory by cp.async.
// The input may be the concatenation of two tensors, the second one at half
// resolution and upsampled (nearest) on load; the output may be split by
// channel into two tensors, each optionally multiplied by a ReLU mask (the
// gradient of a ReLU output), so the decoder's concat/upsample and the ReLU
// backward cost no extra pass.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <cudaTypedefs.h>
#include "otf_common.cuh"
#include "tma.cuh"

namespace otf {
namespace unet {

using bf16 = __nv_bfloat16;
using bf162 = __nv_bfloat162;

constexpr int TW = 16, TH = 8;         // output pixels per CTA (x, y)
constexpr int BN = 32;                 // output channels per CTA
constexpr int KC = 16;                 // input channels per K chunk
constexpr int HWD = TW + 2, HHT = TH + 2;
constexpr int PS = 12;                 // words per staged pixel / weight row (16 BF16 + 8 pad: no bank conflicts)
constexpr int HALO_WORDS = HHT * HWD * PS;
constexpr int WS_WORDS = 9 * BN * PS;
constexpr int STAGE_WORDS = HALO_WORDS + WS_WORDS;

struct ConvArgs {
    const bf16 *src0, *src1;  // input channels [0, c0) from src0, [c0, c0+c1) from src1
    int c0, c1, up1;          // up1: src1 has half the resolution (nearest upsampling)
    const bf16 *w;            // [9][cout][c0+c1]
    const bf16 *wp;           // tcgen05 kernels: the same weights packed [(c0+c1)/8][9][cout][8]
    const float *bias;        // [cout] or null
    int relu;
    bf16 *dst0, *dst1;        // channels [0, split) -> dst0, [split, cout) -> dst1
    const bf16 *mask0, *mask1;
    int split, cout;
    int N, H, W;
};

__device__ __forceinline__ void cp_async16(uint32_t *dst, const void *src, int bytes)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(bytes));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void mma16816(float *c, const uint32_t *a, uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack2(bf16 lo, bf16 hi)
{
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// Address of the 8 channels [ch, ch+8) of input pixel (gy, gx) of image n.
__device__ __forceinline__ const bf16 *in_ptr(const ConvArgs &a, int n, int gy, int gx, int ch)
{
    if (ch < a.c0)
        return a.src0 + (((int64_t)n * a.H + gy) * a.W + gx) * a.c0 + ch;
    if (a.up1)
        return a.src1 + (((int64_t)n * (a.H >> 1) + (gy >> 1)) * (a.W >> 1) + (gx >> 1)) * a.c1 + (ch - a.c0);
    return a.src1 + (((int64_t)n * a.H + gy) * a.W + gx) * a.c1 + (ch - a.c0);
}

__device__ __forceinline__ void load_stage(const ConvArgs &a, uint32_t *st, int kc, int n, int y0, int x0,
                                           int co0, int cin)
{
    for (int i = threadIdx.x; i < HHT * HWD * 2; i += blockDim.x) {
        const int px = i >> 1, half = i & 1;
        const int hy = px / HWD, hx = px - hy * HWD;
        const int gy = y0 + hy - 1, gx = x0 + hx - 1;
        const bool ok = gy >= 0 && gy < a.H && gx >= 0 && gx < a.W;
        const void *src = ok ? (const void *)in_ptr(a, n, gy, gx, kc * KC + half * 8) : (const void *)a.w;
        cp_async16(st + px * PS + half * 4, src, ok ? 16 : 0);
    }
    uint32_t *ws = st + HALO_WORDS;
    for (int i = threadIdx.x; i < 9 * BN * 2; i += blockDim.x) {
        const int row = i >> 1, half = i & 1;
        const int tap = row / BN, co = row - tap * BN;
        cp_async16(ws + row * PS + half * 4, a.w + (int64_t)(tap * a.cout + co0 + co) * cin + kc * KC + half * 8,
                   16);
    }
}

// One CTA: 16 x 8 output pixels of one image x 32 output channels; 4 warps,
// warp w owns tile rows 2w and 2w+1 (one m16 tile each) x 4 n8 tiles.
__global__ void __launch_bounds__(128) k_conv3x3(ConvArgs a)
{
    __shared__ __align__(16) uint32_t sm[2 * STAGE_WORDS];
    const int tiles_x = (a.W + TW - 1) / TW, tiles_y = (a.H + TH - 1) / TH;
    int b = blockIdx.x;
    const int n = b / (tiles_x * tiles_y);
    b -= n * tiles_x * tiles_y;
    const int ty = b / tiles_x, tx = b - ty * tiles_x;
    const int y0 = ty * TH, x0 = tx * TW, co0 = blockIdx.y * BN;
    const int cin = a.c0 + a.c1, nk = cin / KC;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;

    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int k = 0; k < 4; k++)
                acc[i][j][k] = 0.f;

    load_stage(a, sm, 0, n, y0, x0, co0, cin);
    cp_commit();
    for (int kc = 0; kc < nk; kc++) {
        if (kc + 1 < nk)
            load_stage(a, sm + ((kc + 1) & 1) * STAGE_WORDS, kc + 1, n, y0, x0, co0, cin);
        cp_commit();
        cp_wait<1>();
        __syncthreads();
        const uint32_t *hs = sm + (kc & 1) * STAGE_WORDS, *ws = hs + HALO_WORDS;
#pragma unroll
        for (int tap = 0; tap < 9; tap++) {
            const int dy = tap / 3, dx = tap - 3 * (tap / 3);
            uint32_t af[2][4];
#pragma unroll
            for (int i = 0; i < 2; i++) {
                const uint32_t *p0 = hs + ((warp * 2 + i + dy) * HWD + g + dx) * PS + t;
                const uint32_t *p1 = p0 + 8 * PS;
                af[i][0] = p0[0];
                af[i][1] = p1[0];
                af[i][2] = p0[4];
                af[i][3] = p1[4];
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const uint32_t *q = ws + (tap * BN + j * 8 + g) * PS + t;
                const uint32_t b0 = q[0], b1 = q[4];
#pragma unroll
                for (int i = 0; i < 2; i++)
                    mma16816(acc[i][j], af[i], b0, b1);
            }
        }
        __syncthreads();
    }

#pragma unroll
    for (int i = 0; i < 2; i++) {
        const int y = y0 + warp * 2 + i;
        if (y >= a.H)
            continue;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int x = x0 + g + h * 8;
            if (x >= a.W)
                continue;
            const int64_t pix = ((int64_t)n * a.H + y) * a.W + x;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int co = co0 + j * 8 + 2 * t;
                float v0 = acc[i][j][2 * h], v1 = acc[i][j][2 * h + 1];
                if (a.bias) {
                    v0 += a.bias[co];
                    v1 += a.bias[co + 1];
                }
                if (a.relu) {
                    v0 = fmaxf(v0, 0.f);
                    v1 = fmaxf(v1, 0.f);
                }
                const bool lo = co < a.split;
                bf16 *dst = lo ? a.dst0 : a.dst1;
                const bf16 *mask = lo ? a.mask0 : a.mask1;
                const int cc = lo ? a.split : a.cout - a.split, ci = lo ? co : co - a.split;
                if (mask) {
                    const bf162 m = *reinterpret_cast<const bf162 *>(mask + pix * cc + ci);
                    if (!(__low2float(m) > 0.f))
                        v0 = 0.f;
                    if (!(__high2float(m) > 0.f))
                        v1 = 0.f;
                }
                *reinterpret_cast<bf162 *>(dst + pix * cc + ci) = __floats2bfloat162_rn(v0, v1);
            }
        }
    }
}

// ---- weight gradient: dw[tap][co][ci] += sum_p dz[p][co] * x[p + tap][ci]
struct WgradArgs {
    const bf16 *src0, *src1;
    int c0, c1, up1;     // the forward input, as in ConvArgs
    const bf16 *dz;      // [N][H][W][cout] gradient of the pre-activation
    int cout;
    float *dw;           // [9][cout][cin] FP32, accumulated
    int N, H, W;
};

#include "unet_umma.cuh"

constexpr int WG_DZ_LD = TW * TH + 8;   // 136 BF16 per output channel row
constexpr int WG_X_LD = HHT * HWD + 4;  // 184 BF16 per input channel row

// One CTA: 32 output channels x 16 input channels x all 9 taps, looping over
// 16 x 8 pixel slabs (slab = blockIdx.x, += gridDim.x); tiles are staged
// transposed (channel-major) so that K = pixels is contiguous. Warp w owns
// the m16 tile (w >> 1) and the n8 tile (w & 1) for every tap.
__global__ void __launch_bounds__(128) k_conv3x3_wgrad(WgradArgs a)
{
    __shared__ __align__(16) bf16 dzs[BN * WG_DZ_LD];
    __shared__ __align__(16) bf16 xs[KC * WG_X_LD];
    const int co0 = blockIdx.y * BN, ci0 = blockIdx.z * KC;
    const int cin = a.c0 + a.c1;
    const int tiles_x = (a.W + TW - 1) / TW, tiles_y = (a.H + TH - 1) / TH;
    const int n_slabs = tiles_x * tiles_y * a.N;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int mb = (warp >> 1) * 16, nb = (warp & 1) * 8;
    ConvArgs ca{};
    ca.src0 = a.src0;
    ca.src1 = a.src1;
    ca.c0 = a.c0;
    ca.c1 = a.c1;
    ca.up1 = a.up1;
    ca.N = a.N;
    ca.H = a.H;
    ca.W = a.W;

    float acc[9][4];
#pragma unroll
    for (int k = 0; k < 9; k++)
        acc[k][0] = acc[k][1] = acc[k][2] = acc[k][3] = 0.f;

    for (int s = blockIdx.x; s < n_slabs; s += gridDim.x) {
        int b = s;
        const int n = b / (tiles_x * tiles_y);
        b -= n * tiles_x * tiles_y;
        const int ty = b / tiles_x, tx = b - ty * tiles_x;
        const int y0 = ty * TH, x0 = tx * TW;
        __syncthreads();  // previous slab consumed
        // dz tile: 128 pixels x 32 channels, 8 channels per load
        for (int i = threadIdx.x; i < TW * TH * (BN / 8); i += blockDim.x) {
            const int px = i / (BN / 8), q = i - px * (BN / 8);
            const int y = y0 + px / TW, x = x0 + (px % TW);
            uint4 v = make_uint4(0, 0, 0, 0);
            if (y < a.H && x < a.W)
                v = *reinterpret_cast<const uint4 *>(a.dz + (((int64_t)n * a.H + y) * a.W + x) * a.cout + co0 + q * 8);
            const bf16 *e = reinterpret_cast<const bf16 *>(&v);
#pragma unroll
            for (int k = 0; k < 8; k++)
                dzs[(q * 8 + k) * WG_DZ_LD + px] = e[k];
        }
        // input halo: 10 x 18 pixels x 16 channels
        for (int i = threadIdx.x; i < HHT * HWD * 2; i += blockDim.x) {
            const int px = i >> 1, half = i & 1;
            const int hy = px / HWD, hx = px - hy * HWD;
            const int gy = y0 + hy - 1, gx = x0 + hx - 1;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gy >= 0 && gy < a.H && gx >= 0 && gx < a.W)
                v = *reinterpret_cast<const uint4 *>(in_ptr(ca, n, gy, gx, ci0 + half * 8));
            const bf16 *e = reinterpret_cast<const bf16 *>(&v);
#pragma unroll
            for (int k = 0; k < 8; k++)
                xs[(half * 8 + k) * WG_X_LD + px] = e[k];
        }
        __syncthreads();
#pragma unroll 1
        for (int r = 0; r < TH; r++) {  // K step = one row of 16 pixels
            uint32_t af[4];
            const bf16 *d0 = dzs + (mb + g) * WG_DZ_LD + r * TW + 2 * t;
            const bf16 *d1 = d0 + 8 * WG_DZ_LD;
            af[0] = *reinterpret_cast<const uint32_t *>(d0);
            af[1] = *reinterpret_cast<const uint32_t *>(d1);
            af[2] = *reinterpret_cast<const uint32_t *>(d0 + 8);
            af[3] = *reinterpret_cast<const uint32_t *>(d1 + 8);
#pragma unroll
            for (int tap = 0; tap < 9; tap++) {
                const int dy = tap / 3, dx = tap - 3 * (tap / 3);
                const bf16 *xr = xs + (nb + g) * WG_X_LD + (r + dy) * HWD + dx + 2 * t;
                const uint32_t b0 = pack2(xr[0], xr[1]), b1 = pack2(xr[8], xr[9]);
                mma16816(acc[tap], af, b0, b1);
            }
        }
    }
#pragma unroll
    for (int tap = 0; tap < 9; tap++) {
        float *d = a.dw + ((int64_t)tap * a.cout + co0 + mb + g) * cin + ci0 + nb + 2 * t;
        atomicAdd(d, acc[tap][0]);
        atomicAdd(d + 1, acc[tap][1]);
        atomicAdd(d + 8 * (int64_t)cin, acc[tap][2]);
        atomicAdd(d + 8 * (int64_t)cin + 1, acc[tap][3]);
    }
}

// db[c] += sum over pixels of dz[p][c]; C divides 256.
__global__ void k_bias_grad(const bf16 *__restrict__ dz, int C, int64_t npix, float *__restrict__ db)
{
    const int per = 256 / C;
    const int c = threadIdx.x % C;
    float s = 0.f;
    for (int64_t p = (int64_t)blockIdx.x * per + threadIdx.x / C; p < npix; p += (int64_t)gridDim.x * per)
        s += __bfloat162float(dz[p * C + c]);
    atomicAdd(db + c, s);
}

// 2x2 average pooling, 8 channels per thread.
__global__ void k_pool2(const bf16 *__restrict__ x, bf16 *__restrict__ y, int N, int H, int W, int C)
{
    const int C8 = C / 8, Ho = H / 2, Wo = W / 2;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, tot = (int64_t)N * Ho * Wo * C8;
    if (i >= tot)
        return;
    const int q = (int)(i % C8);
    int64_t p = i / C8;
    const int xo = (int)(p % Wo);
    p /= Wo;
    const int yo = (int)(p % Ho);
    const int n = (int)(p / Ho);
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int d = 0; d < 4; d++) {
        const uint4 v = *reinterpret_cast<const uint4 *>(
            x + (((int64_t)n * H + 2 * yo + (d >> 1)) * W + 2 * xo + (d & 1)) * C + q * 8);
        const bf16 *e = reinterpret_cast<const bf16 *>(&v);
#pragma unroll
        for (int k = 0; k < 8; k++)
            acc[k] += __bfloat162float(e[k]);
    }
    uint4 o;
    bf16 *oe = reinterpret_cast<bf16 *>(&o);
#pragma unroll
    for (int k = 0; k < 8; k++)
        oe[k] = __float2bfloat16_rn(0.25f * acc[k]);
    *reinterpret_cast<uint4 *>(y + (((int64_t)n * Ho + yo) * Wo + xo) * C + q * 8) = o;
}

// Pooling backward into an existing gradient: dx += 0.25 * dy(parent) * (x > 0).
__global__ void k_pool2_bwd(const bf16 *__restrict__ dy, const bf16 *__restrict__ x, bf16 *__restrict__ dx,
                            int N, int H, int W, int C)
{
    const int C8 = C / 8;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, tot = (int64_t)N * H * W * C8;
    if (i >= tot)
        return;
    const int q = (int)(i % C8);
    int64_t p = i / C8;
    const int xx = (int)(p % W);
    p /= W;
    const int yy = (int)(p % H);
    const int n = (int)(p / H);
    const int64_t o = (((int64_t)n * H + yy) * W + xx) * C + q * 8;
    const uint4 vx = *reinterpret_cast<const uint4 *>(x + o);
    uint4 vd = *reinterpret_cast<const uint4 *>(dx + o);
    const uint4 vy = *reinterpret_cast<const uint4 *>(
        dy + (((int64_t)n * (H / 2) + yy / 2) * (W / 2) + xx / 2) * C + q * 8);
    const bf16 *ex = reinterpret_cast<const bf16 *>(&vx), *ey = reinterpret_cast<const bf16 *>(&vy);
    bf16 *ed = reinterpret_cast<bf16 *>(&vd);
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const float add = __bfloat162float(ex[k]) > 0.f ? 0.25f * __bfloat162float(ey[k]) : 0.f;
        ed[k] = __float2bfloat16_rn(__bfloat162float(ed[k]) + add);
    }
    *reinterpret_cast<uint4 *>(dx + o) = vd;
}

// Nearest-upsampling backward: dx[q] = (x[q] > 0) * sum of dy over the 4 children.
__global__ void k_up2_bwd(const bf16 *__restrict__ dy, const bf16 *__restrict__ x, bf16 *__restrict__ dx,
                          int N, int Hh, int Wh, int C)
{
    const int C8 = C / 8;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, tot = (int64_t)N * Hh * Wh * C8;
    if (i >= tot)
        return;
    const int q = (int)(i % C8);
    int64_t p = i / C8;
    const int xx = (int)(p % Wh);
    p /= Wh;
    const int yy = (int)(p % Hh);
    const int n = (int)(p / Hh);
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int d = 0; d < 4; d++) {
        const uint4 v = *reinterpret_cast<const uint4 *>(
            dy + (((int64_t)n * 2 * Hh + 2 * yy + (d >> 1)) * 2 * Wh + 2 * xx + (d & 1)) * C + q * 8);
        const bf16 *e = reinterpret_cast<const bf16 *>(&v);
#pragma unroll
        for (int k = 0; k < 8; k++)
            acc[k] += __bfloat162float(e[k]);
    }
    const int64_t o = (((int64_t)n * Hh + yy) * Wh + xx) * C + q * 8;
    const uint4 vx = *reinterpret_cast<const uint4 *>(x + o);
    const bf16 *ex = reinterpret_cast<const bf16 *>(&vx);
    uint4 r;
    bf16 *er = reinterpret_cast<bf16 *>(&r);
#pragma unroll
    for (int k = 0; k < 8; k++)
        er[k] = __float2bfloat16_rn(__bfloat162float(ex[k]) > 0.f ? acc[k] : 0.f);
    *reinterpret_cast<uint4 *>(dx + o) = r;
}

// Network input: FP32 [npix][cin] -> BF16 [npix][16] (channels >= cin zero).
__global__ void k_pack_input(const float *__restrict__ x, int cin, int64_t npix, bf16 *__restrict__ y)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix * 16)
        return;
    const int c = (int)(i % 16);
    const int64_t p = i / 16;
    y[i] = __float2bfloat16_rn(c < cin ? x[p * cin + c] : 0.f);
}

// 1x1 output head: out[p] = b + sum_c x[p][c] * w[c] (FP32 out, C == 32).
__global__ void k_head(const bf16 *__restrict__ x, const float *__restrict__ w, const float *__restrict__ b,
                       int64_t npix, float *__restrict__ out)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix)
        return;
    float s = 0.f;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const uint4 v = *reinterpret_cast<const uint4 *>(x + p * 32 + q * 8);
        const bf16 *e = reinterpret_cast<const bf16 *>(&v);
#pragma unroll
        for (int k = 0; k < 8; k++)
            s = fmaf(__bfloat162float(e[k]), w[q * 8 + k], s);
    }
    out[p] = s + b[0];
}

// Head backward: dx[p][c] = dout[p] * w[c] * (x > 0); dw[c] += sum_p dout[p] x[p][c];
// db += sum_p dout[p]. 256 threads; pixel per thread.
__global__ void __launch_bounds__(256) k_head_bwd(const bf16 *__restrict__ x, const float *__restrict__ w,
                                                  const float *__restrict__ dout, int64_t npix,
                                                  bf16 *__restrict__ dx, float *__restrict__ dw,
                                                  float *__restrict__ db)
{
    __shared__ float red[33][8];
    float pw[32], pb = 0.f;
#pragma unroll
    for (int c = 0; c < 32; c++)
        pw[c] = 0.f;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += (int64_t)gridDim.x * blockDim.x) {
        const float d = dout[p];
        pb += d;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const uint4 v = *reinterpret_cast<const uint4 *>(x + p * 32 + q * 8);
            const bf16 *e = reinterpret_cast<const bf16 *>(&v);
            uint4 o;
            bf16 *oe = reinterpret_cast<bf16 *>(&o);
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const float xv = __bfloat162float(e[k]);
                pw[q * 8 + k] = fmaf(d, xv, pw[q * 8 + k]);
                oe[k] = __float2bfloat16_rn(xv > 0.f ? d * w[q * 8 + k] : 0.f);
            }
            *reinterpret_cast<uint4 *>(dx + p * 32 + q * 8) = o;
        }
    }
    // warp reductions, then one atomic per block and value
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 33; c++) {
        float v = c < 32 ? pw[c] : pb;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0)
            red[c][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 33) {
        float v = 0.f;
        for (int k = 0; k < 8; k++)
            v += red[threadIdx.x][k];
        atomicAdd(threadIdx.x < 32 ? dw + threadIdx.x : db, v);
    }
}

// Weighted squared error: loss += sum w (out - target)^2 / norm;
// dout = 2 w (out - target) / norm. w may be null (1).
__global__ void __launch_bounds__(256) k_mse(const float *__restrict__ out, const float *__restrict__ target,
                                             const float *__restrict__ wt, int64_t n, float inv_norm,
                                             float *__restrict__ dout, float *__restrict__ loss)
{
    __shared__ float red[8];
    float s = 0.f;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float w = wt ? wt[i] : 1.f;
        const float d = out[i] - target[i];
        s += w * d * d;
        dout[i] = 2.f * w * d * inv_norm;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0)
        red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float v = 0.f;
        for (int k = 0; k < 8; k++)
            v += red[k];
        atomicAdd(loss, v * inv_norm);
    }
}

// Adam (bias-corrected) on FP32 master parameters.
__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, int64_t n, float lr, float b1, float b2, float eps, float c1,
                       float c2, float wd)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float gi = g[i] + wd * p[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// BF16 working copies of one conv layer: wf[tap][co][ci] (forward) and
// wb[8 - tap][ci][co] (input gradient).
__global__ void k_pack_weights(const float *__restrict__ w, int cout, int cin, bf16 *__restrict__ wf,
                               bf16 *__restrict__ wb)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, tot = (int64_t)9 * cout * cin;
    if (i >= tot)
        return;
    const int ci = (int)(i % cin);
    const int64_t r = i / cin;
    const int co = (int)(r % cout), tap = (int)(r / cout);
    const bf16 v = __float2bfloat16_rn(w[i]);
    wf[i] = v;
    if (wb)
        wb[((int64_t)(8 - tap) * cin + ci) * cout + co] = v;
}

}  // namespace unet
}  // namespace otf

using namespace otf::unet;

namespace {
int g_use_umma = 1;
// persistent convolution for the layers with <= 128 output channels per CTA
// (OTFWI_CONV_PERSISTENT=0: the one-tile kernel for every layer)
const bool g_conv_pers = [] {
    const char *v = getenv("OTFWI_CONV_PERSISTENT");
    return !(v && v[0] == '0');
}();
bool use_umma() { return g_use_umma != 0; }

// Tiled BF16 tensor map (rank 3 or 4, no swizzle, zero fill outside).
int encode_bf16_map(CUtensorMap *m, const void *base, int rank, const cuuint64_t *dims, const cuuint64_t *strides,
                    const cuuint32_t *box)
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        OTF_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        OTF_CHECK(q == cudaDriverEntryPointSuccess && p, 4, "cuTensorMapEncodeTiled is unavailable");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    const cuuint32_t es[4] = {1, 1, 1, 1};
    const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, (cuuint32_t)rank, const_cast<void *>(base), dims,
                          strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    OTF_CHECK(r == CUDA_SUCCESS, 4, "cuTensorMapEncodeTiled failed with code " + std::to_string((int)r));
    return 0;
}

// The maps of the tcgen05 convolutions: the weights (cin, cout, 9) with box
// (8, nb, 9) when no packed copy is given; the inputs (c, W, H, N) with box
// (8, 10, 34, 1).
int conv_maps(ConvMaps *m, const ConvArgs &a, int nb)
{
    std::memset(m, 0, sizeof(*m));
    if (!a.wp) {
        const int cin = a.c0 + a.c1;
        const cuuint64_t dims[3] = {(cuuint64_t)cin, (cuuint64_t)a.cout, 9};
        const cuuint64_t str[2] = {(cuuint64_t)cin * 2, (cuuint64_t)a.cout * cin * 2};
        const cuuint32_t wbox[3] = {8, (cuuint32_t)nb, 9};
        if (encode_bf16_map(&m->w, a.w, 3, dims, str, wbox))
            return -1;
    }
    const cuuint32_t box[4] = {8, (cuuint32_t)umma::HWU, (cuuint32_t)umma::HH2, 1};
    for (int i = 0; i < 2; i++) {
        const int c = i ? a.c1 : a.c0;
        if (c == 0 || (i == 1 && a.up1))
            continue;
        const cuuint64_t dims[4] = {(cuuint64_t)c, (cuuint64_t)a.W, (cuuint64_t)a.H, (cuuint64_t)a.N};
        const cuuint64_t str[3] = {(cuuint64_t)c * 2, (cuuint64_t)a.W * c * 2, (cuuint64_t)a.H * a.W * c * 2};
        if (encode_bf16_map(i ? &m->x1 : &m->x0, i ? (const void *)a.src1 : (const void *)a.src0, 4, dims, str, box))
            return -1;
    }
    return 0;
}

// Stages of k_conv3x3_umma for nb output channels: as many as fit two CTAs
// per SM (one CTA for 256 channels), at most 4.
int conv_stages(int nb)
{
    if (nb > 128)
        return 2;
    int nst = 4;
    while (nst > 2 && umma_smem_bytes(nb, nst) > 113 * 1024)
        nst--;
    return nst;
}
inline unsigned blocks(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }
int launch_status()
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        otf::set_error((int)e, "unet kernel launch", __FILE__, __LINE__);
        return -1;
    }
    return 0;
}
// Launch of the tcgen05 convolution for channel blocks of nb (the weights
// already packed in a.wp): the persistent kernel for nb <= 128, else the
// one-tile kernel.
int conv_umma_launch(const ConvArgs &a, const ConvMaps &maps, int nb, int nk, int tiles, cudaStream_t st)
{
    const int cout = a.cout;
    static const int sms = [] {
        int dev = 0, n = 148;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            n = 148;
        return n;
    }();
    if (g_conv_pers && nb <= 128 && 288 * nb * nk <= kResWeightBytes) {
        // the small layers: persistent CTAs with the weights resident and
        // double-buffered accumulators (with the weights streamed instead,
        // the persistent form measured slower than one tile per CTA)
        const int smem = umma_res_smem_bytes(nb, nk);
        int ncols = 32;
        while (ncols < 4 * nb)
            ncols <<= 1;
        int cps = (228 * 1024) / (smem + 1024);
        cps = cps < 512 / ncols ? cps : 512 / ncols;
        cps = cps < 1 ? 1 : cps;
        const int ncb = cout / nb;
        int gx = sms * cps / ncb;
        gx = gx < 1 ? 1 : (gx > tiles ? tiles : gx);
        OTF_CUDA(cudaFuncSetAttribute(k_conv3x3_umma_res, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        k_conv3x3_umma_res<<<dim3((unsigned)gx, (unsigned)ncb), 256, smem, st>>>(a, maps, nb, tiles);
        return launch_status();
    }
    const dim3 grid((unsigned)tiles, (unsigned)(cout / nb));
    const int nst = conv_stages(nb);
    const int smem = umma_smem_bytes(nb, nst);
    auto kern = nst == 2 ? k_conv3x3_umma<2> : nst == 3 ? k_conv3x3_umma<3> : k_conv3x3_umma<4>;
    OTF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    kern<<<grid, 128, smem, st>>>(a, maps, nb);
    return launch_status();
}
}  // namespace

extern "C" {

int otf_unet_conv3x3_packed(const void *src0, int c0, const void *src1, int c1, int up1, const void *w,
                            const void *wp, const float *bias, int relu, void *dst0, const void *mask0, void *dst1,
                            const void *mask1, int split, int cout, int N, int H, int W, void *stream)
{
    OTF_CHECK(c0 % 16 == 0 && c1 % 16 == 0 && c0 + c1 > 0 && cout % BN == 0, 1,
              "conv3x3: channel counts must be multiples of 16 (input) and 32 (output)");
    OTF_CHECK(split % 2 == 0 && split >= 0 && split <= cout && (split == cout || dst1), 1,
              "conv3x3: bad output split");
    OTF_CHECK(!up1 || (H % 2 == 0 && W % 2 == 0), 1, "conv3x3: upsampled input needs even H, W");
    OTF_CHECK(c1 == 0 || src1, 1, "conv3x3: second input missing");
    ConvArgs a;
    a.src0 = (const bf16 *)src0;
    a.src1 = (const bf16 *)src1;
    a.c0 = c0;
    a.c1 = c1;
    a.up1 = up1;
    a.w = (const bf16 *)w;
    a.wp = (const bf16 *)wp;
    a.bias = bias;
    a.relu = relu;
    a.dst0 = (bf16 *)dst0;
    a.dst1 = (bf16 *)dst1;
    a.mask0 = (const bf16 *)mask0;
    a.mask1 = (const bf16 *)mask1;
    a.split = split;
    a.cout = cout;
    a.N = N;
    a.H = H;
    a.W = W;
    if (use_umma()) {
        // tensor-core (tcgen05) path: every output channel of a pixel tile in
        // one CTA where cout <= 256, else blocks of 256 / 128 / 64 / 32
        int nb = cout;
        for (int c : {256, 128, 64, 32})
            if (nb > 256 && cout % c == 0)
                nb = c;
        const int tiles = ((W + umma::TWU - 1) / umma::TWU) * ((H + umma::TH2 - 1) / umma::TH2) * N;
        // small images (the bottom of the network): split the output channels
        // further while fewer CTAs than SMs would run
        static const int sms = [] {
            int dev = 0, n = 148;
            if (cudaGetDevice(&dev) != cudaSuccess ||
                cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
                n = 148;
            return n;
        }();
        // (blocks stay multiples of 32 channels: the epilogues read the
        // accumulators 32 columns at a time)
        while (nb > 64 && (int64_t)tiles * (cout / nb) < sms && (nb / 2) % 32 == 0 && cout % (nb / 2) == 0)
            nb /= 2;
        OTF_CHECK(nb % 32 == 0 && cout % nb == 0, 1, "conv3x3: internal channel block not a multiple of 32");
        ConvMaps maps;
        if (conv_maps(&maps, a, nb))
            return -1;
        const int nk = (c0 + c1) / KC;
        return conv_umma_launch(a, maps, nb, nk, tiles, (cudaStream_t)stream);
    }
    const int tiles = ((W + TW - 1) / TW) * ((H + TH - 1) / TH) * N;
    k_conv3x3<<<dim3((unsigned)tiles, (unsigned)(cout / BN)), 128, 0, (cudaStream_t)stream>>>(a);
    return launch_status();
}

int otf_unet_conv3x3(const void *src0, int c0, const void *src1, int c1, int up1, const void *w,
                     const float *bias, int relu, void *dst0, const void *mask0, void *dst1,
                     const void *mask1, int split, int cout, int N, int H, int W, void *stream)
{
    return otf_unet_conv3x3_packed(src0, c0, src1, c1, up1, w, nullptr, bias, relu, dst0, mask0, dst1, mask1,
                                   split, cout, N, H, W, stream);
}

int otf_unet_pack_weights_tc(const void *w, int cout, int cin, void *wp, void *stream)
{
    OTF_CHECK(cin % 16 == 0 && cout > 0, 1, "pack_weights_tc: cin must be a multiple of 16");
    const int64_t units = (int64_t)(cin / 8) * 9 * cout;
    const int nbk = (int)std::min<int64_t>((units + 255) / 256, 4 * 148);
    k_pack_w_umma<<<nbk, 256, 0, (cudaStream_t)stream>>>((const bf16 *)w, (bf16 *)wp, cout, cin);
    return launch_status();
}

/* Tensor-core path of the 3x3 convolution and its weight gradient: 1 =
 * tcgen05 (default; the weight gradients of three small layer shapes keep
 * the mma.sync kernel, which is faster there), 2 = tcgen05 for every shape,
 * 0 = the warp-level mma.sync kernels; returns the previous setting. */
int otf_unet_set_umma(int on)
{
    const int prev = g_use_umma;
    g_use_umma = on < 0 ? 0 : (on > 2 ? 2 : on);
    return prev;
}

/* Error bits recorded by the U-Net tensor-core kernels since the last call
 * (1 = a bounded wait timed out; the results of that launch are invalid);
 * cleared by the call. Returns -1 if the flag cannot be read. */
int otf_unet_status(void)
{
    int h = 0;
    const int zero = 0;
    if (cudaMemcpyFromSymbol(&h, g_unet_err, sizeof(int)) != cudaSuccess ||
        cudaMemcpyToSymbol(g_unet_err, &zero, sizeof(int)) != cudaSuccess) {
        otf::set_error_msg(5, "unet status: flag read failed");
        return -1;
    }
    return h;
}

int otf_unet_conv3x3_wgrad(const void *src0, int c0, const void *src1, int c1, int up1, const void *dz,
                           int cout, float *dw, int N, int H, int W, int sm_count, void *stream)
{
    OTF_CHECK(c0 % 16 == 0 && c1 % 16 == 0 && c0 + c1 > 0 && cout % BN == 0, 1,
              "conv3x3_wgrad: channel counts must be multiples of 16 (input) and 32 (output)");
    WgradArgs a;
    a.src0 = (const bf16 *)src0;
    a.src1 = (const bf16 *)src1;
    a.c0 = c0;
    a.c1 = c1;
    a.up1 = up1;
    a.dz = (const bf16 *)dz;
    a.cout = cout;
    a.dw = dw;
    a.N = N;
    a.H = H;
    a.W = W;
    // The tcgen05 weight gradient computes 128 output-channel rows per CTA
    // (rows beyond cout are zeros) and gathers the upsampled input three times
    // (once per dx window): measured per layer of the 16 x 256^2 network it
    // beats the mma.sync kernel on every layer (1.1-1.6x) but three, which
    // keep the mma.sync kernel: 16 input channels (84 against 100 TFLOP/s),
    // 32 -> 64 channels (104 / 112) and 32 + 64 upsampled -> 32 (79 / 129).
    const int cin_all = c0 + c1;
    const bool tc = cin_all >= 32 && !(cout < 128 && cin_all < 64 && cout > cin_all) && !(up1 && c1 > 0 && cout < 64);
    if (use_umma() && (g_use_umma == 2 || tc)) {
        // tensor-core path: 128 output channels x 32 (or 16) input channels x
        // 9 taps per CTA, the pixels split into slab ranges so that about one
        // CTA per SM runs
        const int cin = c0 + c1;
        const int nw = cin % 32 == 0 ? 32 : 16;
        const int n_slabs = ((W + umma::TWU - 1) / umma::TWU) * ((H + umma::THU - 1) / umma::THU) * N;
        const int gy = (cout + 127) / 128, gz = cin / nw;
        const int target = sm_count > 0 ? sm_count : 148;  // one CTA per SM (140-181 KB of stages)
        int gx = target / (gy * gz);
        gx = gx < 1 ? 1 : (gx > n_slabs ? n_slabs : gx);
        const int spc = (n_slabs + gx - 1) / gx;
        gx = (n_slabs + spc - 1) / spc;
        const dim3 grid((unsigned)gx, (unsigned)gy, (unsigned)gz);
        WgradMaps maps;
        std::memset(&maps, 0, sizeof(maps));
        {
            const cuuint64_t dims[4] = {(cuuint64_t)cout, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)N};
            const cuuint64_t str[3] = {(cuuint64_t)cout * 2, (cuuint64_t)W * cout * 2, (cuuint64_t)H * W * cout * 2};
            const cuuint32_t box[4] = {8, (cuuint32_t)umma::TWU, (cuuint32_t)umma::THU, 1};
            if (encode_bf16_map(&maps.dz, dz, 4, dims, str, box))
                return -1;
        }
        for (int i = 0; i < 2; i++) {
            const int c = i ? c1 : c0;
            if (c == 0 || (i == 1 && up1))
                continue;
            const cuuint64_t dims[4] = {(cuuint64_t)c, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)N};
            const cuuint64_t str[3] = {(cuuint64_t)c * 2, (cuuint64_t)W * c * 2, (cuuint64_t)H * W * c * 2};
            const cuuint32_t box[4] = {8, (cuuint32_t)umma::TWU, (cuuint32_t)umma::THU + 2, 1};
            if (encode_bf16_map(i ? &maps.x1 : &maps.x0, i ? src1 : src0, 4, dims, str, box))
                return -1;
        }
        if (nw == 32) {
            const int smem = umma_wg_smem_bytes(32, 3);
            OTF_CUDA(cudaFuncSetAttribute(k_conv3x3_wgrad_umma<32, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          smem));
            k_conv3x3_wgrad_umma<32, 3><<<grid, 128, smem, (cudaStream_t)stream>>>(a, maps, spc);
        } else {
            const int smem = umma_wg_smem_bytes(16, 3);
            OTF_CUDA(cudaFuncSetAttribute(k_conv3x3_wgrad_umma<16, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          smem));
            k_conv3x3_wgrad_umma<16, 3><<<grid, 128, smem, (cudaStream_t)stream>>>(a, maps, spc);
        }
        return launch_status();
    }
    const int slabs = ((W + TW - 1) / TW) * ((H + TH - 1) / TH) * N;
    const int tiles = (cout / BN) * ((c0 + c1) / KC);
    const int target = 4 * (sm_count > 0 ? sm_count : 148);
    int gx = target / tiles;
    gx = gx < 1 ? 1 : (gx > slabs ? slabs : gx);
    k_conv3x3_wgrad<<<dim3((unsigned)gx, (unsigned)(cout / BN), (unsigned)((c0 + c1) / KC)), 128, 0,
                      (cudaStream_t)stream>>>(a);
    return launch_status();
}

int otf_unet_bias_grad(const void *dz, int C, long long npix, float *db, void *stream)
{
    OTF_CHECK(C > 0 && 256 % C == 0, 1, "bias_grad: C must divide 256");
    const int64_t per = 256 / C;
    int64_t nb = (npix + per * 64 - 1) / (per * 64);
    nb = nb < 1 ? 1 : (nb > 1184 ? 1184 : nb);
    k_bias_grad<<<(unsigned)nb, 256, 0, (cudaStream_t)stream>>>((const bf16 *)dz, C, npix, db);
    return launch_status();
}

int otf_unet_pool2(const void *x, void *y, int N, int H, int W, int C, void *stream)
{
    OTF_CHECK(C % 8 == 0 && H % 2 == 0 && W % 2 == 0, 1, "pool2: C % 8, even H, W");
    const int64_t n = (int64_t)N * (H / 2) * (W / 2) * (C / 8);
    k_pool2<<<blocks(n, 256), 256, 0, (cudaStream_t)stream>>>((const bf16 *)x, (bf16 *)y, N, H, W, C);
    return launch_status();
}

int otf_unet_pool2_bwd(const void *dy, const void *x, void *dx, int N, int H, int W, int C, void *stream)
{
    OTF_CHECK(C % 8 == 0 && H % 2 == 0 && W % 2 == 0, 1, "pool2_bwd: C % 8, even H, W");
    const int64_t n = (int64_t)N * H * W * (C / 8);
    k_pool2_bwd<<<blocks(n, 256), 256, 0, (cudaStream_t)stream>>>((const bf16 *)dy, (const bf16 *)x,
                                                                  (bf16 *)dx, N, H, W, C);
    return launch_status();
}

int otf_unet_up2_bwd(const void *dy, const void *x, void *dx, int N, int Hh, int Wh, int C, void *stream)
{
    OTF_CHECK(C % 8 == 0, 1, "up2_bwd: C % 8");
    const int64_t n = (int64_t)N * Hh * Wh * (C / 8);
    k_up2_bwd<<<blocks(n, 256), 256, 0, (cudaStream_t)stream>>>((const bf16 *)dy, (const bf16 *)x,
                                                                (bf16 *)dx, N, Hh, Wh, C);
    return launch_status();
}

int otf_unet_pack_input(const float *x, int cin, long long npix, void *y, void *stream)
{
    OTF_CHECK(cin >= 1 && cin <= 16, 1, "pack_input: 1..16 channels");
    k_pack_input<<<blocks(npix * 16, 256), 256, 0, (cudaStream_t)stream>>>(x, cin, npix, (bf16 *)y);
    return launch_status();
}

int otf_unet_head(const void *x, const float *w, const float *b, long long npix, float *out, void *stream)
{
    k_head<<<blocks(npix, 256), 256, 0, (cudaStream_t)stream>>>((const bf16 *)x, w, b, npix, out);
    return launch_status();
}

int otf_unet_head_bwd(const void *x, const float *w, const float *dout, long long npix, void *dx, float *dw,
                      float *db, void *stream)
{
    int64_t nb = (npix + 256 * 16 - 1) / (256 * 16);
    nb = nb < 1 ? 1 : (nb > 1184 ? 1184 : nb);
    k_head_bwd<<<(unsigned)nb, 256, 0, (cudaStream_t)stream>>>((const bf16 *)x, w, dout, npix, (bf16 *)dx, dw,
                                                               db);
    return launch_status();
}

int otf_unet_mse(const float *out, const float *target, const float *weight, long long n, float inv_norm,
                 float *dout, float *loss, void *stream)
{
    int64_t nb = (n + 256 * 8 - 1) / (256 * 8);
    nb = nb < 1 ? 1 : (nb > 1184 ? 1184 : nb);
    k_mse<<<(unsigned)nb, 256, 0, (cudaStream_t)stream>>>(out, target, weight, n, inv_norm, dout, loss);
    return launch_status();
}

int otf_unet_adam(float *p, const float *g, float *m, float *v, long long n, float lr, float b1, float b2,
                  float eps, int step, float weight_decay, void *stream)
{
    OTF_CHECK(step >= 1, 1, "adam: step counts from 1");
    float c1 = 1.f, c2 = 1.f, p1 = b1, p2 = b2;
    for (int s = step; s > 0; s >>= 1) {  // b^step by squaring
        if (s & 1) {
            c1 *= p1;
            c2 *= p2;
        }
        p1 *= p1;
        p2 *= p2;
    }
    k_adam<<<blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(p, g, m, v, n, lr, b1, b2, eps, 1.f - c1, 1.f - c2,
                                                             weight_decay);
    return launch_status();
}

int otf_unet_pack_weights(const float *w, int cout, int cin, void *wf, void *wb, void *stream)
{
    const int64_t n = (int64_t)9 * cout * cin;
    k_pack_weights<<<blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(w, cout, cin, (bf16 *)wf, (bf16 *)wb);
    return launch_status();
}

}  // extern "C"
