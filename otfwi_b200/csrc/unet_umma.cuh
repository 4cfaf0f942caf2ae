// 3x3 convolution on the 5th-generation tensor cores (tcgen05 / UMMA) for
// the preconditioner U-Net: an implicit GEMM per CTA with
//
//   M = 256 output pixels (a tile 8 wide x 32 tall of one image), as two
//       128-row MMAs (tile rows 0-15 and 16-31) that share every weight stage,
//   N = the CTA's output channels (cout, or a block of 256, <= 256),
//   K = 9 taps x the input channels, taken 16 channels (one MMA K) at a time.
//
// Warp roles, each stage a full / empty mbarrier pair:
//   warps 0, 2, 3 (producers): per 16-channel chunk, warp 0 loads the chunk's
//     weights of every tap ([tap][cout][8 ch] per 8-channel plane: 18 bulk
//     copies from the packed weights, or two tiled loads, load_chunk_weights)
//     and the input halo
//     (34 x 10 pixels x 8 channels per plane: one 4D TMA load per plane; the
//     tensor map's zero fill supplies the image border); a chunk of the upsampled second input is gathered
//     by the three warps with cp.async instead (nearest upsampling on load),
//     then made visible to the tensor cores (fence.proxy.async); each warp
//     arrives on the stage's full barrier;
//   warp 1 (one thread): waits for a stage, issues its 18 MMAs (9 taps x 2
//     halves; kind::f16, BF16 in, FP32 accumulators in tensor memory, 2 x N
//     columns), and commits them to the stage's empty barrier;
//   then all four warps: the epilogue reads the accumulators with tcgen05.ld
//     (warp w owns TMEM lanes 32w .. 32w+31), adds the bias, applies the ReLU
//     and the optional masks, and writes BF16 (16-byte stores) to the split
//     outputs as k_conv3x3 does.
// Both operands use the no-swizzle K-major canonical layout: a core matrix is
// 8 rows of 16 bytes. For tap (dy, dx) and half h the A operand starts at halo
// pixel (dy + 16 h) * 10 + dx: row m (pixel oy = m / 8, ox = m % 8) is 8
// consecutive halo pixels per core matrix, core matrices one halo row (160
// bytes) apart, the second K half in the other plane -- one descriptor per
// (tap, half), no copy.
//
// The weight gradient (k_conv3x3_wgrad_umma, below) keeps the 128-pixel slab
// (8 x 16) of the first version.
//
// Every mbarrier wait is bounded (tma.cuh: 0.5 s); on expiry the kernel sets
// the error flag, stops issuing, waits (bounded) for the copies and MMAs it
// issued, skips the epilogue, frees its tensor memory and exits.
#pragma once
// included inside namespace otf::unet by unet.cu, after tma.cuh

namespace umma {

constexpr int TWU = 8, THU = 16;              // output tile (x, y): 128 pixels
constexpr int HWU = TWU + 2, HHU = THU + 2;   // halo 10 x 18
constexpr int HPIX = HWU * HHU;               // 180 halo pixels
constexpr int PLANE_A = HPIX * 16;            // bytes of one 8-channel plane of the halo
constexpr int A_BYTES = 2 * PLANE_A;          // 5760

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    // start >> 4 [0,14), LBO >> 4 [16,30), SBO >> 4 [32,46), version 1 [46,48),
    // base offset 0, no swizzle (layout type 0 in [61,64))
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: FP32 accumulators, BF16 A and B, both
// K-major, M = 128, N.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int n)
{
    return (1u << 4)                          // D format F32
           | (1u << 7)                        // A format BF16
           | (1u << 10)                       // B format BF16
           | ((uint32_t)(n >> 3) << 17)       // N / 8
           | ((uint32_t)(128 >> 4) << 24);    // M / 16
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, bool acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"((uint32_t)acc)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     otf::smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(otf::smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v)
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,"
        "%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]),
          "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
          "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++)
        v[i] = __uint_as_float(r[i]);
}

}  // namespace umma

__device__ int g_unet_err;  // set by a timed-out wait of a U-Net tensor-core kernel

namespace umma {
constexpr int TH2 = 32;                                    // output tile height: 8 x 32 = 256 pixels
constexpr int HH2 = TH2 + 2;                               // halo 10 x 34
constexpr int HPIX2 = HWU * HH2;                           // 340 halo pixels
constexpr int PLANE2 = ((HPIX2 * 16 + 127) / 128) * 128;   // one 8-channel halo plane, 128-byte aligned
}  // namespace umma

// Tensor maps of one convolution: the inputs [N][H][W][c] as (c, W, H, N),
// box (8, 10, 34, 1) (x1: the second input at full resolution; unused when
// it is upsampled).
struct ConvMaps {
    CUtensorMap w, x0, x1;  // w: weights (cin, cout, 9), box (8, N, 9); used when no packed copy is given
};

// The weights of chunk kc for output channels [co0, co0 + N) into
// [plane][tap][co][8 ch] at dst (2 x 9 x N x 16 bytes, completion on bar).
// With the packed layout a.wp [cin / 8][9][cout][8] (k_pack_w_umma): 18
// contiguous runs of N x 16 bytes, one bulk copy each, whole sectors;
// otherwise two tiled loads of the [9][cout][cin] weights with an 8-channel
// box, 16 bytes per row.
__device__ __forceinline__ void load_chunk_weights(unsigned char *dst, const ConvArgs &a, const ConvMaps &maps,
                                                   int kc, int co0, int N, uint64_t *bar)
{
    if (a.wp) {
        for (int pt = 0; pt < 18; pt++) {  // plane * 9 + tap
            const int plane = pt / 9, tap = pt - 9 * plane;
            const bf16 *src = a.wp + ((int64_t)((kc * 2 + plane) * 9 + tap) * a.cout + co0) * 8;
            otf::bulk_load(dst + pt * N * 16, src, (uint32_t)(N * 16), bar);
        }
    } else {
        for (int h = 0; h < 2; h++)
            otf::tma_load_3d(dst + h * 9 * N * 16, &maps.w, kc * KC + 8 * h, co0, 0, bar);
    }
}

// w [9][cout][cin] -> wp [cin / 8][9][cout][8], 16 bytes per thread and step.
__global__ void k_pack_w_umma(const bf16 *__restrict__ w, bf16 *__restrict__ wp, int cout, int cin)
{
    const int64_t n = (int64_t)(cin / 8) * 9 * cout;
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x) {
        const int co = (int)(u % cout);
        const int64_t r = u / cout;
        const int tap = (int)(r % 9), cp = (int)(r / 9);
        reinterpret_cast<uint4 *>(wp)[u] =
            *reinterpret_cast<const uint4 *>(w + ((int64_t)tap * cout + co) * cin + cp * 8);
    }
}

// dynamic shared memory: NST stages of (two halo planes, two weight planes),
// then 2 NST + 1 barriers, the tensor-memory slot and the failure flag
__host__ __device__ constexpr int umma_stage_bytes(int n) { return 2 * umma::PLANE2 + 2 * 9 * n * 16; }
__host__ __device__ constexpr int umma_smem_bytes(int n, int nst) { return nst * umma_stage_bytes(n) + 256; }

// Epilogue of one 256-pixel tile: the calling warp reads TMEM lanes
// 32 * quarter .. +31 (one output pixel per lane and half) from the
// accumulators at column col0 (half h at col0 + h * N), adds the bias,
// applies the ReLU and the masks, and stores BF16 (16-byte vectors where 8
// channels lie on one side of the split, aligned).
__device__ __forceinline__ void conv_epilogue(const ConvArgs &a, uint32_t tmem, uint32_t quarter, int lane,
                                              uint32_t col0, int N, int n, int y0, int x0, int co0)
{
    const int m = (int)quarter * 32 + lane;
#pragma unroll 1
    for (int h = 0; h < 2; h++) {
        const int y = y0 + 16 * h + m / umma::TWU, x = x0 + (m % umma::TWU);
        const bool inside = y < a.H && x < a.W;
        const int64_t pix = ((int64_t)n * a.H + y) * a.W + x;
#pragma unroll 1
        for (int c0 = 0; c0 < N; c0 += 32) {
            float v[32];
            umma::tmem_ld32(tmem + ((quarter * 32u) << 16) + col0 + (uint32_t)(h * N + c0), v);
            if (!inside)
                continue;
#pragma unroll
            for (int g = 0; g < 32; g += 8) {
                const int co = co0 + c0 + g;
                float r[8];
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    r[j] = v[g + j];
                    if (a.bias)
                        r[j] += a.bias[co + j];
                    if (a.relu)
                        r[j] = fmaxf(r[j], 0.f);
                }
                const bool lo = co < a.split;
                const int cc = lo ? a.split : a.cout - a.split, ci = lo ? co : co - a.split;
                if (lo == (co + 7 < a.split) && ((cc | ci) & 7) == 0) {
                    // the 8 channels on one side, 16-byte aligned
                    bf16 *dst = (lo ? a.dst0 : a.dst1) + pix * cc + ci;
                    const bf16 *mask = lo ? a.mask0 : a.mask1;
                    if (mask) {
                        const uint4 mk = *reinterpret_cast<const uint4 *>(mask + pix * cc + ci);
                        const bf162 *m2 = reinterpret_cast<const bf162 *>(&mk);
#pragma unroll
                        for (int j = 0; j < 4; j++) {
                            if (!(__low2float(m2[j]) > 0.f))
                                r[2 * j] = 0.f;
                            if (!(__high2float(m2[j]) > 0.f))
                                r[2 * j + 1] = 0.f;
                        }
                    }
                    uint4 pk;
                    bf162 *p2 = reinterpret_cast<bf162 *>(&pk);
#pragma unroll
                    for (int j = 0; j < 4; j++)
                        p2[j] = __floats2bfloat162_rn(r[2 * j], r[2 * j + 1]);
                    *reinterpret_cast<uint4 *>(dst) = pk;
                    continue;
                }
#pragma unroll
                for (int j = 0; j < 8; j += 2) {
                    const int cj = co + j;
                    float v0 = r[j], v1 = r[j + 1];
                    const bool l2 = cj < a.split;
                    bf16 *dst = l2 ? a.dst0 : a.dst1;
                    const bf16 *mask = l2 ? a.mask0 : a.mask1;
                    const int c2 = l2 ? a.split : a.cout - a.split, i2 = l2 ? cj : cj - a.split;
                    if (mask) {
                        const bf162 mk = *reinterpret_cast<const bf162 *>(mask + pix * c2 + i2);
                        if (!(__low2float(mk) > 0.f))
                            v0 = 0.f;
                        if (!(__high2float(mk) > 0.f))
                            v1 = 0.f;
                    }
                    *reinterpret_cast<bf162 *>(dst + pix * c2 + i2) = __floats2bfloat162_rn(v0, v1);
                }
            }
        }
    }
}

// The halo planes of one 16-channel chunk (ch) of a 256-pixel tile, gathered
// with cp.async (zero fill outside the image; the second input upsampled on
// load) by `nw` warps, this warp being number `wi`; visible to the tensor
// cores on return.
__device__ __forceinline__ void conv_gather(const ConvArgs &a, unsigned char *st, int ch, int n, int y0, int x0,
                                            int wi, int nw, int lane)
{
    for (int i = wi * 32 + lane; i < umma::HPIX2 * 2; i += 32 * nw) {
        const int px = i >> 1, h = i & 1;
        const int hy = px / umma::HWU, hx = px - hy * umma::HWU;
        const int gy = y0 + hy - 1, gx = x0 + hx - 1;
        const bool in = gy >= 0 && gy < a.H && gx >= 0 && gx < a.W;
        const void *src = in ? (const void *)in_ptr(a, n, gy, gx, ch + 8 * h) : (const void *)a.w;
        cp_async16(reinterpret_cast<uint32_t *>(st + h * umma::PLANE2 + px * 16), src, in ? 16 : 0);
    }
    cp_commit();
    cp_wait<0>();
    umma::fence_proxy_async();  // cp.async writes -> visible to the tensor cores
}

template <int NST>
__global__ void __launch_bounds__(128) k_conv3x3_umma(const __grid_constant__ ConvArgs a,
                                                      const __grid_constant__ ConvMaps maps, int N)
{
    extern __shared__ __align__(1024) unsigned char smu[];
    const int sb = umma_stage_bytes(N);
    uint64_t *full = reinterpret_cast<uint64_t *>(smu + NST * sb);
    uint64_t *empty = full + NST;
    uint64_t *done = empty + NST;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(done + 1);
    int *fail = reinterpret_cast<int *>(tslot + 1);
    const int tiles_x = (a.W + umma::TWU - 1) / umma::TWU, tiles_y = (a.H + umma::TH2 - 1) / umma::TH2;
    int bidx = blockIdx.x;
    const int n = bidx / (tiles_x * tiles_y);
    bidx -= n * tiles_x * tiles_y;
    const int ty = bidx / tiles_x, tx = bidx - ty * tiles_x;
    const int y0 = ty * umma::TH2, x0 = tx * umma::TWU, co0 = blockIdx.y * N;
    const int cin = a.c0 + a.c1, nk = cin / KC;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t ncols = 32;
    while (ncols < 2u * (uint32_t)N)
        ncols <<= 1;

    if (threadIdx.x == 0) {
        for (int s = 0; s < NST; s++)
            otf::mbar_init(&full[s], 3);  // one arrival per producer warp
        for (int s = NST; s < 2 * NST + 1; s++)
            otf::mbar_init(&full[s], 1);  // empty barriers and `done`: one commit each
        *fail = 0;
        otf::fence_barrier_init();
    }
    if (warp == 0)
        umma::tmem_alloc(tslot, ncols);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *tslot;

    if (warp != 1) {
        // producers: warp 0 issues the TMA loads; warps 0, 2 and 3 share the
        // cp.async gather of an upsampled chunk; each arrives once per chunk
        const int pi = warp == 0 ? 0 : warp - 1;
        if (warp == 0 && lane == 0) {
            if (!a.wp)
                otf::tma_prefetch_desc(&maps.w);
            otf::tma_prefetch_desc(&maps.x0);
            if (a.c1 && !a.up1)
                otf::tma_prefetch_desc(&maps.x1);
        }
        const uint32_t wbytes = 2u * 9u * (uint32_t)N * 16u, abytes = 2u * umma::HPIX2 * 16u;
        int issued = 0;
        for (int kc = 0; kc < nk; kc++) {
            const int s = kc % NST;
            if (kc >= NST) {
                int okw = 1;
                if (lane == 0)
                    okw = otf::mbar_wait(&empty[s], (uint32_t)((kc / NST - 1) & 1), &g_unet_err) ? 1 : 0;
                if (!__shfl_sync(0xffffffffu, okw, 0)) {
                    if (lane == 0)
                        *fail = 1;
                    break;
                }
            }
            unsigned char *st = smu + s * sb;
            const int ch = kc * KC;
            const bool from1 = ch >= a.c0;
            const bool gather = from1 && a.up1;
            if (warp == 0 && lane == 0) {
                otf::mbar_expect_tx(&full[s], wbytes + (gather ? 0u : abytes));
                load_chunk_weights(st + 2 * umma::PLANE2, a, maps, kc, co0, N, &full[s]);
                if (!gather) {
                    const CUtensorMap *mx = from1 ? &maps.x1 : &maps.x0;
                    const int c = from1 ? ch - a.c0 : ch;
                    for (int h = 0; h < 2; h++)
                        otf::tma_load_4d(st + h * umma::PLANE2, mx, c + 8 * h, x0 - 1, y0 - 1, n, &full[s]);
                }
            }
            if (gather)
                conv_gather(a, st, ch, n, y0, x0, pi, 3, lane);
            __syncwarp();
            if (lane == 0)
                otf::mbar_arrive(&full[s]);
            issued = kc + 1;
        }
        // wait for every copy the producers issued (the last fill of each stage)
        if (warp == 0 && lane == 0)
            for (int kc = issued > NST ? issued - NST : 0; kc < issued; kc++)
                otf::mbar_wait(&full[kc % NST], (uint32_t)((kc / NST) & 1), &g_unet_err);
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = umma::instr_desc_bf16(N);
            for (int kc = 0; kc < nk; kc++) {
                const int s = kc % NST;
                if (!otf::mbar_wait(&full[s], (uint32_t)((kc / NST) & 1), &g_unet_err)) {
                    *fail = 1;
                    break;
                }
                umma::fence_after_sync();
                const uint32_t abase = otf::smem_u32(smu + s * sb);
                const uint32_t bbase = abase + 2 * umma::PLANE2;
#pragma unroll
                for (int tap = 0; tap < 9; tap++) {
                    const int dy = tap / 3, dx = tap - 3 * (tap / 3);
                    const uint64_t bd = umma::smem_desc(bbase + tap * N * 16, 9 * N * 16, 128);
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const uint64_t ad = umma::smem_desc(abase + ((dy + 16 * h) * umma::HWU + dx) * 16,
                                                            umma::PLANE2, umma::HWU * 16);
                        umma::mma_bf16(tmem + (uint32_t)(h * N), ad, bd, idesc, kc > 0 || tap > 0);
                    }
                }
                umma::mma_commit(&empty[s]);
            }
            umma::mma_commit(done);  // arrives once every MMA issued before it has completed
        }
        __syncwarp();
    }
    // every role done issuing; the accumulators are final once `done` completes
    __syncthreads();
    const bool ok = otf::mbar_wait(done, 0, &g_unet_err) && *fail == 0;
    umma::fence_after_sync();

    if (ok)
        conv_epilogue(a, tmem, (uint32_t)warp, lane, 0u, N, n, y0, x0, co0);
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        umma::fence_after_sync();
        umma::tmem_dealloc(tmem, ncols);
    }
}

// Persistent form for the small layers (at most 128 output channels per CTA
// and all of the CTA's weights within kResWeightBytes): the weights of every
// chunk and tap stay in shared memory for the CTA's life (loaded once at the
// start; then only halo tiles stream); the CTA walks 256-pixel tiles
// blockIdx.x, + gridDim.x, ...; two accumulator buffers (2 x 2N
// tensor-memory columns) let the epilogue of one tile overlap the MMAs of the
// next. (With the weights streamed with the halo instead, the persistent form
// measured slower than one tile per CTA on the large layers.) Warps: 0
// producer (TMA loads; with warps 6 and 7 the cp.async gather of an
// upsampled chunk), 1 the MMA issuer (one thread), 2-5 the epilogue (TMEM
// lane quarters 2, 3, 0, 1). Per halo stage a full (three producer warps) /
// empty (MMA commit) barrier pair; per accumulator buffer a full (MMA commit)
// / empty (four epilogue warps) pair. Bounded waits as the kernel above; a
// failed wait sets the error flag, the role stops, and teardown waits
// (bounded) for the MMAs and copies issued.
constexpr int kResWeightBytes = 96 * 1024;
constexpr int kResStages = 4;
__host__ __device__ constexpr int umma_res_smem_bytes(int n, int nk)
{
    return nk * 2 * 9 * n * 16 + kResStages * 2 * umma::PLANE2 + 256;
}

__global__ void __launch_bounds__(256) k_conv3x3_umma_res(const __grid_constant__ ConvArgs a,
                                                         const __grid_constant__ ConvMaps maps, int N, int n_tiles)
{
    extern __shared__ __align__(1024) unsigned char smu[];
    constexpr int NST = kResStages;
    const int cin = a.c0 + a.c1, nk = cin / KC;
    const int wchunk = 2 * 9 * N * 16;          // bytes of one chunk's weights (two planes)
    unsigned char *wsm = smu;                   // [chunk][plane][tap][co][8 ch]
    unsigned char *hsm = smu + nk * wchunk;     // NST halo stages
    constexpr int SA = 2 * umma::PLANE2;        // a stage: two halo planes
    uint64_t *full = reinterpret_cast<uint64_t *>(hsm + NST * SA);
    uint64_t *empty = full + NST;
    uint64_t *acc_full = empty + NST;
    uint64_t *acc_empty = acc_full + 2;
    uint64_t *wbar = acc_empty + 2;
    uint64_t *done = wbar + 1;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(done + 1);
    int *fail = reinterpret_cast<int *>(tslot + 1);
    const int tiles_x = (a.W + umma::TWU - 1) / umma::TWU, tiles_y = (a.H + umma::TH2 - 1) / umma::TH2;
    const int co0 = blockIdx.y * N;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int my_tiles = (int)blockIdx.x < n_tiles ? (n_tiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    uint32_t ncols = 32;
    while (ncols < 4u * (uint32_t)N)
        ncols <<= 1;

    if (threadIdx.x == 0) {
        for (int i = 0; i < NST; i++) {
            otf::mbar_init(&full[i], 3);   // one arrival per producer warp
            otf::mbar_init(&empty[i], 1);  // one MMA commit
        }
        for (int i = 0; i < 2; i++) {
            otf::mbar_init(&acc_full[i], 1);   // one MMA commit
            otf::mbar_init(&acc_empty[i], 4);  // one arrival per epilogue warp
        }
        otf::mbar_init(wbar, 1);
        otf::mbar_init(done, 1);
        *fail = 0;
        otf::fence_barrier_init();
    }
    if (warp == 0)
        umma::tmem_alloc(tslot, ncols);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *tslot;

    auto origin = [&](int li, int &n, int &y0, int &x0) {
        int t = (int)blockIdx.x + li * (int)gridDim.x;
        n = t / (tiles_x * tiles_y);
        t -= n * tiles_x * tiles_y;
        const int ty = t / tiles_x;
        y0 = ty * umma::TH2;
        x0 = (t - ty * tiles_x) * umma::TWU;
    };

    if (warp == 0 || warp >= 6) {
        // producers
        const int pi = warp == 0 ? 0 : warp - 5;
        if (warp == 0 && lane == 0) {
            if (!a.wp)
                otf::tma_prefetch_desc(&maps.w);
            otf::tma_prefetch_desc(&maps.x0);
            if (a.c1 && !a.up1)
                otf::tma_prefetch_desc(&maps.x1);
            otf::mbar_arrive_expect_tx(wbar, (uint32_t)(nk * wchunk));
            for (int kc = 0; kc < nk; kc++)
                load_chunk_weights(wsm + kc * wchunk, a, maps, kc, co0, N, wbar);
        }
        const uint32_t abytes = 2u * umma::HPIX2 * 16u;
        int g = 0;
        bool ok = true;
        for (int li = 0; li < my_tiles && ok; li++) {
            int n, y0, x0;
            origin(li, n, y0, x0);
            for (int kc = 0; kc < nk; kc++, g++) {
                const int s = g % NST;
                if (g >= NST) {
                    int okw = 1;
                    if (lane == 0)
                        okw = otf::mbar_wait(&empty[s], (uint32_t)((g / NST - 1) & 1), &g_unet_err) ? 1 : 0;
                    if (!__shfl_sync(0xffffffffu, okw, 0)) {
                        if (lane == 0)
                            *fail = 1;
                        ok = false;
                        break;
                    }
                }
                unsigned char *st = hsm + s * SA;
                const int ch = kc * KC;
                const bool from1 = ch >= a.c0;
                const bool gather = from1 && a.up1;
                if (warp == 0 && lane == 0 && !gather) {
                    otf::mbar_expect_tx(&full[s], abytes);
                    const CUtensorMap *mx = from1 ? &maps.x1 : &maps.x0;
                    const int c = from1 ? ch - a.c0 : ch;
                    for (int h = 0; h < 2; h++)
                        otf::tma_load_4d(st + h * umma::PLANE2, mx, c + 8 * h, x0 - 1, y0 - 1, n, &full[s]);
                }
                if (gather)
                    conv_gather(a, st, ch, n, y0, x0, pi, 3, lane);
                __syncwarp();
                if (lane == 0)
                    otf::mbar_arrive(&full[s]);
            }
        }
        // wait for every copy issued: the weights and the last fill of each stage
        if (warp == 0 && lane == 0) {
            otf::mbar_wait(wbar, 0, &g_unet_err);
            for (int gg = g > NST ? g - NST : 0; gg < g; gg++)
                otf::mbar_wait(&full[gg % NST], (uint32_t)((gg / NST) & 1), &g_unet_err);
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = umma::instr_desc_bf16(N);
            bool ok = otf::mbar_wait(wbar, 0, &g_unet_err);
            int g = 0;
            for (int li = 0; li < my_tiles && ok; li++) {
                const int ab = li & 1;
                if (li >= 2 && !otf::mbar_wait(&acc_empty[ab], (uint32_t)(((li >> 1) - 1) & 1), &g_unet_err)) {
                    ok = false;
                    break;
                }
                umma::fence_after_sync();
                const uint32_t d = tmem + (uint32_t)(ab * 2 * N);
                for (int kc = 0; kc < nk; kc++, g++) {
                    const int s = g % NST;
                    if (!otf::mbar_wait(&full[s], (uint32_t)((g / NST) & 1), &g_unet_err)) {
                        ok = false;
                        break;
                    }
                    umma::fence_after_sync();
                    const uint32_t abase = otf::smem_u32(hsm + s * SA);
                    const uint32_t bbase = otf::smem_u32(wsm + kc * wchunk);
#pragma unroll
                    for (int tap = 0; tap < 9; tap++) {
                        const int dy = tap / 3, dx = tap - 3 * (tap / 3);
                        const uint64_t bd = umma::smem_desc(bbase + tap * N * 16, 9 * N * 16, 128);
#pragma unroll
                        for (int h = 0; h < 2; h++) {
                            const uint64_t ad = umma::smem_desc(abase + ((dy + 16 * h) * umma::HWU + dx) * 16,
                                                                umma::PLANE2, umma::HWU * 16);
                            umma::mma_bf16(d + (uint32_t)(h * N), ad, bd, idesc, kc > 0 || tap > 0);
                        }
                    }
                    umma::mma_commit(&empty[s]);
                }
                if (!ok)
                    break;
                umma::mma_commit(&acc_full[ab]);
            }
            if (!ok)
                *fail = 1;
            umma::mma_commit(done);  // arrives once every MMA issued has completed
        }
        __syncwarp();
    } else {
        // epilogue: warps 2-5, TMEM lane quarter warp % 4
        const uint32_t quarter = (uint32_t)(warp & 3);
        for (int li = 0; li < my_tiles; li++) {
            const int ab = li & 1;
            const bool okl = otf::mbar_wait(&acc_full[ab], (uint32_t)((li >> 1) & 1), &g_unet_err);
            if (!__all_sync(0xffffffffu, okl)) {
                if (lane == 0)
                    *fail = 1;
                break;
            }
            umma::fence_after_sync();
            int n, y0, x0;
            origin(li, n, y0, x0);
            conv_epilogue(a, tmem, quarter, lane, (uint32_t)(ab * 2 * N), N, n, y0, x0, co0);
            umma::fence_before_sync();
            __syncwarp();
            if (lane == 0)
                otf::mbar_arrive(&acc_empty[ab]);
        }
    }
    __syncthreads();
    // teardown: every MMA issued has completed before the tensor memory is freed
    if (warp == 0) {
        otf::mbar_wait(done, 0, &g_unet_err);
        umma::fence_after_sync();
        umma::tmem_dealloc(tmem, ncols);
    }
}

// Weight gradient on the tcgen05 tensor cores:
//
//   dW[dy * 3 + dx][co][ci] += sum over pixels p of dz[p][co] * x[p + (dy - 1, dx - 1)][ci],
//
// an implicit GEMM per CTA with M = 128 output channels (rows beyond cout are
// the zero fill of the dz tensor map), N = the three dx taps x NW input
// channels (96 or 48), K = pixels, 16 (two rows of an 8 x 16 slab) per MMA;
// the three dy taps are three accumulators (3 N tensor-memory columns). Both
// operands are MN-major (channels contiguous, as stored): a core matrix is 8
// channels x 8 pixels, 128 contiguous bytes. Per slab a stage holds dz as
// [co / 8][128 pixels][8 co] (16 TMA boxes of 8 channels x 8 x 16 pixels) and,
// for each dx, the input's 8-column window shifted by dx over the slab's 18
// halo rows as [dx][ci / 8][18 x 8 pixels][8 ci] (3 NW / 8 boxes of 8 x 8 x
// 18; an upsampled input gathered by cp.async instead). The B operand of dy
// and K step s then starts at halo row 2 s + dy of every (dx, ci group)
// window: K groups 128 bytes apart, N groups one window (2304 bytes) apart;
// 24 MMAs per slab instead of 72 with one tap per accumulator, and a
// third of the shared-memory operand reads per multiply-add. Warp roles as
// the forward kernel: warps 0, 2, 3 stage (lane 0 of warp 0 the TMA loads,
// the three warps the gather), one thread of warp 1 issues the MMAs, then
// the four warps add the CTA's 9 x 128 x NW partial sums to dw with FP32
// atomics. Bounded waits as the forward kernel.
namespace umma {
constexpr int WG_A = 16 * 128 * 16;   // dz of a slab: 16 groups of 8 channels x 128 pixels x 16 bytes
constexpr int WG_WIN = 18 * 8 * 16;   // one (dx, channel group) window: 18 halo rows x 8 pixels x 16 bytes
}  // namespace umma
__host__ __device__ constexpr int umma_wg_stage_bytes(int nw) { return umma::WG_A + 3 * (nw / 8) * umma::WG_WIN; }
__host__ __device__ constexpr int umma_wg_smem_bytes(int nw, int nst) { return nst * umma_wg_stage_bytes(nw) + 256; }

__host__ __device__ constexpr uint32_t instr_desc_bf16_mn(int n)
{
    return umma::instr_desc_bf16(n) | (1u << 15) | (1u << 16);  // A and B MN-major
}

// Tensor maps of one weight gradient: dz (cout, W, H, N), box (8, 8, 16, 1);
// the inputs (c, W, H, N), box (8, 8, 18, 1) (x1 at full resolution; unused
// when upsampled).
struct WgradMaps {
    CUtensorMap dz, x0, x1;
};

template <int NW, int NST>
__global__ void __launch_bounds__(128) k_conv3x3_wgrad_umma(const __grid_constant__ WgradArgs a,
                                                            const __grid_constant__ WgradMaps maps, int slabs_per_cta)
{
    extern __shared__ __align__(1024) unsigned char smu[];
    constexpr int SB = umma_wg_stage_bytes(NW);
    constexpr int NB = 3 * NW;                       // N of one MMA: 3 dx taps x NW channels
    constexpr uint32_t NCOLS = 3 * NB <= 256 ? 256u : 512u;
    constexpr int NG = NW / 8;                       // input channel groups
    uint64_t *full = reinterpret_cast<uint64_t *>(smu + NST * SB);
    uint64_t *empty = full + NST;
    uint64_t *done = empty + NST;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(done + 1);
    int *fail = reinterpret_cast<int *>(tslot + 1);
    const int co0 = blockIdx.y * 128, ci0 = blockIdx.z * NW;
    const int cin = a.c0 + a.c1;
    const int tiles_x = (a.W + umma::TWU - 1) / umma::TWU, tiles_y = (a.H + umma::THU - 1) / umma::THU;
    const int n_slabs = tiles_x * tiles_y * a.N;
    const int s_begin = blockIdx.x * slabs_per_cta, s_end = min(n_slabs, s_begin + slabs_per_cta);
    const int nsl = s_end > s_begin ? s_end - s_begin : 0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    ConvArgs ca{};
    ca.src0 = a.src0;
    ca.src1 = a.src1;
    ca.c0 = a.c0;
    ca.c1 = a.c1;
    ca.up1 = a.up1;
    ca.N = a.N;
    ca.H = a.H;
    ca.W = a.W;

    if (threadIdx.x == 0) {
        for (int i = 0; i < NST; i++)
            otf::mbar_init(&full[i], 3);  // one arrival per producer warp
        for (int i = NST; i < 2 * NST + 1; i++)
            otf::mbar_init(&full[i], 1);  // empty barriers and `done`: one commit each
        *fail = 0;
        otf::fence_barrier_init();
    }
    if (warp == 0)
        umma::tmem_alloc(tslot, NCOLS);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *tslot;

    if (warp != 1) {
        // producers: warp 0 issues the TMA loads; warps 0, 2 and 3 share the
        // gather of the upsampled channel groups; each arrives once per slab
        const int pi = warp == 0 ? 0 : warp - 1;
        if (warp == 0 && lane == 0) {
            otf::tma_prefetch_desc(&maps.dz);
            otf::tma_prefetch_desc(&maps.x0);
            if (a.c1 && !a.up1)
                otf::tma_prefetch_desc(&maps.x1);
        }
        int issued = 0;
        for (int k = 0; k < nsl; k++) {
            const int s = k % NST;
            if (k >= NST) {
                int okw = 1;
                if (lane == 0)
                    okw = otf::mbar_wait(&empty[s], (uint32_t)((k / NST - 1) & 1), &g_unet_err) ? 1 : 0;
                if (!__shfl_sync(0xffffffffu, okw, 0)) {
                    if (lane == 0)
                        *fail = 1;
                    break;
                }
            }
            int b = s_begin + k;
            const int n = b / (tiles_x * tiles_y);
            b -= n * tiles_x * tiles_y;
            const int ty = b / tiles_x, tx = b - ty * tiles_x;
            const int y0 = ty * umma::THU, x0 = tx * umma::TWU;
            unsigned char *st = smu + s * SB;
            unsigned char *sx = st + umma::WG_A;
            if (warp == 0 && lane == 0) {
                uint32_t bytes = umma::WG_A;
                for (int g = 0; g < NG; g++)
                    if (!(a.up1 && ci0 + 8 * g >= a.c0))
                        bytes += 3u * umma::WG_WIN;
                otf::mbar_expect_tx(&full[s], bytes);
                for (int g = 0; g < 16; g++)
                    otf::tma_load_4d(st + g * 128 * 16, &maps.dz, co0 + 8 * g, x0, y0, n, &full[s]);
                for (int g = 0; g < NG; g++) {
                    const int c = ci0 + 8 * g;
                    if (a.up1 && c >= a.c0)
                        continue;
                    const CUtensorMap *mx = c < a.c0 ? &maps.x0 : &maps.x1;
                    const int cc = c < a.c0 ? c : c - a.c0;
                    for (int dx = 0; dx < 3; dx++)
                        otf::tma_load_4d(sx + (dx * NG + g) * umma::WG_WIN, mx, cc, x0 - 1 + dx, y0 - 1, n,
                                         &full[s]);
                }
            }
            if (a.up1 && ci0 + NW > a.c0) {
                // channel groups of the upsampled second input: gathered
                for (int i = pi * 32 + lane; i < 3 * NG * 144; i += 96) {
                    const int win = i / 144, px = i - win * 144;
                    const int dx = win / NG, g = win - dx * NG;
                    const int c = ci0 + 8 * g;
                    if (c < a.c0)
                        continue;
                    const int gy = y0 - 1 + px / 8, gx = x0 - 1 + dx + (px & 7);
                    const bool in = gy >= 0 && gy < a.H && gx >= 0 && gx < a.W;
                    const void *src = in ? (const void *)in_ptr(ca, n, gy, gx, c) : (const void *)a.dz;
                    cp_async16(reinterpret_cast<uint32_t *>(sx + win * umma::WG_WIN + px * 16), src, in ? 16 : 0);
                }
                cp_commit();
                cp_wait<0>();
                umma::fence_proxy_async();
            }
            __syncwarp();
            if (lane == 0)
                otf::mbar_arrive(&full[s]);
            issued = k + 1;
        }
        if (warp == 0 && lane == 0)
            for (int k = issued > NST ? issued - NST : 0; k < issued; k++)
                otf::mbar_wait(&full[k % NST], (uint32_t)((k / NST) & 1), &g_unet_err);
        __syncwarp();
    } else {
        if (lane == 0) {
            const uint32_t idesc = instr_desc_bf16_mn(NB);
            for (int k = 0; k < nsl; k++) {
                const int s = k % NST;
                if (!otf::mbar_wait(&full[s], (uint32_t)((k / NST) & 1), &g_unet_err)) {
                    *fail = 1;
                    break;
                }
                umma::fence_after_sync();
                const uint32_t abase = otf::smem_u32(smu + s * SB);
                const uint32_t bbase = abase + umma::WG_A;
#pragma unroll
                for (int dy = 0; dy < 3; dy++) {
#pragma unroll
                    for (int ks = 0; ks < 8; ks++) {
                        // A: channel groups 2048 bytes apart, K groups (tile rows) 128 bytes apart
                        const uint64_t ad = umma::smem_desc(abase + ks * 256, 128, 128 * 16);
                        // B: K groups (halo rows) 128 bytes apart, (dx, channel group) windows one window apart
                        const uint64_t bd = umma::smem_desc(bbase + (2 * ks + dy) * 128, 128, umma::WG_WIN);
                        umma::mma_bf16(tmem + (uint32_t)(dy * NB), ad, bd, idesc, k > 0 || ks > 0);
                    }
                }
                umma::mma_commit(&empty[s]);
            }
            umma::mma_commit(done);
        }
        __syncwarp();
    }
    __syncthreads();
    const bool ok = otf::mbar_wait(done, 0, &g_unet_err) && *fail == 0;
    umma::fence_after_sync();

    if (ok && nsl > 0) {
        const int co = co0 + warp * 32 + lane;  // TMEM lane = output channel row
#pragma unroll 1
        for (int dy = 0; dy < 3; dy++) {
#pragma unroll 1
            for (int dx = 0; dx < 3; dx++) {
#pragma unroll 1
                for (int c = 0; c < NW; c += 16) {
                    // 32 columns from (dy, dx, c) (inside the allocation); the
                    // first 16 are channels c .. c+15 of this tap
                    float v[32];
                    umma::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(dy * NB + dx * NW + c), v);
                    if (co < a.cout) {
                        float *d = a.dw + ((int64_t)(dy * 3 + dx) * a.cout + co) * cin + ci0 + c;
#pragma unroll
                        for (int j = 0; j < 16; j++)
                            atomicAdd(d + j, v[j]);
                    }
                }
            }
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        umma::fence_after_sync();
        umma::tmem_dealloc(tmem, NCOLS);
    }
}
