// Headless video frames of the forward modelling.
//
// The reference's cuda_simulate(en_out = 1) (regression_PML_single.cu:
// 619-700) sums Px + Pz into one field after every step (somaFrames,
// :312-327), copies it to the host and hands it to writeFramePipe
// (utils.cu:84-120), which maps the frame's [min, max] linearly onto
// 0..255, (P + (-min)) * (255 / (max - min)) in FP32 converted to an
// unsigned char, marks every receiver 255 and pipes the [Z][X] bytes into
// ffmpeg. Here the whole frame is made on the device: one pass for the
// frame's min and max, one for the bytes, one for the receiver marks; only
// the 8-bit frames cross PCIe. The arithmetic is the reference's, so with
// faithful numerics the bytes are the reference's bytes.
#include <climits>
#include <cstdint>
#include <vector>
#include "engine.h"

namespace otf {

namespace {

// Integer key with the order of the floats (sign-magnitude to two's
// complement); -0.0 sorts below +0.0, which changes neither the frame's
// offset nor its scale.
__device__ __forceinline__ int fkey(float v)
{
    const int b = __float_as_int(v);
    return b >= 0 ? b : b ^ 0x7fffffff;
}

__device__ __forceinline__ float unkey(int k) { return __int_as_float(k >= 0 ? k : k ^ 0x7fffffff); }

// The host's float -> unsigned char conversion as x86-64 compilers emit it:
// a truncating conversion to a 32-bit int (INT_MIN for NaN and out-of-range
// values) of which the low byte is stored. Values inside 0..255 are plain
// truncation; a frame with max == min gives 0 * inf = NaN -> 0.
__device__ __forceinline__ unsigned char to_u8(float q)
{
    const int iv = (q >= -2147483648.0f && q < 2147483648.0f) ? __float2int_rz(q) : INT_MIN;
    return (unsigned char)(iv & 0xff);
}

__device__ __forceinline__ float total_p(const float *__restrict__ px, const float *__restrict__ pz, int64_t o)
{
    return pz ? __fadd_rn(px[o], pz[o]) : px[o];
}

__global__ void k_frame_init(int *__restrict__ stats)
{
    stats[0] = INT_MAX;
    stats[1] = INT_MIN;
}

// stats[0] = key of the frame's minimum, stats[1] = key of its maximum
__global__ void __launch_bounds__(256) k_frame_stats(const float *__restrict__ px, const float *__restrict__ pz,
                                                     Layout L, int *__restrict__ stats)
{
    __shared__ int red[2][8];
    const int64_t n = (int64_t)L.X * L.Z;
    int lo = INT_MAX, hi = INT_MIN;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int z = (int)(i / L.X), x = (int)(i - (int64_t)z * L.X);
        const int k = fkey(total_p(px, pz, L.at(x, z)));
        lo = min(lo, k);
        hi = max(hi, k);
    }
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[0][w] = lo;
        red[1][w] = hi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); k++) {
            lo = min(lo, red[0][k]);
            hi = max(hi, red[1][k]);
        }
        atomicMin(&stats[0], lo);
        atomicMax(&stats[1], hi);
    }
}

// out[z][x] = (P + offset) * scale, offset = -min, scale = 255 / (max - min)
// (utils.cu:102-109), each operation rounded as the host's FP32 does
__global__ void __launch_bounds__(256) k_frame_bytes(const float *__restrict__ px, const float *__restrict__ pz,
                                                     Layout L, const int *__restrict__ stats,
                                                     unsigned char *__restrict__ out)
{
    const int64_t n = (int64_t)L.X * L.Z;
    const float mn = unkey(stats[0]), mx = unkey(stats[1]);
    const float offset = -mn;
    const float scale = __fdiv_rn(255.0f, __fsub_rn(mx, mn));
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int z = (int)(i / L.X), x = (int)(i - (int64_t)z * L.X);
        out[i] = to_u8(__fmul_rn(__fadd_rn(total_p(px, pz, L.at(x, z)), offset), scale));
    }
}

// receivers drawn white (utils.cu:110-113)
__global__ void k_frame_marks(unsigned char *__restrict__ out, const int *__restrict__ rx,
                              const int *__restrict__ rz, int n, int X)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        out[(int64_t)rz[i] * X + rx[i]] = 255;
}

struct FrameRun {
    Engine *eng;
    int every, shot, chunk, n_frames, done;
    int64_t cells;
    const float *px_base[2], *pz_base[2];
    Layout L;
    unsigned blocks;
    unsigned char *dev;
    unsigned char *host;
    int *stats;
    int *marks;
    int n_marks;
    Engine::FrameSink sink;
    void *ctx;
};

int flush(FrameRun &r, int n)
{
    const cudaStream_t st = r.eng->stream();
    OTF_CUDA(cudaMemcpyAsync(r.host, r.dev, (size_t)n * r.cells, cudaMemcpyDeviceToHost, st));
    if (r.eng->sync())
        return -1;
    return r.sink(r.ctx, r.host, n);
}

int on_step(void *ctx, int t, int slot)
{
    FrameRun &r = *static_cast<FrameRun *>(ctx);
    if (t % r.every != 0 || r.done >= r.n_frames)
        return 0;
    const cudaStream_t st = r.eng->stream();
    const int f = r.done % r.chunk;
    int *stats = r.stats + 2 * f;
    unsigned char *out = r.dev + (int64_t)f * r.cells;
    k_frame_init<<<1, 1, 0, st>>>(stats);
    k_frame_stats<<<r.blocks, 256, 0, st>>>(r.px_base[slot], r.pz_base[slot], r.L, stats);
    k_frame_bytes<<<r.blocks, 256, 0, st>>>(r.px_base[slot], r.pz_base[slot], r.L, stats, out);
    if (r.n_marks > 0)
        k_frame_marks<<<(r.n_marks + 127) / 128, 128, 0, st>>>(out, r.marks, r.marks + r.n_marks, r.n_marks, r.L.X);
    OTF_CUDA(cudaGetLastError());
    r.done++;
    if (r.done % r.chunk == 0 || r.done == r.n_frames)
        return flush(r, f + 1);
    return 0;
}

}  // namespace

int Engine::frames(int every, int shot, FrameSink sink, void *ctx)
{
    if (prepare())
        return -1;
    OTF_CHECK(every >= 1, 1, "frame interval must be >= 1");
    OTF_CHECK(shot >= 0 && shot < n_shots_, 1, "frame shot out of range");
    OTF_CHECK(sink != nullptr, 1, "frames: no sink");
    FrameRun r{};
    r.eng = this;
    r.every = every;
    r.shot = shot;
    r.n_frames = (cfg_.T - 1) / every;
    r.cells = (int64_t)cfg_.X * cfg_.Z;
    r.chunk = (int)std::max<int64_t>(1, std::min<int64_t>(r.n_frames, (int64_t(256) << 20) / r.cells));
    r.L = L_;
    r.sink = sink;
    r.ctx = ctx;
    const bool split = variant_in_use() >= 2;  // P total in the first field
    for (int s = 0; s < 2; s++) {
        r.px_base[s] = fld_[0][0][s] + (int64_t)shot * L_.slot;
        r.pz_base[s] = split ? nullptr : fld_[0][1][s] + (int64_t)shot * L_.slot;
    }
    int dev = 0, nsm = 0;
    OTF_CUDA(cudaGetDevice(&dev));
    OTF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    r.blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((r.cells + 255) / 256, (int64_t)nsm * 8));
    // receivers inside the grid, as the reference indexes its frame buffer
    std::vector<int> mk;
    for (int i = 0; i < n_rec_; i++)
        mk.push_back(rec_x_[i]);
    for (int i = 0; i < n_rec_; i++)
        mk.push_back(rec_z_[i]);
    r.n_marks = n_rec_;
    if (r.n_frames == 0)
        return forward(false);
    int rc = -1;
    r.dev = nullptr;
    r.host = nullptr;
    r.stats = nullptr;
    r.marks = nullptr;
    if (cudaMalloc(&r.dev, (size_t)r.chunk * r.cells) != cudaSuccess ||
        cudaMalloc(&r.stats, sizeof(int) * 2 * r.chunk) != cudaSuccess ||
        cudaMalloc(&r.marks, sizeof(int) * (mk.size() + 1)) != cudaSuccess ||
        cudaMallocHost(&r.host, (size_t)r.chunk * r.cells) != cudaSuccess) {
        set_error_msg(3, "frames: buffer allocation failed");
    } else if (cudaMemcpy(r.marks, mk.data(), sizeof(int) * mk.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        set_error_msg(3, "frames: receiver upload failed");
    } else {
        rc = emit_forward(false, on_step, &r);
        if (rc == 0)
            rc = sync();
        else
            cudaStreamSynchronize(stream());  // a failed sink leaves steps queued that write r.dev
    }
    cudaFree(r.dev);
    cudaFree(r.stats);
    cudaFree(r.marks);
    cudaFreeHost(r.host);
    return rc;
}

}  // namespace otf
