// Engine implementation: device buffers, per-tile point tables, CUDA graphs
// of the time loops, and the small helper kernels around the fused steps.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <cudaTypedefs.h>
#include "engine.h"
#include "misfit.h"
#include "pml_step_unfused.cuh"
#include "pml_step_paired.cuh"
#include "pml_step_fused.cuh"

namespace otf {

const TileShape kTileShapes[kNumTileShapes] = {{56, 56}, {120, 24}, {120, 56}, {248, 24}, {56, 24}};

// ---------------------------------------------------------- helper kernels

// Running integral of each row (somaFonteIntegral's "integral[n] +=",
// regression_PML_single.cu:285-288): tab[r][t] = sum_{u=1..t} s[r][u], or of
// the time-flipped series s[r][T-1-u]; sequential FP32 adds in the
// reference's order, tab[r][0] = 0.
__global__ void k_prefix_rows(const float *__restrict__ src, float *__restrict__ tab, int rows,
                              int T, int flip)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows)
        return;
    const float *s = src + (int64_t)r * T;
    float *o = tab + (int64_t)r * T;
    float acc = 0.f;
    o[0] = 0.f;
    for (int t = 1; t < T; t++) {
        acc = __fadd_rn(acc, flip ? s[T - 1 - t] : s[t]);
        o[t] = acc;
    }
}

// Padded P coefficients from c^2: forward / adjoint (c2*dt)/dx
// (regression_PML_single.cu:512) and reconstruction c2*(dt/dx) (:517).
__global__ void k_prep_q(const float *__restrict__ cq, float *__restrict__ qf,
                         float *__restrict__ qr, Layout L, float dx, float dt)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.slot)
        return;
    const int prow = (int)(i / L.pitch), pcol = (int)(i - (int64_t)prow * L.pitch);
    const int x = pcol - PAD, z = prow - PAD;
    float vf = 0.f, vr = 0.f;
    if (x >= 0 && x < L.X && z >= 0 && z < L.Z) {
        const float c = cq[(int64_t)z * L.X + x];
        vf = __fdiv_rn(__fmul_rn(c, dt), dx);
        vr = __fmul_rn(c, __fdiv_rn(dt, dx));
    }
    qf[i] = vf;
    if (qr)
        qr[i] = vr;
}

// Sum of the padded per-shot gradients into an unpadded [Z*X] array, in shot
// order, then either divided by the shot count in FP32 (the wrapper's
// grad_acc += grad; grad_acc / n_source, cuda_interface_pml.py:225-235) when
// scale == 0, or multiplied by scale.
__global__ void k_grad_sum(const float *__restrict__ g, float *__restrict__ out, Layout L,
                           int n_shots, int64_t stride, float scale)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)L.X * L.Z)
        return;
    const int z = (int)(i / L.X), x = (int)(i - (int64_t)z * L.X);
    const int64_t o = L.at(x, z);
    float acc = 0.f;
    for (int s = 0; s < n_shots; s++)
        acc = __fadd_rn(acc, g[o + stride * s]);
    out[i] = scale == 0.f ? __fdiv_rn(acc, (float)n_shots)
                          : (scale == 1.f ? acc : __fmul_rn(acc, scale));
}

// ------------------------------------------------------- kernel dispatch

struct KernelSet {
    // v1: one tile per CTA
    void (*fwd)(const StepParams);
    void (*fwd_ring)(const StepParams);
    void (*rev)(const StepParams);
    size_t smem;
    // v2: persistent, TMA-pipelined (null when the shape does not fit)
    void (*fwd_tma)(const TmaParams);
    void (*fwd_ring_tma)(const TmaParams);
    void (*rev_tma)(const TmaParams);
    size_t smem_fwd_tma, smem_rev_tma;
    int grid_fwd_tma, grid_rev_tma;  // persistent grid sizes (set with the attributes)
    // v3: strip-split kernels (fast numerics only; null when not compiled)
    void (*fwd_split)(const TmaParams);
    void (*fwd_ring_split)(const TmaParams);
    void (*rev_split)(const TmaParams);
    size_t smem_fwd_split, smem_rev_split;
    int grid_fwd_split, grid_rev_split, nth_split;
};

template <int TX, int TZ, class Prec, bool SEP>
static KernelSet make_set()
{
    KernelSet k{};
    k.fwd = k_forward_step<TX, TZ, Prec, SEP, false>;
    k.fwd_ring = k_forward_step<TX, TZ, Prec, SEP, true>;
    k.rev = k_reverse_step<TX, TZ, Prec, SEP>;
    k.smem = (size_t)TileGeom<TX, TZ>::SMEM_FLOATS * sizeof(float);
    return k;
}

template <int TX, int TZ, class Prec, bool SEP, int MINB>
static KernelSet make_set_tma()
{
    KernelSet k = make_set<TX, TZ, Prec, SEP>();
    k.fwd_tma = k_forward_tma<TX, TZ, Prec, SEP, false, MINB>;
    k.fwd_ring_tma = k_forward_tma<TX, TZ, Prec, SEP, true, MINB>;
    k.rev_tma = k_reverse_tma<TX, TZ, Prec, SEP, MINB>;
    k.smem_fwd_tma = TmaGeom<TX, TZ>::FWD_BYTES;
    k.smem_rev_tma = TmaGeom<TX, TZ>::REV_BYTES;
    return k;
}

template <int TX, int TZ, int BH, int NTH, int MINB>
static void add_split(KernelSet &k)
{
    using G = SplitGeom<TX, TZ, BH, NTH>;
    k.fwd_split = k_forward_split<TX, TZ, BH, NTH, false, MINB>;
    k.fwd_ring_split = k_forward_split<TX, TZ, BH, NTH, true, MINB>;
    k.rev_split = k_reverse_split<TX, TZ, BH, NTH, MINB>;
    k.smem_fwd_split = G::FWD_BYTES;
    k.smem_rev_split = G::REV_BYTES;
    k.nth_split = NTH;
}

struct KernelTable {
    KernelSet s[kNumTileShapes][2][2];  // [shape][precision][separable]
    bool attrs_set = false;
    KernelTable()
    {
        memset(s, 0, sizeof(s));
        s[0][kFaithful][1] = make_set_tma<56, 56, Faithful, true, 1>();
        s[0][kFast][1] = make_set_tma<56, 56, Fast, true, 1>();
        s[1][kFaithful][1] = make_set_tma<120, 24, Faithful, true, 1>();
        s[1][kFast][1] = make_set_tma<120, 24, Fast, true, 1>();
        s[2][kFaithful][1] = make_set<120, 56, Faithful, true>();
        s[2][kFast][1] = make_set<120, 56, Fast, true>();
        s[3][kFaithful][1] = make_set<248, 24, Faithful, true>();
        s[3][kFast][1] = make_set<248, 24, Fast, true>();
        s[4][kFaithful][1] = make_set_tma<56, 24, Faithful, true, 2>();
        s[4][kFast][1] = make_set_tma<56, 24, Fast, true, 2>();
        add_split<56, 56, 2, 512, 1>(s[0][kFast][1]);
        add_split<120, 24, 2, 512, 1>(s[1][kFast][1]);
        add_split<56, 24, 2, 256, 2>(s[4][kFast][1]);
        // general (non-separable) damping: compiled for the first shape only
        s[0][kFaithful][0] = make_set_tma<56, 56, Faithful, false, 1>();
        s[0][kFast][0] = make_set_tma<56, 56, Fast, false, 1>();
    }
    int set_attrs()
    {
        if (attrs_set)
            return 0;
        int dev = 0, nsm = 0;
        OTF_CUDA(cudaGetDevice(&dev));
        OTF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        for (auto &a : s)
            for (auto &b : a)
                for (auto &k : b) {
                    if (!k.fwd)
                        continue;
                    void (*fns[3])(const StepParams) = {k.fwd, k.fwd_ring, k.rev};
                    for (auto f : fns)
                        OTF_CUDA(cudaFuncSetAttribute((const void *)f,
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                      (int)k.smem));
                    if (!k.fwd_tma)
                        continue;
                    int nb = 0;
                    void (*ft[2])(const TmaParams) = {k.fwd_tma, k.fwd_ring_tma};
                    for (auto f : ft) {
                        OTF_CUDA(cudaFuncSetAttribute((const void *)f,
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                      (int)k.smem_fwd_tma));
                        OTF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, f, NT, k.smem_fwd_tma));
                        OTF_CHECK(nb >= 1, 4, "persistent forward kernel does not fit on an SM");
                        k.grid_fwd_tma = nb * nsm;
                    }
                    OTF_CUDA(cudaFuncSetAttribute((const void *)k.rev_tma,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)k.smem_rev_tma));
                    OTF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k.rev_tma, NT, k.smem_rev_tma));
                    OTF_CHECK(nb >= 1, 4, "persistent reverse kernel does not fit on an SM");
                    k.grid_rev_tma = nb * nsm;
                    if (!k.fwd_split)
                        continue;
                    void (*fs[2])(const TmaParams) = {k.fwd_split, k.fwd_ring_split};
                    for (auto f : fs) {
                        OTF_CUDA(cudaFuncSetAttribute((const void *)f,
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                      (int)k.smem_fwd_split));
                        OTF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, f, k.nth_split,
                                                                               k.smem_fwd_split));
                        OTF_CHECK(nb >= 1, 4, "strip-split forward kernel does not fit on an SM");
                        k.grid_fwd_split = nb * nsm;
                    }
                    OTF_CUDA(cudaFuncSetAttribute((const void *)k.rev_split,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)k.smem_rev_split));
                    OTF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k.rev_split, k.nth_split,
                                                                           k.smem_rev_split));
                    OTF_CHECK(nb >= 1, 4, "strip-split reverse kernel does not fit on an SM");
                    k.grid_rev_split = nb * nsm;
                }
        attrs_set = true;
        return 0;
    }
};
static KernelTable &ktable()
{
    static KernelTable t;
    return t;
}

// Tiled tensor map over a padded [shots][rows][pitch] float array.
static int encode_map(CUtensorMap *m, const float *base, const Layout &L, int shots, int bx, int bz)
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        OTF_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        OTF_CHECK(q == cudaDriverEntryPointSuccess && p, 4, "cuTensorMapEncodeTiled is unavailable");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    cuuint64_t dims[3] = {(cuuint64_t)L.pitch, (cuuint64_t)L.rows, (cuuint64_t)shots};
    cuuint64_t strides[2] = {(cuuint64_t)L.pitch * sizeof(float), (cuuint64_t)L.slot * sizeof(float)};
    cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)bz, 1};
    cuuint32_t es[3] = {1, 1, 1};
    const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)base, dims, strides, box, es,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    OTF_CHECK(r == CUDA_SUCCESS, 4, "cuTensorMapEncodeTiled failed with code " + std::to_string((int)r));
    return 0;
}

// ----------------------------------------------------------------- Engine

Engine::~Engine() { free_all(); }

void Engine::drop_graphs()
{
    if (g_fwd_)
        cudaGraphExecDestroy(g_fwd_);
    if (g_fwd_ring_)
        cudaGraphExecDestroy(g_fwd_ring_);
    if (g_rev_)
        cudaGraphExecDestroy(g_rev_);
    g_fwd_ = g_fwd_ring_ = g_rev_ = nullptr;
    for (auto &g : g_grad_) {
        if (g)
            cudaGraphExecDestroy(g);
        g = nullptr;
    }
    for (auto &g : g_obj_) {
        if (g)
            cudaGraphExecDestroy(g);
        g = nullptr;
    }
    if (g_illum_)
        cudaGraphExecDestroy(g_illum_);
    g_illum_ = nullptr;
    illum_every_ = 0;
    graph_shots_ = -1;
}

void Engine::free_all()
{
    drop_graphs();
    if (qr_ == qf_)
        qr_ = nullptr;  // aliased when dt == dx == 1: freed once, as qf_
    float **fl[] = {&qf_, &qr_, &dampx_, &dampz_, &dampx2_, &dampz2_, &grad_, &rec_, &ring_,
                    &src_, &tab_src_, &adj_, &tab_adj_, &obs_, &gsum_, &illum_, &cq_stage_};
    for (float **p : fl) {
        if (*p)
            cudaFree(*p);
        *p = nullptr;
    }
    if (mis_)
        cudaFree(mis_);
    mis_ = nullptr;
    if (tot_)
        cudaFree(tot_);
    tot_ = nullptr;
    if (mscratch_)
        cudaFree(mscratch_);
    mscratch_ = nullptr;
    mscratch_bytes_ = 0;
    for (void *p : retired_)
        cudaFree(p);
    retired_.clear();
    for (auto &a : fld_)
        for (auto &b : a)
            for (auto &c : b) {
                if (c)
                    cudaFree(c);
                c = nullptr;
            }
    int **il[] = {&inj_src_, &inj_adj_, &tabs_};
    for (int **p : il) {
        if (*p)
            cudaFree(*p);
        *p = nullptr;
    }
    if (derr_)
        cudaFree(derr_);
    derr_ = nullptr;
    if (ledger_)
        cudaFree(ledger_);
    ledger_ = nullptr;
    if (pair_sync_)
        cudaFree(pair_sync_);
    pair_sync_ = nullptr;
    pair_sync_bytes_ = 0;
    if (ckpt_)
        cudaFree(ckpt_);
    if (seg_)
        cudaFree(seg_);
    ckpt_ = seg_ = nullptr;
    ckpt_bytes_ = seg_bytes_ = 0;
    ck_valid_ = false;
    delete tmap_;
    tmap_ = nullptr;
    maps_dirty_ = true;
    for (int k = 1; k < kMaxLanes; k++) {
        if (lane_st_[k])
            cudaStreamDestroy(lane_st_[k]);
        lane_st_[k] = nullptr;
    }
    for (auto &e : lane_ev_) {
        if (e)
            cudaEventDestroy(e);
        e = nullptr;
    }
    lane_st_[0] = nullptr;
    if (st_)
        cudaStreamDestroy(st_);
    st_ = nullptr;
    ready_ = false;
    (void)cudaGetLastError();  // no stale runtime error may leak into the next launch check
}

int Engine::init(const EngineConfig &cfg, const float *d_x, const float *d_z)
{
    free_all();
    OTF_CHECK(cfg.X >= 9 && cfg.Z >= 9, 1, "grid must be at least 9x9 cells");
    OTF_CHECK(cfg.T >= 2, 1, "T must be at least 2");
    OTF_CHECK(cfg.max_shots >= 1, 1, "max_shots must be >= 1");
    OTF_CHECK(cfg.precision == kFaithful || cfg.precision == kFast, 1, "unknown precision");
    OTF_CHECK(cfg.tile >= 0 && cfg.tile < kNumTileShapes, 1, "unknown tile shape");
    OTF_CHECK(cfg.dx != 0.f, 1, "dx must be non-zero");
    // point tables (sources, receivers, ring cells) hold 32-bit cell offsets
    // into one padded field slot
    OTF_CHECK(Layout::make(cfg.X, cfg.Z).slot <= (int64_t)INT32_MAX, 1,
              "grid too large: one padded field must stay below 2^31 cells");
    cfg_ = cfg;
    L_ = Layout::make(cfg.X, cfg.Z);
    const int X = cfg.X, Z = cfg.Z;
    if (ktable().set_attrs())
        return -1;
    OTF_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    lane_st_[0] = st_;
    for (int k = 1; k < kMaxLanes; k++)
        OTF_CUDA(cudaStreamCreateWithFlags(&lane_st_[k], cudaStreamNonBlocking));
    for (int k = 0; k < kMaxLanes; k++)
        OTF_CUDA(cudaEventCreateWithFlags(&lane_ev_[k], cudaEventDisableTiming));

    // damping multipliers 1 - d*dt at the reference's +1-shifted index
    // (d_x[z][x+1], d_z[z+1][x]: regression_PML_single.cu:505-506)
    sep_ = true;
    for (int z = 0; z < Z && sep_; z++)
        for (int x = 0; x < X; x++)
            if (d_x[(size_t)z * X + x] != d_x[x] || d_z[(size_t)z * X + x] != d_z[(size_t)z * X]) {
                sep_ = false;
                break;
            }
    const float dt = cfg.dt;
    if (sep_) {
        std::vector<float> hx(L_.pitch, 1.f), hz(L_.rows, 1.f);
        for (int x = 0; x + 1 < X; x++)
            hx[x + PAD] = std::fmaf(-d_x[x + 1], dt, 1.f);
        for (int z = 0; z + 1 < Z; z++)
            hz[z + PAD] = std::fmaf(-d_z[(size_t)(z + 1) * X], dt, 1.f);
        OTF_CUDA(cudaMalloc(&dampx_, sizeof(float) * L_.pitch));
        OTF_CUDA(cudaMalloc(&dampz_, sizeof(float) * L_.rows));
        OTF_CUDA(cudaMemcpy(dampx_, hx.data(), sizeof(float) * L_.pitch, cudaMemcpyHostToDevice));
        OTF_CUDA(cudaMemcpy(dampz_, hz.data(), sizeof(float) * L_.rows, cudaMemcpyHostToDevice));
        hdampx_ = hx;
        hdampz_ = hz;
    } else {
        std::vector<float> hx(L_.slot, 1.f), hz(L_.slot, 1.f);
        for (int z = 0; z < Z; z++)
            for (int x = 0; x < X; x++) {
                const size_t i = (size_t)z * X + x;
                if (i + 1 < (size_t)X * Z)
                    hx[L_.at(x, z)] = std::fmaf(-d_x[i + 1], dt, 1.f);
                if (z + 1 < Z)
                    hz[L_.at(x, z)] = std::fmaf(-d_z[i + X], dt, 1.f);
            }
        OTF_CUDA(cudaMalloc(&dampx2_, sizeof(float) * L_.slot));
        OTF_CUDA(cudaMalloc(&dampz2_, sizeof(float) * L_.slot));
        OTF_CUDA(cudaMemcpy(dampx2_, hx.data(), sizeof(float) * L_.slot, cudaMemcpyHostToDevice));
        OTF_CUDA(cudaMemcpy(dampz2_, hz.data(), sizeof(float) * L_.slot, cudaMemcpyHostToDevice));
        cfg_.tile = 0;  // the general-damping kernels are compiled for shape 0
    }

    two_q_ = !(cfg.dt == 1.f && cfg.dx == 1.f);
    OTF_CUDA(cudaMalloc(&qf_, sizeof(float) * L_.slot));
    OTF_CUDA(cudaMemset(qf_, 0, sizeof(float) * L_.slot));
    if (two_q_) {
        OTF_CUDA(cudaMalloc(&qr_, sizeof(float) * L_.slot));
        OTF_CUDA(cudaMemset(qr_, 0, sizeof(float) * L_.slot));
    } else {
        qr_ = qf_;
    }
    const size_t fsz = sizeof(float) * (size_t)L_.slot * cfg.max_shots;
    for (auto &a : fld_)
        for (auto &b : a)
            for (auto &c : b) {
                OTF_CUDA(cudaMalloc(&c, fsz));
                OTF_CUDA(cudaMemset(c, 0, fsz));
            }
    OTF_CUDA(cudaMalloc(&grad_, fsz));
    OTF_CUDA(cudaMemset(grad_, 0, fsz));
    OTF_CUDA(cudaMalloc(&derr_, sizeof(int)));
    OTF_CUDA(cudaMemset(derr_, 0, sizeof(int)));
    OTF_CUDA(cudaMalloc(&ledger_, sizeof(unsigned)));
    OTF_CUDA(cudaMemset(ledger_, 0, sizeof(unsigned)));
    maps_dirty_ = true;
    ready_ = true;
    return 0;
}

int Engine::set_precision(int prec)
{
    OTF_CHECK(prec == kFaithful || prec == kFast, 1, "unknown precision");
    if (prec != cfg_.precision) {
        cfg_.precision = prec;
        drop_graphs();
    }
    return 0;
}

int Engine::set_tile(int tile)
{
    OTF_CHECK(tile >= 0 && tile < kNumTileShapes, 1, "unknown tile shape");
    if (!sep_)
        tile = 0;
    if (tile != cfg_.tile) {
        cfg_.tile = tile;
        tables_dirty_ = true;
        maps_dirty_ = true;
        drop_graphs();
    }
    return 0;
}

int Engine::set_model(const float *cquad, bool on_device)
{
    OTF_CHECK(ready_, 2, "engine not initialised");
    const size_t n = (size_t)cfg_.X * cfg_.Z;
    const float *dsrc = cquad;
    if (!on_device) {
        // a persistent staging buffer: no allocation (and no pool trim) per model update
        if (!cq_stage_)
            OTF_CUDA(cudaMalloc(&cq_stage_, sizeof(float) * n));
        OTF_CUDA(cudaMemcpyAsync(cq_stage_, cquad, sizeof(float) * n, cudaMemcpyHostToDevice, st_));
        dsrc = cq_stage_;
    }
    const int bs = 256;
    const int nb = (int)((L_.slot + bs - 1) / bs);
    k_prep_q<<<nb, bs, 0, st_>>>(dsrc, qf_, two_q_ ? qr_ : nullptr, L_, cfg_.dx, cfg_.dt);
    OTF_CUDA(cudaGetLastError());
    return 0;
}

static bool inside(int x, int z, int X, int Z) { return x >= 0 && z >= 0 && x < X && z < Z; }
static bool interior(int x, int z, int X, int Z) { return x >= 4 && z >= 4 && x < X - 4 && z < Z - 4; }

int Engine::set_sources(int n, const int *x, const int *z, const float *src)
{
    OTF_CHECK(ready_, 2, "engine not initialised");
    OTF_CHECK(n >= 0, 1, "negative source count");
    for (int k = 0; k < n; k++)
        OTF_CHECK(interior(x[k], z[k], cfg_.X, cfg_.Z), 3,
                  "source " + std::to_string(k) + " at (" + std::to_string(x[k]) + "," +
                      std::to_string(z[k]) + ") is outside the updated region 4 <= x < X-4, 4 <= z < Z-4");
    src_x_.assign(x, x + n);
    src_z_.assign(z, z + n);
    n_src_ = n;
    if (src_)
        cudaFree(src_);
    if (tab_src_)
        cudaFree(tab_src_);
    src_ = tab_src_ = nullptr;
    const size_t sz = sizeof(float) * (size_t)std::max(n, 1) * cfg_.T;
    OTF_CUDA(cudaMalloc(&src_, sz));
    OTF_CUDA(cudaMalloc(&tab_src_, sz));
    OTF_CUDA(cudaMemset(tab_src_, 0, sz));
    if (n > 0) {
        OTF_CUDA(cudaMemcpyAsync(src_, src, sizeof(float) * (size_t)n * cfg_.T,
                                 cudaMemcpyHostToDevice, st_));
        k_prefix_rows<<<(n + 127) / 128, 128, 0, st_>>>(src_, tab_src_, n, cfg_.T, 0);
        OTF_CUDA(cudaGetLastError());
    }
    tables_dirty_ = true;
    drop_graphs();
    return 0;
}

int Engine::set_receivers(int n, const int *x, const int *z)
{
    OTF_CHECK(ready_, 2, "engine not initialised");
    OTF_CHECK(n >= 0, 1, "negative receiver count");
    // A receiver may sit on a never-updated cell (within 4 cells of the
    // edge): it records zeros, as in the reference, and takes no part in the
    // adjoint injection (the reference injects there into a cell no stencil reads).
    for (int k = 0; k < n; k++)
        OTF_CHECK(inside(x[k], z[k], cfg_.X, cfg_.Z), 3,
                  "receiver " + std::to_string(k) + " at (" + std::to_string(x[k]) + "," +
                      std::to_string(z[k]) + ") is outside the grid");
    rec_x_.assign(x, x + n);
    rec_z_.assign(z, z + n);
    n_rec_ = n;
    float **bufs[] = {&rec_, &adj_, &tab_adj_, &obs_};
    for (float **b : bufs) {
        if (*b)
            cudaFree(*b);
        *b = nullptr;
    }
    const size_t sz = sizeof(float) * (size_t)std::max(n, 1) * cfg_.T * cfg_.max_shots;
    for (float **b : bufs) {
        OTF_CUDA(cudaMalloc(b, sz));
        OTF_CUDA(cudaMemset(*b, 0, sz));
    }
    if (mis_)
        cudaFree(mis_);
    mis_ = nullptr;
    OTF_CUDA(cudaMalloc(&mis_, sizeof(double) * ((size_t)std::max(n, 1) * cfg_.max_shots + 1)));
    if (mscratch_)
        cudaFree(mscratch_);
    mscratch_ = nullptr;
    mscratch_bytes_ = 0;
    tables_dirty_ = true;
    drop_graphs();
    return 0;
}

int Engine::set_ring(int n, const int *x, const int *z)
{
    OTF_CHECK(ready_, 2, "engine not initialised");
    OTF_CHECK(n >= 0, 1, "negative ring size");
    for (int k = 0; k < n; k++)
        OTF_CHECK(interior(x[k], z[k], cfg_.X, cfg_.Z), 3,
                  "ring cell " + std::to_string(k) + " is outside the updated region");
    ring_x_.assign(x, x + n);
    ring_z_.assign(z, z + n);
    n_ring_ = n;
    if (ring_)
        cudaFree(ring_);
    ring_ = nullptr;
    const size_t sz = sizeof(float) * (size_t)std::max(n, 1) * cfg_.T * cfg_.max_shots;
    OTF_CUDA(cudaMalloc(&ring_, sz));
    OTF_CUDA(cudaMemset(ring_, 0, sz));
    tables_dirty_ = true;
    drop_graphs();
    return 0;
}

int Engine::set_shots(int n_shots, const int *ptr, const int *srcs)
{
    OTF_CHECK(ready_, 2, "engine not initialised");
    OTF_CHECK(n_shots >= 1 && n_shots <= cfg_.max_shots, 1, "shot count out of range");
    for (int s = 0; s < n_shots; s++)
        OTF_CHECK(ptr[s] <= ptr[s + 1], 1, "shot table not monotone");
    for (int k = ptr[0]; k < ptr[n_shots]; k++)
        OTF_CHECK(srcs[k] >= 0 && srcs[k] < n_src_, 1, "shot references an unknown source");
    // capacity of the injection table: every shot may fire every source once
    const size_t cap = (size_t)std::max(n_src_, 1) * cfg_.max_shots;
    OTF_CHECK((size_t)(ptr[n_shots] - ptr[0]) <= cap, 1, "too many source firings in the shot table");
    shot_ptr_.assign(ptr, ptr + n_shots + 1);
    for (auto &v : shot_ptr_)
        v -= ptr[0];
    shot_srcs_.assign(srcs + ptr[0], srcs + ptr[n_shots]);
    if (n_shots != n_shots_) {
        drop_graphs();
        tables_dirty_ = true;  // the adjoint injection table is sized by the shot count
    }
    n_shots_ = n_shots;

    // forward injection CSR in a fixed layout (so captured graphs stay valid
    // when only the firing pattern changes): ptr[max_shots+1] | x[cap] | z[cap] | row[cap]
    // ... | fire[max_shots][n_src]: source k's running-integral row in shot s, -1 if silent
    const size_t np = (size_t)cfg_.max_shots + 1;
    const size_t nf = (size_t)cfg_.max_shots * std::max(n_src_, 1);
    std::vector<int> h(np + 3 * cap + nf, 0);
    std::copy(shot_ptr_.begin(), shot_ptr_.end(), h.begin());
    int *hx = h.data() + np, *hz = hx + cap, *hr = hz + cap, *hf = hr + cap;
    for (size_t k = 0; k < shot_srcs_.size(); k++) {
        hx[k] = src_x_[shot_srcs_[k]];
        hz[k] = src_z_[shot_srcs_[k]];
        hr[k] = shot_srcs_[k];
    }
    std::fill(hf, hf + nf, -1);
    for (int s = 0; s < n_shots; s++)
        for (int k = shot_ptr_[s]; k < shot_ptr_[s + 1]; k++)
            hf[(size_t)s * std::max(n_src_, 1) + shot_srcs_[k]] = shot_srcs_[k];
    if (h.size() != inj_src_cap_) {
        if (inj_src_)
            cudaFree(inj_src_);
        inj_src_ = nullptr;
        OTF_CUDA(cudaMalloc(&inj_src_, sizeof(int) * h.size()));
        inj_src_cap_ = h.size();
        drop_graphs();
    }
    OTF_CUDA(cudaMemcpyAsync(inj_src_, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice, st_));
    OTF_CUDA(cudaStreamSynchronize(st_));
    inj_src_ptr_ = inj_src_;
    inj_src_x_ = inj_src_ + np;
    inj_src_z_ = inj_src_x_ + cap;
    inj_src_row_ = inj_src_z_ + cap;
    fire_row_ = inj_src_row_ + cap;
    return 0;
}

// Per-tile receiver / ring tables and the adjoint injection table; depend on
// the tile shape and the point sets.
int Engine::build_tables()
{
    const TileShape ts = kTileShapes[cfg_.tile];
    const int TX = ts.tx, TZ = ts.tz, X = cfg_.X, Z = cfg_.Z;
    const int ntx = (X + TX - 1) / TX, ntz = (Z + TZ - 1) / TZ, ntiles = ntx * ntz;
    const int EX = TX + 8;
    auto owned = [&](int x, int z, int &tile, int &cell) {
        tile = (z / TZ) * ntx + x / TX;
        cell = (z % TZ) * TX + x % TX;
    };
    std::vector<std::vector<std::pair<int, int>>> sen(ntiles), ringo(ntiles), ringe(ntiles);
    for (int n = 0; n < n_rec_; n++) {
        int tl, c;
        owned(rec_x_[n], rec_z_[n], tl, c);
        sen[tl].push_back({c, n});
    }
    for (int n = 0; n < n_ring_; n++) {
        int tl, c;
        owned(ring_x_[n], ring_z_[n], tl, c);
        ringo[tl].push_back({c, n});
    }
    std::vector<int> h;
    auto flatten = [&](std::vector<std::vector<std::pair<int, int>>> &v, bool with_id,
                       std::vector<int> &ids_out) {
        std::vector<int> ptr(ntiles + 1, 0), cell, id;
        for (int tl = 0; tl < ntiles; tl++) {
            ptr[tl + 1] = ptr[tl] + (int)v[tl].size();
            for (auto &e : v[tl]) {
                cell.push_back(e.first);
                id.push_back(e.second);
            }
        }
        const size_t off = h.size();
        h.insert(h.end(), ptr.begin(), ptr.end());
        h.insert(h.end(), cell.begin(), cell.end());
        h.push_back(0);
        if (with_id) {
            h.insert(h.end(), id.begin(), id.end());
            h.push_back(0);
        }
        ids_out = id;
        return off;
    };
    std::vector<int> sen_ids, ring_order, dummy;
    const size_t o_sen = h.size();
    flatten(sen, true, sen_ids);
    const size_t o_ringo = h.size();
    flatten(ringo, false, ring_order);
    // internal ring id of reference ring index n = its position in ring_order
    std::vector<int> ring_id(n_ring_);
    for (int e = 0; e < (int)ring_order.size(); e++)
        ring_id[ring_order[e]] = e;
    for (int n = 0; n < n_ring_; n++) {
        const int x = ring_x_[n], z = ring_z_[n];
        for (int tz = std::max(0, (z - 4) / TZ - 1); tz <= std::min(ntz - 1, (z + 4) / TZ + 1); tz++)
            for (int tx = std::max(0, (x - 4) / TX - 1); tx <= std::min(ntx - 1, (x + 4) / TX + 1); tx++) {
                const int ex = x - (tx * TX - 4), ez = z - (tz * TZ - 4);
                if (ex >= 0 && ex < EX && ez >= 0 && ez < TZ + 8)
                    ringe[tz * ntx + tx].push_back({ez * EX + ex, ring_id[n]});
            }
    }
    const size_t o_ringe = h.size();
    flatten(ringe, true, dummy);

    // points inside each tile's halo-extended region (strip-split kernels):
    // sources (the shot's firing table decides whether they fire) and the
    // receivers that take adjoint injection
    auto in_regions = [&](int x, int z, int id, std::vector<std::vector<std::pair<int, int>>> &v) {
        for (int tz = std::max(0, (z - 4) / TZ - 1); tz <= std::min(ntz - 1, (z + 4) / TZ + 1); tz++)
            for (int tx = std::max(0, (x - 4) / TX - 1); tx <= std::min(ntx - 1, (x + 4) / TX + 1); tx++) {
                const int ex = x - (tx * TX - 4), ez = z - (tz * TZ - 4);
                if (ex >= 0 && ex < EX && ez >= 0 && ez < TZ + 8)
                    v[tz * ntx + tx].push_back({ez * EX + ex, id});
            }
    };
    std::vector<std::vector<std::pair<int, int>>> srce(ntiles), rcve(ntiles);
    for (int k = 0; k < n_src_; k++)
        in_regions(src_x_[k], src_z_[k], k, srce);
    for (int n = 0; n < n_rec_; n++)
        if (interior(rec_x_[n], rec_z_[n], X, Z))
            in_regions(rec_x_[n], rec_z_[n], n, rcve);
    const size_t o_srce = h.size();
    flatten(srce, true, dummy);
    const size_t o_rcve = h.size();
    flatten(rcve, true, dummy);
    // tiles whose region holds a damped or never-updated cell
    const size_t o_edge = h.size();
    for (int tl = 0; tl < ntiles; tl++) {
        const int x0 = (tl % ntx) * TX, z0 = (tl / ntx) * TZ;
        bool edge = !sep_ || x0 - 4 < 4 || z0 - 4 < 4 || x0 + TX + 4 > X - 4 || z0 + TZ + 4 > Z - 4;
        for (int x = std::max(0, x0 - 4); !edge && x < std::min(X, x0 + TX + 4); x++)
            edge = hdampx_[x + PAD] != 1.f;
        for (int z = std::max(0, z0 - 4); !edge && z < std::min(Z, z0 + TZ + 4); z++)
            edge = hdampz_[z + PAD] != 1.f;
        h.push_back(edge ? 1 : 0);
    }

    // adjoint injection: every receiver of shot s with tab row s*n_rec + n
    const size_t o_adj = h.size();
    {
        const int ni = n_rec_ * n_shots_;
        h.reserve(h.size() + n_shots_ + 1 + 3 * (size_t)ni);
        for (int s = 0; s <= n_shots_; s++)
            h.push_back(s * n_rec_);
        for (int s = 0; s < n_shots_; s++)
            for (int n = 0; n < n_rec_; n++)  // off-grid x disables injection at edge receivers
                h.push_back(interior(rec_x_[n], rec_z_[n], X, Z) ? rec_x_[n] : -(1 << 20));
        for (int s = 0; s < n_shots_; s++)
            for (int n = 0; n < n_rec_; n++)
                h.push_back(rec_z_[n]);
        for (int s = 0; s < n_shots_; s++)
            for (int n = 0; n < n_rec_; n++)
                h.push_back(s * n_rec_ + n);
    }
    // z-streaming kernels: point lists per (padded row, strip), key = (z +
    // PAD) * n_strips + strip, column = x - (x0 - 4) within the strip's
    // computed columns; ring ids of these kernels = position in the owned
    // ring list (row-major order)
    const int NS = (X + SO - 1) / SO, NR = L_.rows, NK = NR * NS;
    struct SL {
        std::vector<std::vector<std::pair<int, int>>> v;
        size_t off = 0, n = 0;
    };
    SL s_src, s_rcv, s_sen, s_ringo, s_ringe;
    for (SL *l : {&s_src, &s_rcv, &s_sen, &s_ringo, &s_ringe})
        l->v.resize(NK);
    auto key_of = [&](int z, int s) { return (z + PAD) * NS + s; };
    auto each_strip = [&](int x, int z, int id, SL &l) {
        for (int s = std::max(0, (x - 4) / SO - 1); s <= std::min(NS - 1, (x + 4) / SO + 1); s++)
            if (x >= s * SO - 4 && x < s * SO + SO + 4)
                l.v[key_of(z, s)].push_back({x - (s * SO - 4), id});
    };
    for (int k = 0; k < n_src_; k++)
        each_strip(src_x_[k], src_z_[k], k, s_src);
    for (int n = 0; n < n_rec_; n++) {
        if (interior(rec_x_[n], rec_z_[n], X, Z))
            each_strip(rec_x_[n], rec_z_[n], n, s_rcv);
        s_sen.v[key_of(rec_z_[n], rec_x_[n] / SO)].push_back({rec_x_[n] % SO + 4, n});
    }
    for (int n = 0; n < n_ring_; n++)
        s_ringo.v[key_of(ring_z_[n], ring_x_[n] / SO)].push_back({ring_x_[n] % SO + 4, n});
    std::vector<int> ring_sid(n_ring_);
    {
        int pos = 0;
        for (auto &v : s_ringo.v)
            for (auto &e : v)
                ring_sid[e.second] = pos++;
    }
    for (int n = 0; n < n_ring_; n++)
        each_strip(ring_x_[n], ring_z_[n], ring_sid[n], s_ringe);
    for (SL *l : {&s_src, &s_rcv, &s_sen, &s_ringo, &s_ringe}) {
        std::vector<int> ptr(NK + 1, 0), col, id;
        for (int k = 0; k < NK; k++) {
            ptr[k + 1] = ptr[k] + (int)l->v[k].size();
            for (auto &e : l->v[k]) {
                col.push_back(e.first);
                id.push_back(e.second);
            }
        }
        l->off = h.size();
        l->n = col.size();
        h.insert(h.end(), ptr.begin(), ptr.end());
        h.insert(h.end(), col.begin(), col.end());
        h.push_back(0);
        h.insert(h.end(), id.begin(), id.end());
        h.push_back(0);
    }
    // unfused kernels: distinct injection cells (padded offset) with their
    // source / receiver indices in increasing order (CSR), the cells grouped
    // by the P-kernel CTA (column block cb, row segment sg; key cb + NCB *
    // sg) that owns them; the ring cells grouped the same way; padded
    // offsets of receivers and ring cells
    const int NCB = (X + kUCols - 1) / kUCols, NSEG = (Z + kURows - 1) / kURows, NC = NCB * NSEG;
    auto cta_of = [&](int x, int z) { return (z / kURows) * NCB + x / kUCols; };
    size_t o_usrc = 0, o_urcv = 0;
    int n_ucells[2] = {0, 0};
    for (int pass = 0; pass < 2; pass++) {
        std::vector<std::array<int, 4>> pts;  // (cta, offset, index)
        if (pass == 0)
            for (int k = 0; k < n_src_; k++)
                pts.push_back({cta_of(src_x_[k], src_z_[k]), (int)L_.at(src_x_[k], src_z_[k]), k, 0});
        else
            for (int n = 0; n < n_rec_; n++)
                if (interior(rec_x_[n], rec_z_[n], X, Z))
                    pts.push_back({cta_of(rec_x_[n], rec_z_[n]), (int)L_.at(rec_x_[n], rec_z_[n]), n, 0});
        std::sort(pts.begin(), pts.end());
        std::vector<int> ptr(1, 0), off, id, cta(NC + 1, 0);
        for (size_t e = 0; e < pts.size(); e++) {
            if (e == 0 || pts[e][1] != pts[e - 1][1]) {
                off.push_back(pts[e][1]);
                cta[pts[e][0] + 1]++;
                if (e > 0)
                    ptr.push_back((int)e);
            }
            id.push_back(pts[e][2]);
        }
        if (!pts.empty())
            ptr.push_back((int)pts.size());
        for (int c = 0; c < NC; c++)
            cta[c + 1] += cta[c];
        n_ucells[pass] = (int)off.size();
        (pass ? o_urcv : o_usrc) = h.size();
        h.insert(h.end(), ptr.begin(), ptr.end());
        h.insert(h.end(), off.begin(), off.end());
        h.push_back(0);
        h.insert(h.end(), id.begin(), id.end());
        h.push_back(0);
        h.insert(h.end(), cta.begin(), cta.end());
    }
    const size_t o_uring = h.size();
    {
        std::vector<std::array<int, 3>> rc;  // (cta, offset, ring index)
        for (int n = 0; n < n_ring_; n++)
            rc.push_back({cta_of(ring_x_[n], ring_z_[n]), (int)L_.at(ring_x_[n], ring_z_[n]), n});
        std::sort(rc.begin(), rc.end());
        std::vector<int> cta(NC + 1, 0);
        for (auto &e : rc)
            cta[e[0] + 1]++;
        for (int c = 0; c < NC; c++)
            cta[c + 1] += cta[c];
        h.insert(h.end(), cta.begin(), cta.end());
        for (auto &e : rc)
            h.push_back(e[1]);
        h.push_back(0);
        for (auto &e : rc)
            h.push_back(e[2]);
        h.push_back(0);
    }
    // every receiver (recording), grouped the same way: cta [NC + 1], offset,
    // receiver index
    const size_t o_urec = h.size();
    {
        std::vector<std::array<int, 3>> rc;  // (cta, offset, receiver index)
        for (int n = 0; n < n_rec_; n++)
            rc.push_back({cta_of(rec_x_[n], rec_z_[n]), (int)L_.at(rec_x_[n], rec_z_[n]), n});
        std::sort(rc.begin(), rc.end());
        std::vector<int> cta(NC + 1, 0);
        for (auto &e : rc)
            cta[e[0] + 1]++;
        for (int c = 0; c < NC; c++)
            cta[c + 1] += cta[c];
        h.insert(h.end(), cta.begin(), cta.end());
        for (auto &e : rc)
            h.push_back(e[1]);
        h.push_back(0);
        for (auto &e : rc)
            h.push_back(e[2]);
        h.push_back(0);
    }
    const size_t o_uoff = h.size();
    for (int n = 0; n < n_rec_; n++)
        h.push_back((int)L_.at(rec_x_[n], rec_z_[n]));
    for (int n = 0; n < n_ring_; n++)
        h.push_back((int)L_.at(ring_x_[n], ring_z_[n]));
    h.push_back(0);
    const size_t o_redge = h.size();
    for (int rr = 0; rr < NR; rr++) {
        const int z = rr - PAD;
        h.push_back((!sep_ || z < 4 || z >= Z - 4 || hdampz_[rr] != 1.f) ? 1 : 0);
    }
    const size_t o_sedge = h.size();
    for (int s = 0; s < NS; s++) {
        bool edge = !sep_;
        for (int x = s * SO - 4; !edge && x < s * SO + SO + 4; x++)
            edge = x < 4 || x >= X - 4 || hdampx_[x + PAD] != 1.f;
        h.push_back(edge ? 1 : 0);
    }
    // row-lag fused kernels: the ring index of every cell (padded layout, -1
    // elsewhere) and per-row CSR lists of the source cells, the injectable
    // receiver cells and every receiver. The map is read 4 cells (16 bytes)
    // at a time, so it starts on a 16-byte boundary of the table (cudaMalloc
    // aligns the table itself to 256 bytes).
    while (h.size() % 4)
        h.push_back(0);
    const size_t o_fmap = h.size();
    fused_ok_ = true;
    {
        const size_t cells = (size_t)L_.rows * L_.pitch;
        h.insert(h.end(), cells, -1);
        for (int n = 0; n < n_ring_; n++) {
            int &m = h[o_fmap + (size_t)L_.at(ring_x_[n], ring_z_[n])];
            if (m >= 0)
                fused_ok_ = false;  // a cell listed twice: one map entry cannot hold both
            m = n;
        }
    }
    auto row_cells = [&](std::vector<std::array<int, 3>> pts, size_t &o_rp, size_t &o_cx, size_t &o_ce,
                         size_t &o_id) {
        // pts: (z, x, id); cells in row order, ids increasing within a cell
        std::sort(pts.begin(), pts.end());
        std::vector<int> rp(Z + 1, 0), cx, ce(1, 0), id;
        for (size_t e = 0; e < pts.size(); e++) {
            if (e == 0 || pts[e][0] != pts[e - 1][0] || pts[e][1] != pts[e - 1][1]) {
                if (e > 0)
                    ce.push_back((int)e);
                cx.push_back(pts[e][1]);
                rp[pts[e][0] + 1]++;
            }
            id.push_back(pts[e][2]);
        }
        ce.push_back((int)pts.size());
        for (int z = 0; z < Z; z++)
            rp[z + 1] += rp[z];
        o_rp = h.size();
        h.insert(h.end(), rp.begin(), rp.end());
        o_cx = h.size();
        h.insert(h.end(), cx.begin(), cx.end());
        h.push_back(0);
        o_ce = h.size();
        h.insert(h.end(), ce.begin(), ce.end());
        o_id = h.size();
        h.insert(h.end(), id.begin(), id.end());
        h.push_back(0);
    };
    size_t f_src[4], f_rcv[4], f_rec[4];
    {
        std::vector<std::array<int, 3>> pts;
        for (int k = 0; k < n_src_; k++)
            pts.push_back({src_z_[k], src_x_[k], k});
        row_cells(pts, f_src[0], f_src[1], f_src[2], f_src[3]);
        pts.clear();
        for (int n = 0; n < n_rec_; n++)
            if (interior(rec_x_[n], rec_z_[n], X, Z))
                pts.push_back({rec_z_[n], rec_x_[n], n});
        row_cells(pts, f_rcv[0], f_rcv[1], f_rcv[2], f_rcv[3]);
        // every receiver its own entry (cells may repeat): ce is unused
        pts.clear();
        for (int n = 0; n < n_rec_; n++)
            pts.push_back({rec_z_[n], rec_x_[n], n});
        std::sort(pts.begin(), pts.end());
        std::vector<int> rp(Z + 1, 0);
        for (auto &e : pts)
            rp[e[0] + 1]++;
        for (int z = 0; z < Z; z++)
            rp[z + 1] += rp[z];
        f_rec[0] = h.size();
        h.insert(h.end(), rp.begin(), rp.end());
        f_rec[1] = h.size();
        for (auto &e : pts)
            h.push_back(e[1]);
        h.push_back(0);
        f_rec[2] = h.size();
        for (auto &e : pts)
            h.push_back(e[2]);
        h.push_back(0);
    }
    if (h.size() > tabs_cap_) {
        if (tabs_)
            cudaFree(tabs_);
        OTF_CUDA(cudaMalloc(&tabs_, sizeof(int) * h.size()));
        tabs_cap_ = h.size();
    }
    OTF_CUDA(cudaMemcpyAsync(tabs_, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice, st_));
    OTF_CUDA(cudaStreamSynchronize(st_));
    int *d = tabs_;
    sen_ptr_ = d + o_sen;
    sen_cell_ = sen_ptr_ + ntiles + 1;
    sen_id_ = sen_cell_ + n_rec_ + 1;
    ringo_ptr_ = d + o_ringo;
    ringo_cell_ = ringo_ptr_ + ntiles + 1;
    ringe_ptr_ = d + o_ringe;
    {
        int ne = 0;
        for (auto &v : ringe)
            ne += (int)v.size();
        ringe_cell_ = ringe_ptr_ + ntiles + 1;
        ringe_id_ = ringe_cell_ + ne + 1;
    }
    inj_adj_ptr_ = d + o_adj;
    inj_adj_x_ = inj_adj_ptr_ + n_shots_ + 1;
    inj_adj_z_ = inj_adj_x_ + n_rec_ * n_shots_;
    inj_adj_row_ = inj_adj_z_ + n_rec_ * n_shots_;
    srce_ptr_ = d + o_srce;
    srce_cell_ = srce_ptr_ + ntiles + 1;
    {
        int ne = 0;
        for (auto &v : srce)
            ne += (int)v.size();
        srce_id_ = srce_cell_ + ne + 1;
        ne = 0;
        for (auto &v : rcve)
            ne += (int)v.size();
        rcve_ptr_ = d + o_rcve;
        rcve_cell_ = rcve_ptr_ + ntiles + 1;
        rcve_id_ = rcve_cell_ + ne + 1;
    }
    tile_edge_ = d + o_edge;
    auto lst = [&](const SL &l, const int *&ptr, const int *&col, const int *&id) {
        ptr = d + l.off;
        col = ptr + NK + 1;
        id = col + l.n + 1;
    };
    const int *unused_id = nullptr;
    lst(s_src, stb_.src_ptr, stb_.src_col, stb_.src_id);
    lst(s_rcv, stb_.rcv_ptr, stb_.rcv_col, stb_.rcv_id);
    lst(s_sen, stb_.sen_ptr, stb_.sen_col, stb_.sen_id);
    lst(s_ringo, stb_.ring_ptr, stb_.ring_col, unused_id);
    lst(s_ringe, stb_.ringe_ptr, stb_.ringe_col, stb_.ringe_id);
    stb_.row_edge = d + o_redge;
    stb_.strip_edge = d + o_sedge;
    n_strips_ = NS;
    // CSR blocks: ptr [cells + 1] (just [0] when empty), off [cells] + 1, id + 1
    {
        // per block: ptr [cells + 1], off [cells] + 1, id [points] + 1, cta [NC + 1]
        int n_pts[2] = {0, 0};
        for (int k = 0; k < n_src_; k++)
            n_pts[0]++;
        for (int n = 0; n < n_rec_; n++)
            n_pts[1] += interior(rec_x_[n], rec_z_[n], X, Z) ? 1 : 0;
        utb_.src_ptr = d + o_usrc;
        utb_.src_off = utb_.src_ptr + n_ucells[0] + 1;
        utb_.src_id = utb_.src_off + n_ucells[0] + 1;
        utb_.src_cta = utb_.src_id + n_pts[0] + 1;
        utb_.rcv_ptr = d + o_urcv;
        utb_.rcv_off = utb_.rcv_ptr + n_ucells[1] + 1;
        utb_.rcv_id = utb_.rcv_off + n_ucells[1] + 1;
        utb_.rcv_cta = utb_.rcv_id + n_pts[1] + 1;
        utb_.ring_cta = d + o_uring;
        utb_.ring_cta_off = utb_.ring_cta + NC + 1;
        utb_.ring_cta_k = utb_.ring_cta_off + n_ring_ + 1;
    }
    utb_.n_src_cells = n_ucells[0];
    utb_.n_rcv_cells = n_ucells[1];
    utb_.rec_off = d + o_uoff;
    utb_.ring_off = utb_.rec_off + n_rec_;
    utb_.rec_cta = d + o_urec;
    utb_.rec_cta_off = utb_.rec_cta + NC + 1;
    utb_.rec_cta_id = utb_.rec_cta_off + n_rec_ + 1;
    utb_.ncb = NCB;
    utb_.nseg = NSEG;
    ftb_.ringmap = d + o_fmap;
    ftb_.src_rp = d + f_src[0];
    ftb_.src_cx = d + f_src[1];
    ftb_.src_ce = d + f_src[2];
    ftb_.src_id = d + f_src[3];
    ftb_.rcv_rp = d + f_rcv[0];
    ftb_.rcv_cx = d + f_rcv[1];
    ftb_.rcv_ce = d + f_rcv[2];
    ftb_.rcv_id = d + f_rcv[3];
    ftb_.rec_rp = d + f_rec[0];
    ftb_.rec_cx = d + f_rec[1];
    ftb_.rec_id = d + f_rec[2];
    {
        // paired kernels' counters: the tickets (one per shot, rounded up to
        // 256 bytes), then the done counts of every (shot, row segment)
        const size_t need = pair_ticket_bytes() + sizeof(unsigned) * (size_t)std::max(cfg_.max_shots, n_shots_) * NSEG;
        if (need > pair_sync_bytes_) {
            if (pair_sync_)
                cudaFree(pair_sync_);
            pair_sync_ = nullptr;
            pair_sync_bytes_ = 0;
            OTF_CUDA(cudaMalloc(&pair_sync_, need));
            pair_sync_bytes_ = need;
        }
    }
    tables_dirty_ = false;
    drop_graphs();
    return 0;
}

StepParams Engine::base_params() const
{
    const TileShape ts = kTileShapes[cfg_.tile];
    StepParams p;
    memset(&p, 0, sizeof(p));
    p.X = cfg_.X;
    p.Z = cfg_.Z;
    p.pitch = L_.pitch;
    p.rows = L_.rows;
    p.T = cfg_.T;
    p.ntx = (cfg_.X + ts.tx - 1) / ts.tx;
    p.shot_stride = L_.slot;
    p.r = cfg_.dt / cfg_.dx;
    p.dampx = dampx_;
    p.dampz = dampz_;
    p.dampx2 = dampx2_;
    p.dampz2 = dampz2_;
    p.sen_ptr = sen_ptr_;
    p.sen_cell = sen_cell_;
    p.sen_id = sen_id_;
    p.rec = rec_;
    p.n_sen = n_rec_;
    p.ringo_ptr = ringo_ptr_;
    p.ringo_cell = ringo_cell_;
    p.ringe_ptr = ringe_ptr_;
    p.ringe_cell = ringe_cell_;
    p.ringe_id = ringe_id_;
    p.ring = ring_;
    p.n_ring = n_ring_;
    p.grad = grad_;
    p.tile_edge = tile_edge_;
    p.srce_ptr = srce_ptr_;
    p.srce_cell = srce_cell_;
    p.srce_id = srce_id_;
    p.fire_row = fire_row_;
    p.n_src = std::max(n_src_, 1);
    p.rcve_ptr = rcve_ptr_;
    p.rcve_cell = rcve_cell_;
    p.rcve_id = rcve_id_;
    return p;
}

// Kernel variant actually used: the requested one where compiled for the
// tile shape and numerics, else the next simpler one (2 -> 1 -> 0). The
// strip-split kernels (2) implement the fast numerics only; -1 = automatic
// (4, the unfused kernels, for fast numerics with separable damping, else 2
// for fast, 1 for faithful).
static int resolve_variant(const KernelSet &k, int requested, int precision)
{
    int v = requested < 0 ? (precision == kFast ? 2 : 1) : requested;
    if (v == 2 && !(precision == kFast && k.fwd_split))
        v = 1;
    if (v == 1 && !k.fwd_tma)
        v = 0;
    return v;
}

int Engine::variant_in_use() const
{
    const KernelSet &k = ktable().s[cfg_.tile][cfg_.precision][sep_ ? 1 : 0];
    if (variant_ == 3 && cfg_.precision == kFast && sep_ && cfg_.X % 4 == 0)
        return 3;
    // the unfused streaming half-steps are the default of the fast numerics
    // (separable damping), measured fastest; the paired kernels (both
    // half-steps in one launch, P and A items ordered by tickets) run the same
    // device functions and are selectable (measured slower: 0.47 against
    // 0.39 ms per gradient step at 512^2 x 64 shots)
    if (variant_ == 6 && cfg_.precision == kFast && sep_ && fused_ok_)
        return 6;
    if (variant_ == 5 && cfg_.precision == kFast && sep_)
        return 5;
    if ((variant_ == 4 || variant_ < 0) && cfg_.precision == kFast && sep_)
        return 4;
    return resolve_variant(k, variant_ >= 3 ? 2 : variant_, cfg_.precision);
}

// Launch with programmatic stream serialization (programmatic dependent
// launch): the kernel may begin launching while its predecessor drains; the
// kernels synchronise on the predecessor themselves (pdl_enter). OTFWI_PDL=0
// launches them plainly.
template <class... A>
static cudaError_t launch_pdl(void (*kernel)(A...), dim3 grid, dim3 block, cudaStream_t st, A... args)
{
    static const bool use = [] {
        const char *v = getenv("OTFWI_PDL");
        return !(v && v[0] == '0');
    }();
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = use ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Unfused half-step launches (pml_step_unfused.cuh): forward P (with the
// sources) then A (with the receiver / ring recording CTAs); reverse P of
// both sets (with the ring overwrite and the adjoint sources), then A of
// both sets with the imaging condition.
UnfusedParams Engine::unfused_params(const StepParams &p, int kind) const
{
    UnfusedParams U;
    U.p = p;
    U.ncb = utb_.ncb;
    U.nseg = utb_.nseg;
    U.src_ptr = utb_.src_ptr;
    U.src_off = utb_.src_off;
    U.src_id = utb_.src_id;
    U.n_src_cells = utb_.n_src_cells;
    U.rcv_ptr = utb_.rcv_ptr;
    U.rcv_off = utb_.rcv_off;
    U.rcv_id = utb_.rcv_id;
    U.n_rcv_cells = utb_.n_rcv_cells;
    U.src_cta = utb_.src_cta;
    U.rcv_cta = utb_.rcv_cta;
    U.ring_cta = utb_.ring_cta;
    U.ring_cta_off = utb_.ring_cta_off;
    U.ring_cta_k = utb_.ring_cta_k;
    U.rec_off = utb_.rec_off;
    U.ring_off = utb_.ring_off;
    U.record_ring = kind == 1;
    U.ledger = ledger_;
    U.shot0 = ushots_ ? ushot0_ : 0;
    return U;
}

int Engine::launch_unfused(const StepParams &p, int kind)
{
    const UnfusedParams U = unfused_params(p, kind);
    // the shots of this launch: a lane's group inside a lane loop, else all
    const int ns = ushots_ ? ushots_ : n_shots_;
    const cudaStream_t st = ushots_ && ust_ ? ust_ : st_;
    const dim3 grid(U.ncb, U.nseg, ns);
    if (kind < 2) {
        OTF_CUDA(launch_pdl(k_unfused_p_fwd, grid, dim3(kUThreads), st, U));
        const int extra = n_rec_ + (kind == 1 ? n_ring_ : 0);
        const int per_row = U.ncb * kUThreads * kUTailPer;
        const int tail = (extra + per_row - 1) / per_row;
        OTF_CUDA(launch_pdl(k_unfused_a_fwd, dim3(U.ncb, U.nseg + tail, ns), dim3(kUThreads), st, U));
    } else {
        OTF_CUDA(launch_pdl(k_unfused_p_rev, dim3(U.ncb, U.nseg, 2 * ns), dim3(kUThreads), st, U));
        // A half-steps of the two sets as separate CTAs (default; measured 4.6%
        // faster on the reverse step than both sets in one CTA, which
        // OTFWI_AREV_SETS=0 selects)
        static const bool sets = [] {
            const char *v = getenv("OTFWI_AREV_SETS");
            return !(v && v[0] == '0');
        }();
        if (sets)
            OTF_CUDA(launch_pdl(k_unfused_a_rev_sets<kUARevMinBlocks>, dim3(U.ncb, U.nseg, 2 * ns), dim3(kUThreads),
                                st, U));
        else
            OTF_CUDA(launch_pdl(k_unfused_a_rev, grid, dim3(kUThreads), st, U));
    }
    OTF_CUDA(cudaGetLastError());
    return 0;
}

// Paired launches (pml_step_paired.cuh): one per step, P and A items of
// every shot handed out by tickets; register caps per direction as the
// unfused kernels (the reverse A items need their 128 registers).
constexpr int kPairFwdMinBlocks = 24;
constexpr int kPairRevMinBlocks = 16;

// Ticket scope of the paired kernels: one counter for the launch (default,
// measured faster) or one per shot (OTFWI_PAIRED_PER_SHOT=1).
static bool paired_per_shot()
{
    static const bool per_shot = [] {
        const char *v = getenv("OTFWI_PAIRED_PER_SHOT");
        return v && v[0] == '1';
    }();
    return per_shot;
}

int Engine::paired_lead(int kind) const
{
    const int ncb = utb_.ncb, nc = utb_.ncb * utb_.nseg;
    const int np = paired_per_shot() ? nc : nc * n_shots_;
    int lead = pair_lead_;
    if (lead <= 0) {
        if (paired_per_shot()) {
            // half of a shot's P items ahead of its first A item
            lead = nc / 2;
        } else {
            // about one generation of resident CTAs: the awaited P items
            // have mostly finished, their data is still in L2
            int dev = 0, nsm = 148;
            if (cudaGetDevice(&dev) == cudaSuccess)
                cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
            lead = nsm * (kind < 2 ? kPairFwdMinBlocks : kPairRevMinBlocks);
        }
    }
    return std::max(std::min(lead, np), std::min(2 * ncb, np));
}

int Engine::launch_paired(const StepParams &p, int kind)
{
    PairedParams Q;
    Q.U = unfused_params(p, kind);
    Q.ticket = reinterpret_cast<unsigned long long *>(pair_sync_);
    Q.done = reinterpret_cast<unsigned *>(reinterpret_cast<char *>(pair_sync_) + pair_ticket_bytes());
    Q.err = derr_;
    Q.n_shots = n_shots_;
    Q.lead = paired_lead(kind);
    Q.rec_cta = utb_.rec_cta;
    Q.rec_cta_off = utb_.rec_cta_off;
    Q.rec_cta_id = utb_.rec_cta_id;
    const unsigned per = 2u * (unsigned)(Q.U.ncb * Q.U.nseg);
    if (paired_per_shot()) {
        const dim3 grid(per, (unsigned)n_shots_);
        if (kind < 2)
            OTF_CUDA(launch_pdl(k_paired_fwd<kPairFwdMinBlocks, true>, grid, dim3(kUThreads), st_, Q));
        else
            OTF_CUDA(launch_pdl(k_paired_rev<kPairRevMinBlocks, true>, grid, dim3(kUThreads), st_, Q));
    } else {
        const dim3 grid(per * (unsigned)n_shots_);
        if (kind < 2)
            OTF_CUDA(launch_pdl(k_paired_fwd<kPairFwdMinBlocks, false>, grid, dim3(kUThreads), st_, Q));
        else
            OTF_CUDA(launch_pdl(k_paired_rev<kPairRevMinBlocks, false>, grid, dim3(kUThreads), st_, Q));
    }
    OTF_CUDA(cudaGetLastError());
    return 0;
}

// Row-lag fused launches (pml_step_fused.cuh): one per step, no dependency
// between CTAs; register caps from the kernels' own needs.
constexpr int kFusedFwdMinBlocks = 16;
constexpr int kFusedRevMinBlocks = 6;

int Engine::launch_fused(const StepParams &p, int kind)
{
    FusedParams F;
    F.p = p;
    F.nxb = (cfg_.X + kFInner - 1) / kFInner;
    F.chunk = fused_rows_;
    F.ringmap = ftb_.ringmap;
    F.src_rp = ftb_.src_rp;
    F.src_cx = ftb_.src_cx;
    F.src_ce = ftb_.src_ce;
    F.src_id = ftb_.src_id;
    F.rcv_rp = ftb_.rcv_rp;
    F.rcv_cx = ftb_.rcv_cx;
    F.rcv_ce = ftb_.rcv_ce;
    F.rcv_id = ftb_.rcv_id;
    F.rec_rp = ftb_.rec_rp;
    F.rec_cx = ftb_.rec_cx;
    F.rec_id = ftb_.rec_id;
    F.record_ring = kind == 1;
    const dim3 grid((unsigned)F.nxb, (unsigned)((cfg_.Z + F.chunk - 1) / F.chunk), (unsigned)n_shots_);
    if (kind < 2)
        OTF_CUDA(launch_pdl(k_fused_fwd<kFusedFwdMinBlocks>, grid, dim3(kFLanes), st_, F));
    else
        OTF_CUDA(launch_pdl(k_fused_rev<kFusedRevMinBlocks>, grid, dim3(2 * kFLanes), st_, F));
    OTF_CUDA(cudaGetLastError());
    return 0;
}

// Before a time loop of step launches: the paired kernels' tickets and done
// counts start from zero.
int Engine::begin_steps()
{
    if (variant_in_use() == 4) {
        OTF_CUDA(cudaMemsetAsync(ledger_, 0, sizeof(unsigned), st_));
        return 0;
    }
    if (variant_in_use() != 5)
        return 0;
    const size_t need = pair_ticket_bytes() + sizeof(unsigned) * (size_t)n_shots_ * utb_.nseg;
    OTF_CHECK(pair_sync_ && need <= pair_sync_bytes_, 2, "paired-kernel counters not allocated");
    OTF_CUDA(cudaMemsetAsync(pair_sync_, 0, need, st_));
    return 0;
}

// After a loop of n_steps step launches: every unfused launch counted (two
// per step), every paired ticket handed out once.
int Engine::end_steps(int n_steps, int lanes)
{
    if (n_steps <= 0)
        return 0;
    if (variant_in_use() == 4) {
        k_ledger_check<<<1, 1, 0, st_>>>(ledger_, 2u * (unsigned)n_steps * (unsigned)lanes, derr_);
        OTF_CUDA(cudaGetLastError());
        return 0;
    }
    if (variant_in_use() != 5)
        return 0;
    const bool ps = paired_per_shot();
    const unsigned long long per = 2ull * utb_.ncb * utb_.nseg * (ps ? 1 : n_shots_);
    k_paired_check<<<1, 1, 0, st_>>>(reinterpret_cast<const unsigned long long *>(pair_sync_), ps ? n_shots_ : 1,
                                     per * (unsigned long long)n_steps, derr_);
    OTF_CUDA(cudaGetLastError());
    return 0;
}

// Persistent grid of a z-streaming kernel: resident CTAs per SM x SMs.
template <class F>
static int stream_grid(F f)
{
    int dev = 0, nsm = 0, nb = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, f, SC, 0) != cudaSuccess)
        return 0;
    return nb * nsm;
}

int Engine::launch_stream(const StepParams &p, int kind)
{
    static int grid[3] = {0, 0, 0};  // forward, forward with ring, reverse
    StreamParams P;
    P.p = p;
    P.tb = stb_;
    P.n_strips = n_strips_;
    P.seg_h = seg_h_;
    P.n_segs = (cfg_.Z + seg_h_ - 1) / seg_h_;
    P.n_items = n_strips_ * P.n_segs * n_shots_;
    P.err = derr_;
    const void *fn = kind == 0 ? (const void *)k_forward_stream<false>
                   : kind == 1 ? (const void *)k_forward_stream<true> : (const void *)k_reverse_stream<3>;
    if (!grid[kind]) {
        grid[kind] = kind == 0 ? stream_grid(k_forward_stream<false>)
                   : kind == 1 ? stream_grid(k_forward_stream<true>) : stream_grid(k_reverse_stream<3>);
        OTF_CHECK(grid[kind] > 0, 4, "z-streaming kernel does not fit on an SM");
    }
    void *args[] = {(void *)&P};
    OTF_CUDA(cudaLaunchKernel(fn, dim3((unsigned)std::min(grid[kind], P.n_items)), dim3(SC), args, 0, st_));
    return 0;
}

// One forward step launch. pin / ain: slots holding P(t-1) / A(t-1).
int Engine::launch_forward_step(const StepParams &p, bool with_ring, dim3 grid, int pin, int ain)
{
    const KernelSet &k = ktable().s[cfg_.tile][cfg_.precision][sep_ ? 1 : 0];
    const int v = variant_in_use();
    if (v == 6)
        return launch_fused(p, with_ring ? 1 : 0);
    if (v == 5)
        return launch_paired(p, with_ring ? 1 : 0);
    if (v == 4)
        return launch_unfused(p, with_ring ? 1 : 0);
    if (v == 3)
        return launch_stream(p, with_ring ? 1 : 0);
    if (v >= 1) {
        TmaParams P = *tmap_;
        P.p = p;
        P.s0_p_in = pin;
        P.s0_a_in = ain;
        P.s1_in = 0;
        P.n_tiles = (int)grid.x;
        P.n_items = (int)(grid.x * grid.y);
        P.err = derr_;
        void *args[] = {(void *)&P};
        if (v == 2)
            OTF_CUDA(cudaLaunchKernel((const void *)(with_ring ? k.fwd_ring_split : k.fwd_split),
                                      dim3(std::min(k.grid_fwd_split, P.n_items)), dim3(k.nth_split),
                                      args, k.smem_fwd_split, st_));
        else
            OTF_CUDA(cudaLaunchKernel((const void *)(with_ring ? k.fwd_ring_tma : k.fwd_tma),
                                      dim3(std::min(k.grid_fwd_tma, P.n_items)), dim3(NT), args,
                                      k.smem_fwd_tma, st_));
        return 0;
    }
    void *args[] = {(void *)&p};
    OTF_CUDA(cudaLaunchKernel((const void *)(with_ring ? k.fwd_ring : k.fwd), grid, dim3(NT),
                              args, k.smem, st_));
    return 0;
}

// One reverse step launch: set 0 reads P from slot pin, A from ain; set 1 reads slot in1.
int Engine::launch_reverse_step(const StepParams &p, dim3 grid, int pin, int ain, int in1)
{
    const KernelSet &k = ktable().s[cfg_.tile][cfg_.precision][sep_ ? 1 : 0];
    const int v = variant_in_use();
    if (v == 6)
        return launch_fused(p, 2);
    if (v == 5)
        return launch_paired(p, 2);
    if (v == 4)
        return launch_unfused(p, 2);
    if (v == 3)
        return launch_stream(p, 2);
    if (v >= 1) {
        TmaParams P = *tmap_;
        P.p = p;
        P.s0_p_in = pin;
        P.s0_a_in = ain;
        P.s1_in = in1;
        P.n_tiles = (int)grid.x;
        P.n_items = (int)(grid.x * grid.y);
        P.err = derr_;
        void *args[] = {(void *)&P};
        if (v == 2)
            OTF_CUDA(cudaLaunchKernel((const void *)k.rev_split,
                                      dim3(std::min(k.grid_rev_split, P.n_items)), dim3(k.nth_split),
                                      args, k.smem_rev_split, st_));
        else
            OTF_CUDA(cudaLaunchKernel((const void *)k.rev_tma, dim3(std::min(k.grid_rev_tma, P.n_items)),
                                      dim3(NT), args, k.smem_rev_tma, st_));
        return 0;
    }
    void *args[] = {(void *)&p};
    OTF_CUDA(cudaLaunchKernel((const void *)k.rev, grid, dim3(NT), args, k.smem, st_));
    return 0;
}

// Tensor maps of every field buffer and slot (boxes of the current tile shape).
int Engine::build_maps()
{
    if (!tmap_) {
        tmap_ = new (std::nothrow) TmaParams();
        OTF_CHECK(tmap_ != nullptr, 2, "host allocation of the tensor-map block failed");
    }
    memset((void *)tmap_, 0, sizeof(TmaParams));
    const TileShape ts = kTileShapes[cfg_.tile];
    const int TX = ts.tx, TZ = ts.tz, S = cfg_.max_shots;
    SetMaps *sets[2] = {&tmap_->s0, &tmap_->s1};
    for (int s = 0; s < 2; s++)
        for (int l = 0; l < 2; l++) {
            if (encode_map(&sets[s]->px[l], fld_[s][0][l], L_, S, TX + 8, TZ + 8) ||
                encode_map(&sets[s]->pz[l], fld_[s][1][l], L_, S, TX + 8, TZ + 8) ||
                encode_map(&sets[s]->ax[l], fld_[s][2][l], L_, S, TX + 16, TZ + 8) ||
                encode_map(&sets[s]->az[l], fld_[s][3][l], L_, S, TX + 8, TZ + 16))
                return -1;
        }
    if (encode_map(&tmap_->qf, qf_, L_, 1, TX + 8, TZ + 8) ||
        encode_map(&tmap_->qr, qr_, L_, 1, TX + 8, TZ + 8) ||
        encode_map(&tmap_->grad, grad_, L_, S, TX, TZ))
        return -1;
    maps_dirty_ = false;
    return 0;
}

int Engine::set_stream_rows(int rows)
{
    OTF_CHECK(rows >= 8, 1, "stream segment rows must be >= 8");
    if (rows != seg_h_) {
        seg_h_ = rows;
        drop_graphs();
    }
    return 0;
}

int Engine::set_variant(int variant)
{
    OTF_CHECK(variant >= -1 && variant <= 6, 1, "unknown kernel variant");
    if (variant != variant_) {
        variant_ = variant;
        drop_graphs();
    }
    return 0;
}

static dim3 step_grid(const EngineConfig &c, int n_shots)
{
    const TileShape ts = kTileShapes[c.tile];
    const int ntx = (c.X + ts.tx - 1) / ts.tx, ntz = (c.Z + ts.tz - 1) / ts.tz;
    return dim3((unsigned)(ntx * ntz), (unsigned)n_shots, 1);
}

// Emit (into the stream, normally under capture) the forward time loop:
// Shot groups of the unfused time loops: one per 16 shots (up to kMaxLanes)
// unless set; other variants, and batches of fewer than 32 shots, one.
// Measured (64 shots, 512^2): four groups of 16 running as parallel chains
// fill each other's launch tails, 5-6% faster than one chain over all 64.
int Engine::lanes_in_use() const
{
    if (variant_in_use() != 4)
        return 1;
    static const int env = [] {
        const char *v = getenv("OTFWI_LANES");
        return v ? atoi(v) : 0;
    }();
    int k = lanes_req_ ? lanes_req_ : (env > 0 ? env : n_shots_ / 16);
    k = std::min(std::min(k, kMaxLanes), n_shots_);
    return k < 1 ? 1 : k;
}

// step(t) for t = 1 .. T-1 on every lane's shots: lanes > 1 fork from st_
// into parallel launch chains (lane k: shots [k n / lanes, (k + 1) n / lanes))
// and join back; the shots of each launch come from ushot0_ / ushots_.
template <class Step>
int Engine::lane_loop(int lanes, Step step)
{
    if (lanes > 1) {
        OTF_CUDA(cudaEventRecord(lane_ev_[0], st_));
        for (int k = 1; k < lanes; k++)
            OTF_CUDA(cudaStreamWaitEvent(lane_st_[k], lane_ev_[0], 0));
    }
    int rc = 0;
    for (int k = 0; k < lanes && !rc; k++) {
        const int lo = (int)((int64_t)n_shots_ * k / lanes), hi = (int)((int64_t)n_shots_ * (k + 1) / lanes);
        ust_ = lane_st_[k];
        ushot0_ = lo;
        ushots_ = lanes > 1 ? hi - lo : 0;
        for (int t = 1; t < cfg_.T && !rc; t++)
            rc = step(t);
    }
    ust_ = nullptr;
    ushot0_ = ushots_ = 0;
    if (lanes > 1) {
        for (int k = 1; k < lanes; k++) {
            OTF_CUDA(cudaEventRecord(lane_ev_[k], lane_st_[k]));
            OTF_CUDA(cudaStreamWaitEvent(st_, lane_ev_[k], 0));
        }
    }
    return rc;
}

// zero the fields, then one fused launch per step.
int Engine::emit_forward(bool with_ring, StepHook hook, void *ctx)
{
    StepParams p = base_params();
    p.q0 = qf_;
    p.q1 = qf_;
    p.inj_ptr = inj_src_ptr_;
    p.inj_x = inj_src_x_;
    p.inj_z = inj_src_z_;
    p.inj_row = inj_src_row_;
    p.inj_tab = tab_src_;
    const dim3 grid = step_grid(cfg_, n_shots_);
    const size_t fbytes = sizeof(float) * (size_t)L_.slot * n_shots_;
    for (int f = 0; f < 4; f++)
        for (int s = 0; s < 2; s++)
            OTF_CUDA(cudaMemsetAsync(fld_[0][f][s], 0, fbytes, st_));
    if (begin_steps())
        return -1;
    const int lanes = hook ? 1 : lanes_in_use();
    const int rc = lane_loop(lanes, [&](int t) -> int {
        const int i = (t - 1) & 1, o = t & 1;
        p.t = t;
        p.f0 = Fields{fld_[0][0][i], fld_[0][1][i], fld_[0][2][i], fld_[0][3][i],
                      fld_[0][0][o], fld_[0][1][o], fld_[0][2][o], fld_[0][3][o]};
        if (launch_forward_step(p, with_ring, grid, i, i))
            return -1;
        return hook && hook(ctx, t, o) ? -1 : 0;
    });
    if (rc)
        return -1;
    return end_steps(cfg_.T - 1, lanes);
}

// Emit the reverse time loop: running integral of the time-flipped adjoint
// source, zeroed adjoint fields and gradient, one fused launch per step.
int Engine::emit_reverse()
{
    const int rows = n_rec_ * n_shots_;
    if (rows > 0) {
        k_prefix_rows<<<(rows + 127) / 128, 128, 0, st_>>>(adj_, tab_adj_, rows, cfg_.T, 1);
        OTF_CUDA(cudaGetLastError());
    }
    StepParams p = base_params();
    p.q0 = qr_;
    p.q1 = qf_;
    p.inj_ptr = inj_adj_ptr_;
    p.inj_x = inj_adj_x_;
    p.inj_z = inj_adj_z_;
    p.inj_row = inj_adj_row_;
    p.inj_tab = tab_adj_;
    const dim3 grid = step_grid(cfg_, n_shots_);
    const size_t fbytes = sizeof(float) * (size_t)L_.slot * n_shots_;
    const int T = cfg_.T;
    for (int f = 0; f < 4; f++)
        for (int s = 0; s < 2; s++)
            OTF_CUDA(cudaMemsetAsync(fld_[1][f][s], 0, fbytes, st_));
    OTF_CUDA(cudaMemsetAsync(grad_, 0, fbytes, st_));
    if (begin_steps())
        return -1;
    const int lanes = lanes_in_use();
    const int rc = lane_loop(lanes, [&](int t) -> int {
        // reconstruction starts from P(T-1) (slot (T-1)%2) and A(T-2)
        // (slot (T-2)%2) (regression_PML_single.cu:787-790) and ping-pongs
        const int pi = (T + t) & 1, po = (T + t + 1) & 1;
        const int ai = (T + t + 1) & 1, ao = (T + t) & 1;
        const int i = (t - 1) & 1, o = t & 1;
        p.t = t;
        p.f0 = Fields{fld_[0][0][pi], fld_[0][1][pi], fld_[0][2][ai], fld_[0][3][ai],
                      fld_[0][0][po], fld_[0][1][po], fld_[0][2][ao], fld_[0][3][ao]};
        p.f1 = Fields{fld_[1][0][i], fld_[1][1][i], fld_[1][2][i], fld_[1][3][i],
                      fld_[1][0][o], fld_[1][1][o], fld_[1][2][o], fld_[1][3][o]};
        return launch_reverse_step(p, grid, pi, ai, i) ? -1 : 0;
    });
    if (rc)
        return -1;
    return end_steps(T - 1, lanes);
}

// Capture whatever `emit` puts on the stream into an instantiated graph.
template <class Emit>
int Engine::capture(cudaGraphExec_t *out, Emit emit)
{
    cudaGraph_t g = nullptr;
    OTF_CUDA(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
    const int rc = emit();
    const cudaError_t ec = cudaStreamEndCapture(st_, &g);
    if (rc) {
        if (g)
            cudaGraphDestroy(g);
        return rc;
    }
    OTF_CUDA(ec);
    const cudaError_t ei = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    OTF_CUDA(ei);
    return 0;
}

int Engine::prepare()
{
    OTF_CHECK(ready_, 2, "engine not initialised");
    OTF_CHECK(!shot_ptr_.empty(), 2, "no shots configured");
    if (tables_dirty_ && build_tables())
        return -1;
    if (variant_in_use() >= 1 && maps_dirty_ && build_maps())
        return -1;
    return 0;
}

int Engine::forward(bool with_ring)
{
    if (prepare())
        return -1;
    cudaGraphExec_t *g = with_ring ? &g_fwd_ring_ : &g_fwd_;
    if (!*g && capture(g, [&] { return emit_forward(with_ring); }))
        return -1;
    OTF_CUDA(cudaGraphLaunch(*g, st_));
    return 0;
}

int Engine::reverse()
{
    if (prepare())
        return -1;
    if (!g_rev_ && capture(&g_rev_, [&] { return emit_reverse(); }))
        return -1;
    OTF_CUDA(cudaGraphLaunch(g_rev_, st_));
    return 0;
}

// The whole multi-shot gradient as one graph: forward with ring recording,
// device misfit and adjoint sources, reverse phase, and the shot mean of the
// gradients into grad_mean_dev() / the misfit total into misfit_total_dev().
// Buffers the gradient graph writes outside the per-step state; allocated
// before any capture (no allocation inside a graph).
int Engine::prepare_gradient(int kind)
{
    if (prepare())
        return -1;
    OTF_CHECK(kind >= 0 && kind < kNumMisfits, 1, "unknown misfit kind");
    if (!gsum_) {
        OTF_CUDA(cudaMalloc(&gsum_, sizeof(float) * (size_t)cfg_.X * cfg_.Z));
        OTF_CUDA(cudaMalloc(&tot_, sizeof(double)));
    }
    if (kind == kMisfitQuadEnvelope && envelope_prepare(n_shots_ * n_rec_, cfg_.T))
        return -1;
    const int64_t need = misfit_scratch_per_trace(kind, cfg_.T) * n_shots_ * n_rec_;
    return grow_scratch(need);
}

// A larger misfit scratch: this engine's graphs are dropped (re-captured on
// next use) and the old buffer retired, not freed, since a multi-instance
// graph composed earlier may still reference it.
int Engine::grow_scratch(int64_t need)
{
    if (need <= mscratch_bytes_)
        return 0;
    drop_graphs();
    if (mscratch_)
        retired_.push_back(mscratch_);
    mscratch_ = nullptr;
    mscratch_bytes_ = 0;
    OTF_CUDA(cudaMalloc(&mscratch_, (size_t)need));
    mscratch_bytes_ = need;
    return 0;
}

int Engine::emit_gradient(int kind)
{
    if (emit_forward(true) || misfit(kind, tot_) || emit_reverse() || grad_sum(gsum_, 0.0f))
        return -1;
    return 0;
}

int Engine::gradient(int kind)
{
    if (prepare_gradient(kind))
        return -1;
    if (!g_grad_[kind] && capture(&g_grad_[kind], [&] { return emit_gradient(kind); }))
        return -1;
    OTF_CUDA(cudaGraphLaunch(g_grad_[kind], st_));
    return 0;
}

// Forward of every shot and the device misfit only (no ring, no reverse
// phase): the objective evaluations of a line search.
int Engine::objective(int kind)
{
    if (prepare_gradient(kind))
        return -1;
    if (!g_obj_[kind] &&
        capture(&g_obj_[kind], [&] { return (emit_forward(false) || misfit(kind, tot_)) ? -1 : 0; }))
        return -1;
    OTF_CUDA(cudaGraphLaunch(g_obj_[kind], st_));
    return 0;
}

// illum[z][x] += sum over shots of P(x, z)^2 at the current output slot.
// P is the total pressure: the split field P of the strip-split kernels, or
// Px + Pz of the others.
__global__ void k_illum(const float *__restrict__ px, const float *__restrict__ pz,
                        float *__restrict__ illum, Layout L, int n_shots, int64_t stride)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)L.X * L.Z)
        return;
    const int z = (int)(i / L.X), x = (int)(i - (int64_t)z * L.X);
    const int64_t o = L.at(x, z);
    float acc = 0.f;
    for (int s = 0; s < n_shots; s++) {
        const float v = pz ? px[o + stride * s] + pz[o + stride * s] : px[o + stride * s];
        acc = fmaf(v, v, acc);
    }
    illum[i] += acc;
}

// Source illumination: sum over shots and over every `every`-th forward step
// of P^2, into illum_dev() ([Z*X], overwritten). A diagonal pseudo-Hessian
// used to normalise gradients; one forward per call.
int Engine::illumination(int every)
{
    if (prepare())
        return -1;
    OTF_CHECK(every >= 1, 1, "illumination interval must be >= 1");
    if (!illum_)
        OTF_CUDA(cudaMalloc(&illum_, sizeof(float) * (size_t)cfg_.X * cfg_.Z));
    float *illum_dev = illum_;
    if (g_illum_ && illum_every_ != every) {
        cudaGraphExecDestroy(g_illum_);
        g_illum_ = nullptr;
    }
    const bool split = variant_in_use() >= 2;  // P total in the first field
    const int64_t n = (int64_t)cfg_.X * cfg_.Z;
    const unsigned nb = (unsigned)((n + 255) / 256);
    auto emit = [&]() -> int {
        OTF_CUDA(cudaMemsetAsync(illum_dev, 0, sizeof(float) * (size_t)n, st_));
        StepParams p = base_params();
        p.q0 = qf_;
        p.q1 = qf_;
        p.inj_ptr = inj_src_ptr_;
        p.inj_x = inj_src_x_;
        p.inj_z = inj_src_z_;
        p.inj_row = inj_src_row_;
        p.inj_tab = tab_src_;
        const dim3 grid = step_grid(cfg_, n_shots_);
        const size_t fbytes = sizeof(float) * (size_t)L_.slot * n_shots_;
        for (int f = 0; f < 4; f++)
            for (int s = 0; s < 2; s++)
                OTF_CUDA(cudaMemsetAsync(fld_[0][f][s], 0, fbytes, st_));
        if (begin_steps())
            return -1;
        for (int t = 1; t < cfg_.T; t++) {
            const int i = (t - 1) & 1, o = t & 1;
            p.t = t;
            p.f0 = Fields{fld_[0][0][i], fld_[0][1][i], fld_[0][2][i], fld_[0][3][i],
                          fld_[0][0][o], fld_[0][1][o], fld_[0][2][o], fld_[0][3][o]};
            if (launch_forward_step(p, false, grid, i, i))
                return -1;
            if (t % every == 0) {
                k_illum<<<nb, 256, 0, st_>>>(fld_[0][0][o], split ? nullptr : fld_[0][1][o], illum_dev, L_,
                                             n_shots_, L_.slot);
                OTF_CUDA(cudaGetLastError());
            }
        }
        return end_steps(cfg_.T - 1);
    };
    if (!g_illum_ && capture(&g_illum_, emit))
        return -1;
    illum_every_ = every;
    OTF_CUDA(cudaGraphLaunch(g_illum_, st_));
    return 0;
}

int Engine::gradient_graph(int kind, cudaGraph_t *out)
{
    *out = nullptr;
    if (prepare_gradient(kind))
        return -1;
    OTF_CUDA(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
    const int rc = emit_gradient(kind);
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(st_, &g);
    if (rc) {
        if (g)
            cudaGraphDestroy(g);
        return rc;
    }
    OTF_CUDA(ec);
    *out = g;
    return 0;
}

int Engine::copy_traces(float *dst, int shot0, int n, cudaMemcpyKind kind)
{
    const size_t per = (size_t)n_rec_ * cfg_.T;
    OTF_CUDA(cudaMemcpyAsync(dst, rec_ + per * shot0, sizeof(float) * per * n, kind, st_));
    return 0;
}

int Engine::copy_grad_shot(int shot, float *dst, cudaMemcpyKind kind)
{
    const float *src = grad_ + L_.slot * shot + L_.at(0, 0);
    OTF_CUDA(cudaMemcpy2DAsync(dst, sizeof(float) * cfg_.X, src, sizeof(float) * L_.pitch,
                               sizeof(float) * cfg_.X, cfg_.Z, kind, st_));
    return 0;
}

int Engine::grad_sum(float *dst, float scale)
{
    const int64_t n = (int64_t)cfg_.X * cfg_.Z;
    k_grad_sum<<<(unsigned)((n + 255) / 256), 256, 0, st_>>>(grad_, dst, L_, n_shots_, L_.slot, scale);
    OTF_CUDA(cudaGetLastError());
    return 0;
}

int Engine::sync()
{
    OTF_CUDA(cudaStreamSynchronize(st_));
    if (derr_) {
        int h = 0;
        OTF_CUDA(cudaMemcpy(&h, derr_, sizeof(int), cudaMemcpyDeviceToHost));
        if (h) {
            OTF_CUDA(cudaMemset(derr_, 0, sizeof(int)));
            std::string m;
            if (h & kErrWaitTimeout)
                m += "a bounded wait for tensor-memory copies timed out in a step kernel; ";
            if (h & kErrDepTimeout)
                m += "a paired step kernel's wait for the P half-step of its neighbour rows timed out; ";
            if (h & kErrTicketRange)
                m += "paired step launches ran out of order or not at all (work tickets out of range); ";
            if (h & kErrLedger)
                m += "step launches of a time loop did not all run (launch count short); ";
            OTF_CHECK(false, 5, m + "results of this call are invalid");
        }
    }
    return 0;
}

int Engine::set_observed(const float *obs, cudaMemcpyKind kind)
{
    OTF_CHECK(ready_ && obs_, 2, "receivers not configured");
    const size_t n = (size_t)n_shots_ * n_rec_ * cfg_.T;
    OTF_CUDA(cudaMemcpyAsync(obs_, obs, sizeof(float) * n, kind, st_));
    return 0;
}

// Sum of the per-trace misfits in trace order (FP64), one thread.
__global__ void k_sum_misfit(const double *__restrict__ m, int n, double *__restrict__ out)
{
    double s = 0.0;
    for (int i = 0; i < n; i++)
        s += m[i];
    *out = s;
}

int Engine::misfit(int kind, double *total_dev)
{
    OTF_CHECK(ready_ && obs_, 2, "receivers not configured");
    const int n = n_shots_ * n_rec_;
    // inside a capture the gradient / objective preparation has sized it
    if (grow_scratch(misfit_scratch_per_trace(kind, cfg_.T) * n))
        return -1;
    if (launch_misfit(kind, rec_, obs_, adj_, mis_, n, cfg_.T, mscratch_, mscratch_bytes_, st_))
        return -1;
    if (total_dev) {
        k_sum_misfit<<<1, 1, 0, st_>>>(mis_, n, total_dev);
        OTF_CUDA(cudaGetLastError());
    }
    return 0;
}

}  // namespace otf

namespace {
__global__ void k_selftest_wait(const unsigned *cnt, int *err)
{
    if (threadIdx.x == 0)
        otf::wait_geq(cnt, 1u, err);
}
}  // namespace

extern "C" int otf_selftest_paired_faults(int *bits)
{
    otf::clear_error();
    OTF_CHECK(bits != nullptr, 1, "otf_selftest_paired_faults: bits is null");
    *bits = 0;
    void *buf = nullptr;
    cudaStream_t st = nullptr;
    int rc = -1, h = 0;
    if (cudaMalloc(&buf, 256) == cudaSuccess && cudaMemset(buf, 0, 256) == cudaSuccess &&
        cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess) {
        unsigned *cnt = reinterpret_cast<unsigned *>(buf);
        int *err = reinterpret_cast<int *>(reinterpret_cast<char *>(buf) + 128);
        auto *ticket = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(buf) + 64);
        k_selftest_wait<<<1, 32, 0, st>>>(cnt, err);
        otf::k_paired_check<<<1, 1, 0, st>>>(ticket, 1, 1ull, err);
        // a time loop of one step whose two unfused launches were never counted
        otf::k_ledger_check<<<1, 1, 0, st>>>(reinterpret_cast<unsigned *>(reinterpret_cast<char *>(buf) + 32), 2u,
                                              err);
        if (cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(st) == cudaSuccess &&
            cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess) {
            *bits = h;
            rc = (h & otf::kErrDepTimeout) && (h & otf::kErrTicketRange) && (h & otf::kErrLedger) ? 0 : -1;
            if (rc)
                otf::set_error_msg(5, "otf_selftest_paired_faults: a fault path was not reported");
        } else {
            otf::set_error_msg(5, "otf_selftest_paired_faults: CUDA call failed");
        }
    } else {
        otf::set_error_msg(3, "otf_selftest_paired_faults: set-up failed");
    }
    if (st)
        cudaStreamDestroy(st);
    if (buf)
        cudaFree(buf);
    return rc;
}
