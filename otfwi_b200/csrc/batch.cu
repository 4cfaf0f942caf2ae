// Batched C ABI: every shot of a full-matrix capture (or any shot table)
// advanced together by the fused step kernels, with the misfit and adjoint
// sources computed on the device and the whole gradient replayed as one CUDA
// graph. No reference counterpart: the reference runs one shot per
// cuda_grad_ext call from a Python loop (cuda_interface_pml.py:225-236) with
// the misfit on the host (adjoint_functions.py).
#include <cuda_runtime.h>
#include <memory>
#include <vector>
#include <cstring>
#include "engine.h"
#include "misfit.h"
#include "../../include/otfwi.h"

struct otf_batch {
    otf::Engine eng;
};

namespace {
cudaMemcpyKind kind_in(int on_device) { return on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice; }
cudaMemcpyKind kind_out(int on_device) { return on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost; }
}  // namespace

extern "C" {

otf_batch *otf_batch_create(int X, int Z, int T, const float *constvec, const float *d_x,
                            const float *d_z, int n_src, const int *src_x, const int *src_z,
                            const float *source, int n_rec, const int *rec_x, const int *rec_z,
                            int n_ring, const int *ring_x, const int *ring_z, int max_shots,
                            int precision, int tile)
{
    otf::clear_error();
    std::unique_ptr<otf_batch> b(new otf_batch());
    otf::EngineConfig cfg;
    cfg.X = X;
    cfg.Z = Z;
    cfg.T = T;
    cfg.dx = constvec[0];
    cfg.dz = constvec[1];
    cfg.dt = constvec[2];
    cfg.max_shots = max_shots;
    cfg.precision = precision;
    cfg.tile = tile;
    if (b->eng.init(cfg, d_x, d_z) || b->eng.set_sources(n_src, src_x, src_z, source) ||
        b->eng.set_receivers(n_rec, rec_x, rec_z) || b->eng.set_ring(n_ring, ring_x, ring_z))
        return nullptr;
    return b.release();
}

void otf_batch_destroy(otf_batch *b) { delete b; }

int otf_batch_set_shots(otf_batch *b, int n_shots, const int *ptr, const int *srcs)
{
    return b->eng.set_shots(n_shots, ptr, srcs);
}

int otf_batch_set_model(otf_batch *b, const float *cquad, int on_device)
{
    return b->eng.set_model(cquad, on_device != 0);
}

int otf_batch_set_observed(otf_batch *b, const float *obs, int on_device)
{
    return b->eng.set_observed(obs, kind_in(on_device));
}

int otf_batch_set_precision(otf_batch *b, int precision) { return b->eng.set_precision(precision); }
int otf_batch_set_tile(otf_batch *b, int tile) { return b->eng.set_tile(tile); }
int otf_batch_set_kernel(otf_batch *b, int variant) { return b->eng.set_variant(variant); }
int otf_batch_set_stream_rows(otf_batch *b, int rows) { return b->eng.set_stream_rows(rows); }
int otf_batch_set_lanes(otf_batch *b, int lanes)
{
    OTF_CHECK(b && lanes >= 0, 1, "otf_batch_set_lanes: bad arguments");
    b->eng.set_lanes(lanes);
    return 0;
}

int otf_batch_lanes(otf_batch *b) { return b ? b->eng.lanes_in_use() : -1; }

int otf_batch_set_fused_rows(otf_batch *b, int rows)
{
    OTF_CHECK(rows >= 8, 1, "fused rows per chunk must be >= 8");
    b->eng.set_fused_rows(rows);
    return 0;
}

int otf_batch_set_paired_lead(otf_batch *b, int lead)
{
    OTF_CHECK(lead >= 0, 1, "paired lead must be >= 0");
    b->eng.set_paired_lead(lead);
    return 0;
}

int otf_batch_forward(otf_batch *b, float *traces, int on_device)
{
    if (b->eng.forward(false))
        return -1;
    if (traces && b->eng.copy_traces(traces, 0, b->eng.n_shots(), kind_out(on_device)))
        return -1;
    return 0;
}

int otf_batch_gradient(otf_batch *b, int misfit_kind, float *grad, double *misfit, int on_device)
{
    if (b->eng.gradient(misfit_kind))
        return -1;
    const otf::EngineConfig &c = b->eng.config();
    if (grad)
        OTF_CUDA(cudaMemcpyAsync(grad, b->eng.grad_mean_dev(), sizeof(float) * (size_t)c.X * c.Z,
                                 kind_out(on_device), b->eng.stream()));
    if (misfit)
        OTF_CUDA(cudaMemcpyAsync(misfit, b->eng.misfit_total_dev(), sizeof(double),
                                 kind_out(on_device), b->eng.stream()));
    return 0;
}

int otf_batch_forward_ring(otf_batch *b, float *traces, int on_device)
{
    if (b->eng.forward(true))
        return -1;
    if (traces && b->eng.copy_traces(traces, 0, b->eng.n_shots(), kind_out(on_device)))
        return -1;
    return 0;
}

int otf_batch_reverse(otf_batch *b, const float *adj, int on_device, float *grad, float scale,
                      int grad_on_device)
{
    const otf::EngineConfig &c = b->eng.config();
    const size_t n = (size_t)b->eng.n_shots() * b->eng.n_rec() * c.T;
    if (adj)
        OTF_CUDA(cudaMemcpyAsync(b->eng.adj_dev(), adj, sizeof(float) * n, kind_in(on_device),
                                 b->eng.stream()));
    if (b->eng.reverse())
        return -1;
    if (grad) {
        if (grad_on_device)
            return b->eng.grad_sum(grad, scale);
        float *tmp = nullptr;
        OTF_CUDA(cudaMallocAsync(&tmp, sizeof(float) * (size_t)c.X * c.Z, b->eng.stream()));
        if (b->eng.grad_sum(tmp, scale))
            return -1;
        OTF_CUDA(cudaMemcpyAsync(grad, tmp, sizeof(float) * (size_t)c.X * c.Z,
                                 cudaMemcpyDeviceToHost, b->eng.stream()));
        OTF_CUDA(cudaFreeAsync(tmp, b->eng.stream()));
    }
    return 0;
}

int otf_batch_shot_grad(otf_batch *b, int shot, float *grad, int on_device)
{
    return b->eng.copy_grad_shot(shot, grad, kind_out(on_device));
}

int otf_batch_misfit(otf_batch *b, int misfit_kind, double *per_trace, int on_device)
{
    if (b->eng.misfit(misfit_kind, nullptr))
        return -1;
    if (per_trace)
        OTF_CUDA(cudaMemcpyAsync(per_trace, b->eng.misfit_dev(),
                                 sizeof(double) * (size_t)b->eng.n_shots() * b->eng.n_rec(),
                                 kind_out(on_device), b->eng.stream()));
    return 0;
}

int otf_batch_adjoint(otf_batch *b, float *adj, int on_device)
{
    const size_t n = (size_t)b->eng.n_shots() * b->eng.n_rec() * b->eng.config().T;
    OTF_CUDA(cudaMemcpyAsync(adj, b->eng.adj_dev(), sizeof(float) * n, kind_out(on_device),
                             b->eng.stream()));
    return 0;
}

int otf_batch_forward_ckpt(otf_batch *b, int every, float *traces, int on_device)
{
    if (b->eng.forward_checkpointed(every))
        return -1;
    if (traces && b->eng.copy_traces(traces, 0, b->eng.n_shots(), kind_out(on_device)))
        return -1;
    return 0;
}

int otf_batch_backward_exact(otf_batch *b, const float *g, int g_on_device, float *grad_c2,
                             int grad_on_device)
{
    const otf::EngineConfig &c = b->eng.config();
    const size_t ng = (size_t)b->eng.n_shots() * b->eng.n_rec() * c.T, nz = (size_t)c.X * c.Z;
    float *gd = const_cast<float *>(g), *out = grad_c2;
    cudaStream_t st = b->eng.stream();
    if (!g_on_device) {
        OTF_CUDA(cudaMallocAsync(&gd, sizeof(float) * ng, st));
        OTF_CUDA(cudaMemcpyAsync(gd, g, sizeof(float) * ng, cudaMemcpyHostToDevice, st));
    }
    if (!grad_on_device)
        OTF_CUDA(cudaMallocAsync(&out, sizeof(float) * nz, st));
    const int rc = b->eng.backward_exact(gd, out);
    if (!rc && !grad_on_device)
        OTF_CUDA(cudaMemcpyAsync(grad_c2, out, sizeof(float) * nz, cudaMemcpyDeviceToHost, st));
    if (!g_on_device)
        cudaFreeAsync(gd, st);
    if (!grad_on_device)
        cudaFreeAsync(out, st);
    return rc;
}

int otf_batch_sync(otf_batch *b) { return b->eng.sync(); }

int otf_batch_objective(otf_batch *b, int misfit_kind, double *misfit, int on_device)
{
    if (b->eng.objective(misfit_kind))
        return -1;
    if (misfit)
        OTF_CUDA(cudaMemcpyAsync(misfit, b->eng.misfit_total_dev(), sizeof(double), kind_out(on_device),
                                 b->eng.stream()));
    return 0;
}

int otf_batch_illumination(otf_batch *b, int every, float *illum, int on_device)
{
    if (b->eng.illumination(every))
        return -1;
    const otf::EngineConfig &c = b->eng.config();
    if (illum)
        OTF_CUDA(cudaMemcpyAsync(illum, b->eng.illum_dev(), sizeof(float) * (size_t)c.X * c.Z,
                                 kind_out(on_device), b->eng.stream()));
    return 0;
}

namespace {
struct FrameCopy {
    unsigned char *dst;
    size_t frame_bytes;
};
int copy_frames(void *ctx, const unsigned char *frames, int n)
{
    FrameCopy &c = *static_cast<FrameCopy *>(ctx);
    memcpy(c.dst, frames, (size_t)n * c.frame_bytes);
    c.dst += (size_t)n * c.frame_bytes;
    return 0;
}
}  // namespace

int otf_batch_frames(otf_batch *b, int every, int shot, unsigned char *frames)
{
    OTF_CHECK(frames != nullptr, 1, "otf_batch_frames: no output buffer");
    const otf::EngineConfig &c = b->eng.config();
    FrameCopy fc{frames, (size_t)c.X * c.Z};
    return b->eng.frames(every, shot, copy_frames, &fc);
}

int otf_batch_last_gradient(otf_batch *b, float *grad, double *misfit, int on_device)
{
    const otf::EngineConfig &c = b->eng.config();
    OTF_CHECK(b->eng.grad_mean_dev() != nullptr, 2, "no gradient has been computed on this batch");
    if (grad)
        OTF_CUDA(cudaMemcpyAsync(grad, b->eng.grad_mean_dev(), sizeof(float) * (size_t)c.X * c.Z,
                                 kind_out(on_device), b->eng.stream()));
    if (misfit)
        OTF_CUDA(cudaMemcpyAsync(misfit, b->eng.misfit_total_dev(), sizeof(double), kind_out(on_device),
                                 b->eng.stream()));
    return 0;
}

}  // extern "C"

// Several independent inversions (different grids, shot counts and T) in one
// CUDA graph: each instance's complete gradient graph is a parallel branch,
// so one launch runs them all and the GPU fills its SMs from every branch.
struct otf_multi {
    std::vector<otf_batch *> b;
    int chains = 0;  // > 0: instance i runs after instance i - chains (that many branches at once)
    cudaStream_t st = nullptr;
    cudaGraphExec_t exec[otf::kNumMisfits] = {};
    ~otf_multi()
    {
        for (auto &e : exec)
            if (e)
                cudaGraphExecDestroy(e);
        if (st)
            cudaStreamDestroy(st);
    }
};

extern "C" {

otf_multi *otf_multi_create(int n, otf_batch **batches)
{
    otf::clear_error();
    if (n < 1 || !batches) {
        otf::set_error_msg(1, "otf_multi_create: no instances");
        return nullptr;
    }
    std::unique_ptr<otf_multi> m(new otf_multi());
    m->b.assign(batches, batches + n);
    if (cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking) != cudaSuccess) {
        otf::set_error_msg(2, "otf_multi_create: stream creation failed");
        return nullptr;
    }
    return m.release();
}

void otf_multi_destroy(otf_multi *m) { delete m; }

int otf_multi_set_chains(otf_multi *m, int chains)
{
    OTF_CHECK(m && chains >= 0, 1, "otf_multi_set_chains: bad arguments");
    if (chains != m->chains)
        for (auto &e : m->exec)
            if (e) {
                cudaGraphExecDestroy(e);
                e = nullptr;
            }
    m->chains = chains;
    return 0;
}

int otf_multi_gradient(otf_multi *m, int misfit_kind)
{
    OTF_CHECK(misfit_kind >= 0 && misfit_kind < otf::kNumMisfits, 1, "unknown misfit kind");
    if (!m->exec[misfit_kind]) {
        cudaGraph_t parent = nullptr;
        OTF_CUDA(cudaGraphCreate(&parent, 0));
        std::vector<cudaGraphNode_t> nodes;
        for (otf_batch *b : m->b) {
            cudaGraph_t child = nullptr;
            if (b->eng.gradient_graph(misfit_kind, &child)) {
                cudaGraphDestroy(parent);
                return -1;
            }
            cudaGraphNode_t node;
            const size_t i = nodes.size();
            const bool dep = m->chains > 0 && i >= (size_t)m->chains;
            const cudaError_t e =
                cudaGraphAddChildGraphNode(&node, parent, dep ? &nodes[i - m->chains] : nullptr, dep ? 1 : 0, child);
            nodes.push_back(node);
            cudaGraphDestroy(child);
            if (e != cudaSuccess) {
                cudaGraphDestroy(parent);
                OTF_CUDA(e);
            }
        }
        const cudaError_t ei = cudaGraphInstantiate(&m->exec[misfit_kind], parent, 0);
        cudaGraphDestroy(parent);
        OTF_CUDA(ei);
    }
    // every instance's own stream work (model / observed uploads) precedes the launch
    for (otf_batch *b : m->b)
        if (b->eng.sync())
            return -1;
    OTF_CUDA(cudaGraphLaunch(m->exec[misfit_kind], m->st));
    return 0;
}

int otf_multi_sync(otf_multi *m)
{
    OTF_CUDA(cudaStreamSynchronize(m->st));
    for (otf_batch *b : m->b)
        if (b->eng.sync())  // surfaces a device-side wait timeout of any instance
            return -1;
    return 0;
}

void *otf_batch_stream(otf_batch *b) { return (void *)b->eng.stream(); }

long long otf_misfit_scratch_bytes(int kind, int n_traces, int T)
{
    return otf::misfit_scratch_per_trace(kind, T) * n_traces;
}

int otf_misfit(int kind, const float *sim, const float *obs, float *adj, double *misfit,
               int n_traces, int T, void *scratch, long long scratch_bytes, void *stream)
{
    return otf::launch_misfit(kind, sim, obs, adj, misfit, n_traces, T, scratch, scratch_bytes,
                              (cudaStream_t)stream);
}

}  // extern "C"
