// Batched C ABI: every shot of a full-matrix capture (or any shot table)
// advanced together by the fused step kernels, with the misfit and adjoint
// sources computed on the device and the whole gradient replayed as one CUDA
// graph. No reference counterpart: the reference runs one shot per
// cuda_grad_ext call from a Python loop (cuda_interface_pml.py:225-236) with
// the misfit on the host (adjoint_functions.py).
#include <cuda_runtime.h>
#include <memory>
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

int otf_batch_sync(otf_batch *b) { return b->eng.sync(); }

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
