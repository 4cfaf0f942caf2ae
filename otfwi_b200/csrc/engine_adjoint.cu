// Differentiable path of the engine: checkpointed forward and the exact
// discrete adjoint with segment recompute (sqrt(T) memory in time).
//
// Memory: the full state (Px, Pz, Ax, Az) of every shot at t = 0, k, 2k, ...
// (k = checkpoint interval) plus the A history of one segment (k steps),
// i.e. about (T/k + 2k/4) field-states per shot instead of T; k = sqrt(T)
// minimises it. Each segment's forward is recomputed once from its
// checkpoint, so the backward costs one extra forward in total.
#include <algorithm>
#include <cmath>
#include <cstring>
#include "engine.h"
#include "pml_adjoint.cuh"

namespace otf {

namespace {
constexpr int ATX = 56, ATZ = 24, ABH = 2;  // tile of the adjoint step kernel
using AG = AdjGeom<ATX, ATZ, ABH>;
bool g_adj_attr = false;
}  // namespace

int Engine::forward_checkpointed(int every)
{
    if (prepare())
        return -1;
    OTF_CHECK(every >= 1, 1, "checkpoint interval must be >= 1");
    OTF_CHECK(sep_, 1, "the differentiable path needs separable damping");
    const int T = cfg_.T;
    const int n_seg = (T - 1 + every - 1) / every;
    const size_t field = sizeof(float) * (size_t)L_.slot * cfg_.max_shots;
    const size_t need_ck = field * 4 * n_seg, need_seg = field * 2 * every;
    if (need_ck > ckpt_bytes_) {
        if (ckpt_)
            OTF_CUDA(cudaFree(ckpt_));
        ckpt_ = nullptr;
        ckpt_bytes_ = 0;
        OTF_CUDA(cudaMalloc(&ckpt_, need_ck));
        ckpt_bytes_ = need_ck;
    }
    if (need_seg > seg_bytes_) {
        if (seg_)
            OTF_CUDA(cudaFree(seg_));
        seg_ = nullptr;
        seg_bytes_ = 0;
        OTF_CUDA(cudaMalloc(&seg_, need_seg));
        seg_bytes_ = need_seg;
    }
    ck_every_ = every;
    n_ck_ = n_seg;
    // the checkpoints hold split-field states: the strip-split kernels (a
    // different state layout) are not used on this path
    const int saved = variant_;
    variant_ = std::min(variant_in_use(), 1);
    if (variant_ == 1 && maps_dirty_ && build_maps()) {
        variant_ = saved;
        return -1;
    }
    StepParams p = base_params();
    p.q0 = qf_;
    p.q1 = qf_;
    p.inj_ptr = inj_src_ptr_;
    p.inj_x = inj_src_x_;
    p.inj_z = inj_src_z_;
    p.inj_row = inj_src_row_;
    p.inj_tab = tab_src_;
    const TileShape ts = kTileShapes[cfg_.tile];
    const dim3 grid((unsigned)(((cfg_.X + ts.tx - 1) / ts.tx) * ((cfg_.Z + ts.tz - 1) / ts.tz)),
                    (unsigned)n_shots_);
    const size_t fb = sizeof(float) * (size_t)L_.slot * n_shots_;
    int rc = 0;
    for (int f = 0; f < 4 && !rc; f++)
        for (int s = 0; s < 2 && !rc; s++)
            if (cudaMemsetAsync(fld_[0][f][s], 0, fb, st_) != cudaSuccess)
                rc = -1;
    for (int f = 0; f < 4 && !rc; f++)  // checkpoint 0: the state at rest
        if (cudaMemsetAsync(ckpt_ + (size_t)f * L_.slot * cfg_.max_shots, 0, fb, st_) != cudaSuccess)
            rc = -1;
    for (int t = 1; t < T && !rc; t++) {
        const int i = (t - 1) & 1, o = t & 1;
        p.t = t;
        p.f0 = Fields{fld_[0][0][i], fld_[0][1][i], fld_[0][2][i], fld_[0][3][i],
                      fld_[0][0][o], fld_[0][1][o], fld_[0][2][o], fld_[0][3][o]};
        rc = launch_forward_step(p, false, grid, i, i);
        if (!rc && t % every == 0 && t / every < n_seg) {
            float *ck = ckpt_ + (size_t)(t / every) * 4 * L_.slot * cfg_.max_shots;
            for (int f = 0; f < 4 && !rc; f++)
                if (cudaMemcpyAsync(ck + (size_t)f * L_.slot * cfg_.max_shots, fld_[0][f][o], fb,
                                    cudaMemcpyDeviceToDevice, st_) != cudaSuccess)
                    rc = -1;
        }
    }
    variant_ = saved;
    if (rc) {
        OTF_CHECK(otf::last_status() != 0, 2, "checkpointed forward failed to launch");
        return -1;
    }
    ck_valid_ = true;
    return 0;
}

int Engine::backward_exact(const float *g_dev, float *grad_c2_dev)
{
    OTF_CHECK(ck_valid_, 2, "backward_exact needs a preceding forward_checkpointed");
    if (prepare())
        return -1;
    if (!g_adj_attr) {
        OTF_CUDA(cudaFuncSetAttribute((const void *)k_adjoint_step<ATX, ATZ, ABH>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(sizeof(float) * AG::FLOATS)));
        g_adj_attr = true;
    }
    const int T = cfg_.T, every = ck_every_;
    const size_t fs = (size_t)L_.slot * cfg_.max_shots;  // floats per field buffer
    const size_t fb = sizeof(float) * (size_t)L_.slot * n_shots_;
    const int saved = variant_;
    variant_ = std::min(variant_in_use(), 1);
    if (variant_ == 1 && maps_dirty_ && build_maps()) {
        variant_ = saved;
        return -1;
    }
    StepParams p = base_params();
    p.q0 = qf_;
    p.q1 = qf_;
    p.inj_ptr = inj_src_ptr_;
    p.inj_x = inj_src_x_;
    p.inj_z = inj_src_z_;
    p.inj_row = inj_src_row_;
    p.inj_tab = tab_src_;
    const TileShape ts = kTileShapes[cfg_.tile];
    const dim3 grid((unsigned)(((cfg_.X + ts.tx - 1) / ts.tx) * ((cfg_.Z + ts.tz - 1) / ts.tz)),
                    (unsigned)n_shots_);
    AdjParams a;
    memset(&a, 0, sizeof(a));
    a.X = cfg_.X;
    a.Z = cfg_.Z;
    a.pitch = L_.pitch;
    a.rows = L_.rows;
    a.T = T;
    a.ntx = (cfg_.X + ATX - 1) / ATX;
    a.n_rec = n_rec_;
    a.shot_stride = L_.slot;
    a.r = cfg_.dt / cfg_.dx;
    a.q = qf_;
    a.dampx = dampx_;
    a.dampz = dampz_;
    a.g = g_dev;
    a.rcve_ptr = nullptr;
    a.grad_q = grad_;
    const dim3 agrid((unsigned)(a.ntx * ((cfg_.Z + ATZ - 1) / ATZ)), (unsigned)n_shots_);
    // receivers per adjoint tile (the engine's own tables are built for the step tile shape)
    {
        const int ntx = a.ntx, ntz = (cfg_.Z + ATZ - 1) / ATZ, nt = ntx * ntz, EX = ATX + 8;
        std::vector<std::vector<std::pair<int, int>>> v(nt);
        for (int n = 0; n < n_rec_; n++) {
            const int x = rec_x_[n], z = rec_z_[n];
            if (!(x >= 4 && z >= 4 && x < cfg_.X - 4 && z < cfg_.Z - 4))
                continue;
            for (int tz = std::max(0, (z - 4) / ATZ - 1); tz <= std::min(ntz - 1, (z + 4) / ATZ + 1); tz++)
                for (int tx = std::max(0, (x - 4) / ATX - 1); tx <= std::min(ntx - 1, (x + 4) / ATX + 1); tx++) {
                    const int ex = x - (tx * ATX - 4), ez = z - (tz * ATZ - 4);
                    if (ex >= 0 && ex < EX && ez >= 0 && ez < ATZ + 8)
                        v[tz * ntx + tx].push_back({ez * EX + ex, n});
                }
        }
        std::vector<int> h(nt + 1, 0), cell, id;
        for (int i = 0; i < nt; i++) {
            h[i + 1] = h[i] + (int)v[i].size();
            for (auto &e : v[i]) {
                cell.push_back(e.first);
                id.push_back(e.second);
            }
        }
        const size_t n1 = h.size(), n2 = cell.size();
        h.insert(h.end(), cell.begin(), cell.end());
        h.push_back(0);
        h.insert(h.end(), id.begin(), id.end());
        h.push_back(0);
        int *d = nullptr;
        OTF_CUDA(cudaMallocAsync(&d, sizeof(int) * h.size(), st_));
        OTF_CUDA(cudaMemcpyAsync(d, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice, st_));
        OTF_CUDA(cudaStreamSynchronize(st_));
        a.rcve_ptr = d;
        a.rcve_cell = d + n1;
        a.rcve_id = d + n1 + n2 + 1;
    }
    int rc = 0;
    for (int f = 0; f < 4 && !rc; f++)
        for (int s = 0; s < 2 && !rc; s++)
            if (cudaMemsetAsync(fld_[1][f][s], 0, fb, st_) != cudaSuccess)
                rc = -1;
    if (!rc && cudaMemsetAsync(grad_, 0, fb, st_) != cudaSuccess)
        rc = -1;
    int cur = 0;  // slot of the adjoint state of the step about to be reversed
    for (int j = n_ck_ - 1; j >= 0 && !rc; j--) {
        const int t0 = j * every, t1 = std::min(t0 + every, T - 1);
        // restore the checkpoint into the slot parity of t0
        const float *ck = ckpt_ + (size_t)j * 4 * fs;
        for (int f = 0; f < 4 && !rc; f++)
            if (cudaMemcpyAsync(fld_[0][f][t0 & 1], ck + (size_t)f * fs, fb, cudaMemcpyDeviceToDevice,
                                st_) != cudaSuccess)
                rc = -1;
        // A(t0) .. A(t1-1) into the segment buffer
        for (int f = 0; f < 2 && !rc; f++)
            if (cudaMemcpyAsync(seg_ + (size_t)f * fs, ck + (size_t)(2 + f) * fs, fb,
                                cudaMemcpyDeviceToDevice, st_) != cudaSuccess)
                rc = -1;
        for (int t = t0 + 1; t < t1 && !rc; t++) {
            const int i = (t - 1) & 1, o = t & 1;
            p.t = t;
            p.f0 = Fields{fld_[0][0][i], fld_[0][1][i], fld_[0][2][i], fld_[0][3][i],
                          fld_[0][0][o], fld_[0][1][o], fld_[0][2][o], fld_[0][3][o]};
            rc = launch_forward_step(p, false, grid, i, i);
            float *sg = seg_ + (size_t)(t - t0) * 2 * fs;
            for (int f = 0; f < 2 && !rc; f++)
                if (cudaMemcpyAsync(sg + (size_t)f * fs, fld_[0][2 + f][o], fb, cudaMemcpyDeviceToDevice,
                                    st_) != cudaSuccess)
                    rc = -1;
        }
        // adjoint steps t1 .. t0+1
        for (int t = t1; t > t0 && !rc; t--) {
            const float *sg = seg_ + (size_t)(t - 1 - t0) * 2 * fs;
            a.t = t;
            a.lx_in = fld_[1][0][cur];
            a.lz_in = fld_[1][1][cur];
            a.mx_in = fld_[1][2][cur];
            a.mz_in = fld_[1][3][cur];
            a.lx_out = fld_[1][0][cur ^ 1];
            a.lz_out = fld_[1][1][cur ^ 1];
            a.mx_out = fld_[1][2][cur ^ 1];
            a.mz_out = fld_[1][3][cur ^ 1];
            a.ax_prev = sg;
            a.az_prev = sg + fs;
            k_adjoint_step<ATX, ATZ, ABH><<<agrid, NT, sizeof(float) * AG::FLOATS, st_>>>(a);
            if (cudaGetLastError() != cudaSuccess) {
                set_error_msg(2, "adjoint step launch failed");
                rc = -1;
            }
            cur ^= 1;
        }
    }
    variant_ = saved;
    cudaFreeAsync((void *)a.rcve_ptr, st_);
    if (rc)
        return -1;
    // dL/d(c^2) = (dt/dx) dL/dq, summed over shots
    return grad_sum(grad_c2_dev, cfg_.dt / cfg_.dx);
}

}  // namespace otf
