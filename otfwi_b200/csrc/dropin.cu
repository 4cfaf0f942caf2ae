// The reference's C-ABI (regression_PML_single.cu, the library
// cuda_interface_pml.py loads as simulator/bin/cuda_regression_PML_single.so),
// re-implemented on the fused B200 engine. Same symbol names, argument
// meaning and ownership rules; differences are listed in include/otfwi.h.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <memory>
#include <vector>
#include "engine.h"
#include "../../include/otfwi.h"

namespace otf {
int last_status();
const char *last_error();
}  // namespace otf

namespace {

struct DropIn {
    otf::Engine eng;
    int X = 0, Z = 0, T = 0, n_src = 0, n_sen = 0;
    float *rec_h = nullptr;   // pinned [n_sen*T], returned through init_memory_sim
    float *grad_h = nullptr;  // pinned [Z*X], returned through init_memory_reg
    float *sim_h = nullptr;   // pinned [n_sen*T], handed to the adjoint callback
    float *adj_h = nullptr;   // pinned [n_sen*T], filled by the adjoint callback
    void *python_adj = nullptr;
    bool reg_ready = false;

    ~DropIn() { free_host(); }
    void free_host()
    {
        float **b[] = {&rec_h, &grad_h, &sim_h, &adj_h};
        for (float **p : b) {
            if (*p)
                cudaFreeHost(*p);
            *p = nullptr;
        }
    }
};

std::unique_ptr<DropIn> g_state;

int env_int(const char *name, int dflt)
{
    const char *v = getenv(name);
    return (v && *v) ? atoi(v) : dflt;
}

// Choose which sources fire: idx == -1 fires all of them, otherwise only
// source idx (somaFonteIntegral's "idx!=-1 && idx!=n" test,
// regression_PML_single.cu:282); an index that matches no source fires none.
int select_shot(DropIn &s, int idx)
{
    std::vector<int> srcs;
    if (idx == -1) {
        for (int k = 0; k < s.n_src; k++)
            srcs.push_back(k);
    } else if (idx >= 0 && idx < s.n_src) {
        srcs.push_back(idx);
    }
    int ptr[2] = {0, (int)srcs.size()};
    return s.eng.set_shots(1, ptr, srcs.empty() ? ptr : srcs.data());
}

}  // namespace

extern "C" {

int otf_last_status(void) { return otf::last_status(); }
const char *otf_last_error(void) { return otf::last_error(); }
void otf_clear_error(void) { otf::clear_error(); }

void init_memory_sim(int x, int z, int t, float *cq, float *const_vec, float *d_x_h, float *d_z_h,
                     int ns, int *ps_x, int *ps_z, int nm, int *pm_x, int *pm_z, float *src,
                     float *init, float **rec)
{
    (void)init;  // the reference never allocates its `initial` buffer; runs start from rest
    otf::clear_error();
    g_state.reset(new DropIn());
    DropIn &s = *g_state;
    s.X = x;
    s.Z = z;
    s.T = t;
    s.n_src = ns;
    s.n_sen = nm;
    otf::EngineConfig cfg;
    cfg.X = x;
    cfg.Z = z;
    cfg.T = t;
    cfg.dx = const_vec[0];
    cfg.dz = const_vec[1];
    cfg.dt = const_vec[2];
    cfg.max_shots = 1;
    cfg.precision = env_int("OTFWI_PRECISION", otf::kFaithful);
    cfg.tile = env_int("OTFWI_TILE", 0);
    if (s.eng.init(cfg, d_x_h, d_z_h) || s.eng.set_variant(env_int("OTFWI_KERNEL", -1)) ||
        s.eng.set_stream_rows(env_int("OTFWI_STREAM_ROWS", 64)) ||
        s.eng.set_model(cq, false) ||
        s.eng.set_sources(ns, ps_x, ps_z, src) || s.eng.set_receivers(nm, pm_x, pm_z) ||
        s.eng.set_ring(0, nullptr, nullptr) || select_shot(s, -1))
        return;
    const size_t n = sizeof(float) * (size_t)(nm > 0 ? nm : 1) * t;
    if (cudaMallocHost(&s.rec_h, n) != cudaSuccess) {
        otf::set_error_msg(2, "pinned allocation of the recording buffer failed");
        return;
    }
    memset(s.rec_h, 0, n);
    if (rec)
        *rec = s.rec_h;
}

void init_memory_reg(float *obs, float **grad_ptr, int *p_rev_x, int *p_rev_z, int nr)
{
    (void)obs;  // copied by the reference into a device buffer nothing reads
    if (!g_state) {
        otf::set_error_msg(2, "init_memory_reg called before init_memory_sim");
        return;
    }
    DropIn &s = *g_state;
    if (s.eng.set_ring(nr, p_rev_x, p_rev_z))
        return;
    // the recording buffer handed out by init_memory_sim stays valid
    float **b[] = {&s.grad_h, &s.sim_h, &s.adj_h};
    for (float **p : b) {
        if (*p)
            cudaFreeHost(*p);
        *p = nullptr;
    }
    const size_t nt = sizeof(float) * (size_t)(s.n_sen > 0 ? s.n_sen : 1) * s.T;
    const size_t ng = sizeof(float) * (size_t)s.X * s.Z;
    if (cudaMallocHost(&s.sim_h, nt) != cudaSuccess ||
        cudaMallocHost(&s.adj_h, nt) != cudaSuccess || cudaMallocHost(&s.grad_h, ng) != cudaSuccess) {
        otf::set_error_msg(2, "pinned allocation failed");
        return;
    }
    memset(s.grad_h, 0, ng);
    s.reg_ready = true;
    if (grad_ptr)
        *grad_ptr = s.grad_h;
}

void setCquad(float *cq)
{
    if (!g_state) {
        otf::set_error_msg(2, "setCquad called before init_memory_sim");
        return;
    }
    if (g_state->eng.set_model(cq, false))
        return;
    g_state->eng.sync();
}

void set_source(int n_source, int *src_x, int *src_z, float *source)
{
    if (!g_state) {
        otf::set_error_msg(2, "set_source called before init_memory_sim");
        return;
    }
    DropIn &s = *g_state;
    if (s.eng.set_sources(n_source, src_x, src_z, source))
        return;
    s.n_src = n_source;
    select_shot(s, -1);
}

void def_python_adj(void *fn)
{
    if (g_state)
        g_state->python_adj = fn;
}

namespace {
struct FrameFile {
    FILE *fp;
    size_t frame_bytes;
};
int write_frames(void *ctx, const unsigned char *frames, int n)
{
    FrameFile &f = *static_cast<FrameFile *>(ctx);
    if (fwrite(frames, 1, (size_t)n * f.frame_bytes, f.fp) != (size_t)n * f.frame_bytes) {
        otf::set_error_msg(3, "cuda_simulate: writing the video frames failed");
        return -1;
    }
    return 0;
}

// en_out = 1: the frames the reference pipes into ffmpeg (8-bit grey [Z][X]
// per step t = 1..T-1, regression_PML_single.cu:619-700) are written raw to
// OTFWI_FRAMES_PATH, default output/outputPML.gray (the reference's
// output/outputPML.mp4 without the encoder; `ffmpeg -f rawvideo -pix_fmt
// gray -s XxZ -i output/outputPML.gray ...` encodes it).
int simulate_with_frames(DropIn &s)
{
    const char *env = getenv("OTFWI_FRAMES_PATH");
    std::string path = env && *env ? env : "output/outputPML.gray";
    const size_t cut = path.find_last_of('/');
    if (cut != std::string::npos && cut > 0)
        mkdir(path.substr(0, cut).c_str(), 0755);  // as the reference's "mkdir -p output/..."
    FILE *fp = fopen(path.c_str(), "wb");
    if (!fp) {
        otf::set_error_msg(3, "cuda_simulate: cannot open " + path);
        return -1;
    }
    const otf::EngineConfig &c = s.eng.config();
    FrameFile ff{fp, (size_t)c.X * c.Z};
    const int rc = s.eng.frames(1, 0, write_frames, &ff);
    if (fclose(fp) != 0 && rc == 0) {
        otf::set_error_msg(3, "cuda_simulate: closing " + path + " failed");
        return -1;
    }
    return rc;
}
}  // namespace

void cuda_simulate(int en_out, int idx_source)
{
    if (!g_state) {
        otf::set_error_msg(2, "cuda_simulate called before init_memory_sim");
        return;
    }
    DropIn &s = *g_state;
    if (select_shot(s, idx_source) || (en_out ? simulate_with_frames(s) : s.eng.forward(false)) ||
        s.eng.copy_traces(s.rec_h, 0, 1, cudaMemcpyDeviceToHost) || s.eng.sync())
        return;
}

void cuda_grad_ext(float *mse_h, void (*adj_calc)(float *, float *), int idx_source)
{
    if (!g_state || !g_state->reg_ready) {
        otf::set_error_msg(2, "cuda_grad_ext called before init_memory_reg");
        return;
    }
    DropIn &s = *g_state;
    if (select_shot(s, idx_source) || s.eng.forward(true) ||
        s.eng.copy_traces(s.sim_h, 0, 1, cudaMemcpyDeviceToHost) || s.eng.sync())
        return;
    const size_t nt = (size_t)s.n_sen * s.T;
    memset(s.adj_h, 0, sizeof(float) * nt);
    if (adj_calc)
        adj_calc(s.sim_h, s.adj_h);
    if (cudaMemcpyAsync(s.eng.adj_dev(), s.adj_h, sizeof(float) * nt, cudaMemcpyHostToDevice,
                        s.eng.stream()) != cudaSuccess) {
        otf::set_error_msg(2, "adjoint source upload failed");
        return;
    }
    if (s.eng.reverse() || s.eng.copy_grad_shot(0, s.grad_h, cudaMemcpyDeviceToHost) || s.eng.sync())
        return;
    if (mse_h)
        *mse_h = 0.f;  // as the reference (:840): the misfit comes back through the callback
}

int otf_set_precision(int precision)
{
    if (!g_state) {
        otf::set_error_msg(2, "otf_set_precision called before init_memory_sim");
        return -1;
    }
    return g_state->eng.set_precision(precision);
}

int otf_set_tile(int tile)
{
    if (!g_state) {
        otf::set_error_msg(2, "otf_set_tile called before init_memory_sim");
        return -1;
    }
    return g_state->eng.set_tile(tile);
}

void otf_release(void) { g_state.reset(); }

}  // extern "C"
