// Host-side engine: owns the device state of one problem (grid, model,
// receivers, sources, boundary ring) for a batch of shots and drives the
// fused step kernels through captured CUDA graphs.
#pragma once
#include <cuda_runtime.h>
#include <algorithm>
#include <vector>
#include "otf_common.cuh"
#include "pml_step.cuh"
#include "pml_step_tma.cuh"
#include "pml_step_split.cuh"
#include "pml_step_stream.cuh"
#include "misfit.h"

namespace otf {

struct UnfusedParams;  // pml_step_unfused.cuh

enum Precision : int { kFaithful = 0, kFast = 1 };

// Tile shapes compiled into the library (owned cells per CTA).
struct TileShape {
    int tx, tz;
};
constexpr int kNumTileShapes = 5;
extern const TileShape kTileShapes[kNumTileShapes];

struct EngineConfig {
    int X = 0, Z = 0, T = 0;
    float dx = 1.f, dz = 1.f, dt = 1.f;  // the reference's constvec {dx, dz, dt}
    int max_shots = 1;
    int precision = kFaithful;
    int tile = 0;  // index into kTileShapes
};

class Engine {
  public:
    Engine() = default;
    ~Engine();
    Engine(const Engine &) = delete;
    Engine &operator=(const Engine &) = delete;

    // Set-up. All host arrays; d_x / d_z are [Z*X] damping profiles as the
    // reference takes them (cuda_interface_pml.py:116-132 builds them).
    int init(const EngineConfig &cfg, const float *d_x, const float *d_z);
    int set_model(const float *cquad, bool on_device);  // c^2 in the reference's nondimensional units, [Z*X]
    int set_sources(int n, const int *x, const int *z, const float *src);  // src [n*T]
    int set_receivers(int n, const int *x, const int *z);
    int set_ring(int n, const int *x, const int *z);
    // Which sources fire in each shot: shot s fires srcs[ptr[s] .. ptr[s+1]).
    int set_shots(int n_shots, const int *ptr, const int *srcs);

    // Forward modelling of all shots; receivers recorded into rec_dev()
    // ([n_shots][n_rec][T], column 0 zero). With ring, the boundary ring is
    // recorded too (gradient phase 1).
    int forward(bool with_ring);
    // Reverse phase of the gradient (phase 2) given adjoint sources already in
    // adj_dev() ([n_shots][n_rec][T]); per-shot gradients land in grad_dev().
    int reverse();

    // Copies of results.
    int copy_traces(float *dst, int shot0, int n, cudaMemcpyKind kind);
    int copy_grad_shot(int shot, float *dst, cudaMemcpyKind kind);  // unpadded [Z*X]
    // sum over shots * scale; scale == 0: sum / n_shots (FP32 division)
    int grad_sum(float *dst_dev_unpadded, float scale);

    // Observed traces [n_shots][n_rec][T] and the device misfit: fills
    // adj_dev() from rec_dev() vs observed, per-trace misfits into
    // misfit_dev() [n_shots*n_rec] and their sum into *total_dev (device).
    int set_observed(const float *obs, cudaMemcpyKind kind);
    int misfit(int kind, double *total_dev);
    // forward + misfit + reverse + shot mean, replayed as one CUDA graph
    int gradient(int kind);
    // the same work as an uninstantiated graph (caller owns it), for
    // composing several engines into one launch
    int gradient_graph(int kind, cudaGraph_t *out);
    // forward + device misfit of every shot; total in misfit_total_dev()
    int objective(int kind);
    // sum over shots and every `every`-th step of P^2 into illum_dev() [Z*X]
    int illumination(int every);
    // Headless video of the forward modelling (frames.cu): the forward of
    // every shot (receivers recorded as by forward(false)), and at every
    // `every`-th step t the total pressure of shot `shot` quantised on the
    // device to an 8-bit grey frame [Z][X] as the reference's video writer
    // does; frames reach `sink` in order, in chunks of at most 256 MiB.
    using FrameSink = int (*)(void *ctx, const unsigned char *frames, int n_frames);
    int frames(int every, int shot, FrameSink sink, void *ctx);
    float *illum_dev() { return illum_; }

    // Differentiable path (engine_adjoint.cu): forward of every shot keeping
    // the full state every `every` steps (sqrt(T) checkpoints), then the
    // exact discrete adjoint, recomputing each segment's forward states:
    // grad_c2 [Z*X] (device, unpadded) = sum over shots of dL/d(c^2) for
    // dL/drec = g [n_shots][n_rec][T] (device).
    int forward_checkpointed(int every);
    int backward_exact(const float *g_dev, float *grad_c2_dev);
    float *grad_mean_dev() { return gsum_; }
    double *misfit_total_dev() { return tot_; }

    float *rec_dev() { return rec_; }
    float *adj_dev() { return adj_; }
    double *misfit_dev() { return mis_; }
    cudaStream_t stream() const { return st_; }
    int n_shots() const { return n_shots_; }
    int n_rec() const { return n_rec_; }
    const EngineConfig &config() const { return cfg_; }
    const Layout &layout() const { return L_; }
    int set_precision(int prec);
    int set_tile(int tile);
    // -1 automatic (default); 0 one tile per CTA; 1 persistent TMA-pipelined;
    // 2 persistent strip-split (fast numerics); 3 z-streaming strips (fast
    // numerics, separable damping, X a multiple of 4); 4 unfused streaming
    // half-steps (fast numerics, separable damping); 5 paired half-steps, one
    // launch per step (fast numerics, separable damping); 6 row-lag fused
    // half-steps, one pass per step (fast numerics, separable damping, no
    // ring cell listed twice). Falls back where not compiled or not
    // applicable.
    int set_variant(int variant);
    // paired kernels: P items issued before the first A item (0 = one
    // generation of resident CTAs)
    void set_paired_lead(int lead) { pair_lead_ = lead; drop_graphs(); }
    // fused kernels: rows per chunk (>= 8)
    void set_fused_rows(int rows) { fused_rows_ = rows < 8 ? 8 : rows; drop_graphs(); }
    // shot groups run as parallel launch chains by the unfused kernels (0:
    // automatic, one per 16 shots up to kMaxLanes; 1: one chain)
    void set_lanes(int lanes) { lanes_req_ = lanes < 0 ? 0 : lanes; drop_graphs(); }
    int lanes_in_use() const;  // lanes of the time loops with the current settings
    // rows per segment of the z-streaming kernels (>= 8)
    int set_stream_rows(int rows);
    int variant_in_use() const;
    // waits for the stream and reports a timed-out bounded wait in a kernel
    int sync();

  private:
    int build_tables();
    int build_maps();
    int prepare();
    int prepare_gradient(int kind);
    int emit_gradient(int kind);
    // hook(ctx, t, slot) runs after the step-t launch (slot: P's output slot)
    using StepHook = int (*)(void *ctx, int t, int slot);
    int emit_forward(bool with_ring, StepHook hook = nullptr, void *ctx = nullptr);
    int emit_reverse();
    template <class Emit>
    int capture(cudaGraphExec_t *out, Emit emit);
    int launch_forward_step(const StepParams &p, bool with_ring, dim3 grid, int pin, int ain);
    int launch_reverse_step(const StepParams &p, dim3 grid, int pin, int ain, int in1);
    int launch_stream(const StepParams &p, int kind);  // 0 forward, 1 forward + ring, 2 reverse
    int launch_unfused(const StepParams &p, int kind);  // 0 forward, 1 forward + ring, 2 reverse
    int launch_paired(const StepParams &p, int kind);   // 0 forward, 1 forward + ring, 2 reverse
    int launch_fused(const StepParams &p, int kind);    // 0 forward, 1 forward + ring, 2 reverse
    UnfusedParams unfused_params(const StepParams &p, int kind) const;
    int paired_lead(int kind) const;
    int begin_steps();             // before a time loop of step launches
    int end_steps(int n_steps, int lanes = 1);  // after it
    template <class Step>
    int lane_loop(int lanes, Step step);  // step(t) for every lane's shots, lanes as parallel chains
    void drop_graphs();
    StepParams base_params() const;
    void free_all();

    EngineConfig cfg_;
    Layout L_;
    bool ready_ = false;
    bool sep_ = true;
    bool two_q_ = false;
    int n_src_ = 0, n_rec_ = 0, n_ring_ = 0, n_shots_ = 1;
    std::vector<int> src_x_, src_z_, rec_x_, rec_z_, ring_x_, ring_z_;
    std::vector<int> shot_ptr_, shot_srcs_;

    cudaStream_t st_ = nullptr;
    // lanes: the unfused time loops split the shots into up to kMaxLanes
    // groups, each its own chain of launches (lane 0 on st_), forked from and
    // joined back into st_ inside the captured graph
    static constexpr int kMaxLanes = 4;
    cudaStream_t lane_st_[kMaxLanes] = {};
    cudaEvent_t lane_ev_[kMaxLanes] = {};
    int lanes_req_ = 0;  // 0: automatic
    // launch context of the unfused kernels inside a time loop (0: every shot on st_)
    cudaStream_t ust_ = nullptr;
    int ushot0_ = 0, ushots_ = 0;
    // device buffers
    float *qf_ = nullptr, *qr_ = nullptr;                            // padded P coefficients
    float *cq_stage_ = nullptr;                                      // [Z*X] staging of a host model
    float *dampx_ = nullptr, *dampz_ = nullptr;                      // separable multipliers
    float *dampx2_ = nullptr, *dampz2_ = nullptr;                    // general multipliers
    float *fld_[2][4][2] = {};  // [set][Px,Pz,Ax,Az][slot], each [max_shots][slot floats]
    float *grad_ = nullptr;     // [max_shots][slot floats]
    float *rec_ = nullptr;      // [max_shots][n_rec][T]
    float *ring_ = nullptr;     // [max_shots][T][n_ring]
    float *src_ = nullptr, *tab_src_ = nullptr;  // [n_src][T]
    float *adj_ = nullptr, *tab_adj_ = nullptr;  // [max_shots][n_rec][T]
    float *obs_ = nullptr;                       // [max_shots][n_rec][T]
    double *mis_ = nullptr;                      // [max_shots*n_rec]
    void *mscratch_ = nullptr;                   // misfit CDF scratch
    int64_t mscratch_bytes_ = 0;
    // scratch buffers outgrown while graphs (this engine's, or multi-instance
    // graphs composed from them) may still hold their addresses: freed with
    // the engine, never while such a graph could still run
    std::vector<void *> retired_;
    int grow_scratch(int64_t need);
    int *inj_src_ = nullptr;   // CSR: ptr[max_shots+1] | x | z | row
    int *inj_adj_ = nullptr;
    int *tabs_ = nullptr;      // per-tile receiver / ring tables
    size_t inj_src_cap_ = 0, tabs_cap_ = 0;
    int *sen_ptr_ = nullptr, *sen_cell_ = nullptr, *sen_id_ = nullptr;
    int *ringo_ptr_ = nullptr, *ringo_cell_ = nullptr;
    int *ringe_ptr_ = nullptr, *ringe_cell_ = nullptr, *ringe_id_ = nullptr;
    int *inj_src_ptr_ = nullptr, *inj_src_x_ = nullptr, *inj_src_z_ = nullptr, *inj_src_row_ = nullptr;
    int *inj_adj_ptr_ = nullptr, *inj_adj_x_ = nullptr, *inj_adj_z_ = nullptr, *inj_adj_row_ = nullptr;

    cudaGraphExec_t g_fwd_ = nullptr, g_fwd_ring_ = nullptr, g_rev_ = nullptr;
    cudaGraphExec_t g_grad_[kNumMisfits] = {};  // per misfit kind
    cudaGraphExec_t g_obj_[kNumMisfits] = {};   // forward + misfit
    cudaGraphExec_t g_illum_ = nullptr;
    int illum_every_ = 0;
    float *illum_ = nullptr;  // [Z*X] illumination of the last illumination()
    float *gsum_ = nullptr;  // [Z*X] shot-mean gradient of the last gradient()
    double *tot_ = nullptr;  // misfit total of the last gradient()
    int graph_shots_ = -1;
    bool tables_dirty_ = true;

    // strip-split (fast) kernel tables
    int *srce_ptr_ = nullptr, *srce_cell_ = nullptr, *srce_id_ = nullptr;
    int *rcve_ptr_ = nullptr, *rcve_cell_ = nullptr, *rcve_id_ = nullptr;
    int *tile_edge_ = nullptr, *fire_row_ = nullptr;
    std::vector<float> hdampx_, hdampz_;  // host copies of the separable multipliers (padded index)

    // differentiable path: checkpoints [n_ck][4 fields][max_shots][slot] and
    // the recomputed A history of one segment [every][2][max_shots][slot]
    float *ckpt_ = nullptr, *seg_ = nullptr;
    size_t ckpt_bytes_ = 0, seg_bytes_ = 0;
    int ck_every_ = 0, n_ck_ = 0;
    bool ck_valid_ = false;

    int variant_ = -1;
    // z-streaming kernel tables (built with the other tables)
    StreamTabs stb_{};
    // unfused kernels: per-CTA injection lists, receiver and ring offsets
    struct {
        const int *src_ptr, *src_off, *src_id, *src_cta, *rcv_ptr, *rcv_off, *rcv_id, *rcv_cta;
        const int *rec_off, *ring_off, *ring_cta, *ring_cta_off, *ring_cta_k;
        const int *rec_cta, *rec_cta_off, *rec_cta_id;  // every receiver grouped by owning block
        int n_src_cells, n_rcv_cells, ncb, nseg;
    } utb_{};
    // row-lag fused kernels: ring index map and per-row point lists (in tabs_)
    struct {
        const int *ringmap, *src_rp, *src_cx, *src_ce, *src_id, *rcv_rp, *rcv_cx, *rcv_ce, *rcv_id;
        const int *rec_rp, *rec_cx, *rec_id;
    } ftb_{};
    bool fused_ok_ = true;   // no ring cell listed twice
    int fused_rows_ = 64;    // rows per chunk of the fused kernels
    // paired kernels: ticket counter (first 256 bytes) and done counts
    // [max_shots][nseg]
    void *pair_sync_ = nullptr;
    size_t pair_sync_bytes_ = 0;
    int pair_lead_ = 0;
    size_t pair_ticket_bytes() const
    {
        return ((size_t)std::max(cfg_.max_shots, n_shots_) * sizeof(unsigned long long) + 255) / 256 * 256;
    }
    int n_strips_ = 0, seg_h_ = 64;
    int *derr_ = nullptr;         // device error flag of the bounded waits
    unsigned *ledger_ = nullptr;  // launches of the unfused step kernels in the current time loop
    TmaParams *tmap_ = nullptr;   // tensor maps of every field, slot and coefficient
    bool maps_dirty_ = true;
};

}  // namespace otf
