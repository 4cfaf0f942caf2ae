/*
 * otfwi.h -- C ABI of the Otfwi B200 library (libotfwi.so).
 *
 * Part 1 is the drop-in boundary: the exact symbols and signatures of the
 * reference library that cuda_interface_pml.py loads
 * (simulator/bin/cuda_regression_PML_single.so, cuda_interface_pml.py:9-30),
 * so the reference's ctypes wrapper runs unchanged against this library.
 * Citations are to the reference project's files.
 *
 * Conventions kept from the reference:
 *  - plain pointers and ints, process-global state, single-threaded use;
 *  - the library owns every device buffer and the pinned host buffers it
 *    returns through rec / grad_ptr; those stay valid until the next
 *    init_memory_sim;
 *  - functions return void; a failure is recorded (never an abort) and read
 *    with otf_last_status() / otf_last_error().
 * Deliberate differences from the reference:
 *  - no cudaDeviceReset() in init_memory_sim (regression_PML_single.cu:116),
 *    so the library can share a process and its CUDA context with PyTorch;
 *  - recorded traces have column t = 0 set to zero (the reference leaves it
 *    uninitialised, regression_PML_single.cu:661);
 *  - sources, receivers and ring cells must lie in the updated region
 *    4 <= x < X-4, 4 <= z < Z-4 (the reference silently writes cells its
 *    stencils never read); a violation is reported, not simulated;
 *  - en_out (video through an ffmpeg pipe) is accepted and ignored.
 */
#ifndef OTFWI_H
#define OTFWI_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Part 1: drop-in boundary (regression_PML_single.cu) ---------------- */

/* Replaces init_memory_sim, regression_PML_single.cu:102-153.
 * cquad [Z*X] = (c*dt/dx)^2, const_vec = {dx, dz, dt}, d_x/d_z [Z*X] damping
 * profiles, sources (ns, ps_x, ps_z, src [ns*T]), receivers (nm, pm_x, pm_z).
 * init [Z*X*2] is ignored (the reference never allocates its copy target).
 * *rec receives a library-owned pinned buffer [nm*T] that cuda_simulate fills. */
void init_memory_sim(int X, int Z, int T, float *cquad, float *const_vec, float *d_x, float *d_z,
                     int ns, int *ps_x, int *ps_z, int nm, int *pm_x, int *pm_z, float *src,
                     float *init, float **rec);

/* Replaces init_memory_reg, regression_PML_single.cu:229-250. Sets the
 * boundary ring (n_revert cells, rev_x/rev_z) used to reconstruct the forward
 * field backwards in time. obs is ignored (the reference copies it to a
 * buffer nothing reads). *grad_ptr receives a pinned buffer [Z*X] that
 * cuda_grad_ext fills. */
void init_memory_reg(float *obs, float **grad_ptr, int *rev_x, int *rev_z, int n_revert);

/* Replaces setCquad, regression_PML_single.cu:253-257: new model c^2 [Z*X]. */
void setCquad(float *cquad);

/* Replaces cuda_simulate, regression_PML_single.cu:618-702: forward modelling;
 * idx_source == -1 fires every source, otherwise only source idx_source.
 * en_out != 0: the video frames the reference pipes into ffmpeg (8-bit grey
 * [Z][X] per step t = 1..T-1, utils.cu:84-120) are written raw to
 * $OTFWI_FRAMES_PATH, default output/outputPML.gray (no encoder). */
void cuda_simulate(int en_out, int idx_source);

/* Replaces cuda_grad_ext, regression_PML_single.cu:704-846: forward with ring
 * recording, adj(sim [nm*T], adj_src [nm*T]) called once on this thread, then
 * adjoint + reconstruction + imaging condition; gradient into *grad_ptr.
 * *mse is set to 0 as in the reference (the misfit returns via the callback). */
void cuda_grad_ext(float *mse, void (*adj)(float *sim, float *adj_src), int idx_source);

/* Replaces def_python_adj, regression_PML_single.cu:39-43 (stored, unused). */
void def_python_adj(void *fn);

/* Replaces hilbert, simulator/src/hilbert.cpp:15-79: analytic-signal Hilbert
 * transform of signal [N] (spectrum indices [N/2, 2*(N/2)) zeroed):
 * signal90 = 2*Im/N, envelope = 2*|.|/N. Host arrays. */
void hilbert(float *signal, float *signal90, float *envelope, int N);

/* Called by cuda_interface_pml.py:183 (Cuda_interface_PML._set_source) but
 * absent from the reference library: replaces the sources and their
 * waveforms [n_source*T]. */
void set_source(int n_source, int *src_x, int *src_z, float *source);

/* ---- Part 2: status (additive; no reference counterpart) ---------------- */

int otf_last_status(void);        /* 0 = ok */
const char *otf_last_error(void); /* message of the last failure, "" if none */
void otf_clear_error(void);

/* Numerics of the drop-in path: 0 = faithful (the reference's FP64 staggered
 * sums, default), 1 = fast (FP32 pair-form sums). */
int otf_set_precision(int precision);
/* Tile shape of the fused step kernels (index into the compiled shapes). */
int otf_set_tile(int tile);
/* Free every buffer of the drop-in state. */
void otf_release(void);
/* Exercises the failure reporting of the step kernels' device-side checks
 * without any GPU fault: one bounded wait on a counter that nothing
 * increments (it gives up after its 0.5 s limit), one check of a paired
 * ticket count and one of an unfused launch count against wrong
 * expectations. Writes the error bits the device recorded to *bits (2 = a
 * dependency wait timed out, 4 = tickets out of range, 8 = a time loop's
 * launches short); returns 0 when all three were reported, -1 otherwise. */
int otf_selftest_paired_faults(int *bits);

/* ---- Part 3: batched shots (additive) -----------------------------------
 * Replaces the per-shot loops of Cuda_interface_PML.simulate / calc_grad
 * (cuda_interface_pml.py:185-236) and the host misfit callback
 * (cuda_interface_pml.py:238-249 -> adjoint_functions.py): every shot of a
 * shot table advances in the same launches, the misfit and adjoint sources
 * are computed on the device, and the whole gradient is one CUDA graph.
 * Pointers flagged on_device are device pointers (e.g. torch tensors on the
 * same device), otherwise host pointers. Calls are asynchronous on the
 * handle's stream (otf_batch_stream); otf_batch_sync waits. Return 0 on
 * success, -1 on failure (message in otf_last_error). */
typedef struct otf_batch otf_batch;

/* Same inputs as init_memory_sim + init_memory_reg: grid, constvec, damping
 * [Z*X], sources with waveforms [n_src*T], receivers, boundary ring; room for
 * max_shots shots; precision 0 faithful / 1 fast; tile shape index. */
otf_batch *otf_batch_create(int X, int Z, int T, const float *constvec, const float *d_x,
                            const float *d_z, int n_src, const int *src_x, const int *src_z,
                            const float *source, int n_rec, const int *rec_x, const int *rec_z,
                            int n_ring, const int *ring_x, const int *ring_z, int max_shots,
                            int precision, int tile);
void otf_batch_destroy(otf_batch *b);
/* Shot s fires sources srcs[ptr[s] .. ptr[s+1]) (full-matrix capture: ptr =
 * 0..n, srcs = 0..n-1). The reference's idx_source == -1 is one shot firing
 * every source. */
int otf_batch_set_shots(otf_batch *b, int n_shots, const int *ptr, const int *srcs);
int otf_batch_set_model(otf_batch *b, const float *cquad, int on_device);       /* [Z*X] */
int otf_batch_set_observed(otf_batch *b, const float *obs, int on_device);      /* [n_shots*n_rec*T] */
int otf_batch_set_precision(otf_batch *b, int precision);
int otf_batch_set_tile(otf_batch *b, int tile);
/* -1 (default): automatic -- 4 with fast numerics and separable damping, 2
 * with fast numerics otherwise, 1 with faithful numerics; 0: one tile per
 * CTA per step; 1: persistent CTAs with TMA double-buffered halo tiles (tile
 * shapes 0, 1 and 4; others use 0); 2: persistent strip-split kernels, fast
 * numerics only (tile shapes 0, 1 and 4); 3: z-streaming strips of 120
 * columns, fast numerics, separable damping, X a multiple of 4 (else 2); 4:
 * unfused half-steps, a launch each, fast numerics, separable damping; 5:
 * paired half-steps, both in one launch per step (P and A work items handed
 * out in order by a ticket counter), fast numerics, separable damping; 6:
 * row-lag fused half-steps, one pass over the fields per step (a warp
 * computes P(t) of a row and the A half-step four rows behind it from a
 * register window), fast numerics, separable damping, no ring cell listed
 * twice (else 4). 0 and 1 give bit-identical results, and so do 4, 5 and 6. */
int otf_batch_set_kernel(otf_batch *b, int variant);
/* Rows per segment of the z-streaming kernels (variant 3; default 64, >= 8). */
int otf_batch_set_stream_rows(otf_batch *b, int rows);
/* Paired kernels (variant 5): P work items issued before the first A item
 * (0, the default: one generation of resident CTAs; clamped to [2 column
 * blocks, all P items]). */
int otf_batch_set_paired_lead(otf_batch *b, int lead);
/* Row-lag fused kernels (variant 6): rows per chunk of a CTA (default 64,
 * >= 8; each chunk recomputes P(t) on 4 rows above and below it). */
int otf_batch_set_fused_rows(otf_batch *b, int rows);
/* Unfused kernels (variant 4): the shots split into `lanes` groups whose time
 * loops run as parallel launch chains inside the captured graph (0, the
 * default: one per 16 shots, at most 4; 1: one chain; OTFWI_LANES sets the
 * default). Results are bit-identical for every setting. */
int otf_batch_set_lanes(otf_batch *b, int lanes);
/* The lanes the batch's time loops use with its current settings (1 for
 * every variant but the unfused kernels). */
int otf_batch_lanes(otf_batch *b);
/* Forward modelling of every shot; traces [n_shots][n_rec][T] (NULL: keep). */
int otf_batch_forward(otf_batch *b, float *traces, int on_device);
/* Forward with boundary-ring recording (gradient phase 1). */
int otf_batch_forward_ring(otf_batch *b, float *traces, int on_device);
/* Full gradient: forward, device misfit (0 = L2, 1 = Wasserstein as
 * adjoint_functions.wasserstein, 2 = Wasserstein on softplus-normalised
 * traces, 3 = adjoint_functions.wasserstein_quad, 4 = adjoint_functions.
 * quad_envelope, 5 = adjoint_functions.wasserstein_pm with its negative-part
 * CDFs taken from the negative parts), reverse phase; grad [Z*X]
 * = mean over shots of the per-shot gradients, *misfit = sum over every
 * trace (both optional). */
int otf_batch_gradient(otf_batch *b, int misfit_kind, float *grad, double *misfit, int on_device);
/* Device misfit of the last forward traces against the observed traces:
 * per-trace misfits [n_shots*n_rec] (optional) and the adjoint sources. */
int otf_batch_misfit(otf_batch *b, int misfit_kind, double *per_trace, int on_device);
int otf_batch_adjoint(otf_batch *b, float *adj, int on_device);  /* copy out the adjoint sources */
/* Reverse phase after otf_batch_forward_ring, with adjoint sources adj
 * [n_shots][n_rec][T] (NULL: those of otf_batch_misfit); grad [Z*X] =
 * scale * sum over shots. */
int otf_batch_reverse(otf_batch *b, const float *adj, int on_device, float *grad, float scale,
                      int grad_on_device);
int otf_batch_shot_grad(otf_batch *b, int shot, float *grad, int on_device); /* one shot's [Z*X] */
/* Differentiable forward: traces of every shot while keeping the full
 * wavefield every `every` steps (sqrt(T) is the memory optimum). */
int otf_batch_forward_ckpt(otf_batch *b, int every, float *traces, int on_device);
/* Exact discrete adjoint of the last otf_batch_forward_ckpt:
 * grad_c2 [Z*X] = sum over shots of dL/d(c^2) for dL/dtraces = g
 * [n_shots][n_rec][T]. Each checkpoint segment's forward is recomputed once.
 * No reference counterpart: the reference's gradient (cuda_grad_ext)
 * cross-correlates a reconstructed field, an approximation of this one. */
int otf_batch_backward_exact(otf_batch *b, const float *g, int g_on_device, float *grad_c2,
                             int grad_on_device);
int otf_batch_sync(otf_batch *b);
void *otf_batch_stream(otf_batch *b);
/* Forward of every shot and the device misfit only (a line-search objective
 * evaluation): *misfit = sum over every trace. */
int otf_batch_objective(otf_batch *b, int misfit_kind, double *misfit, int on_device);
/* Source illumination illum [Z*X] = sum over shots and over every `every`-th
 * forward step of P^2 (one forward modelling). */
int otf_batch_illumination(otf_batch *b, int every, float *illum, int on_device);
/* Headless video (replaces the ffmpeg pipe of cuda_simulate(en_out = 1),
 * regression_PML_single.cu:619-700 / utils.cu:84-120 writeFramePipe): one
 * forward modelling of every shot (traces recorded as by
 * otf_batch_forward), and at every `every`-th step t = every, 2 every, ...
 * <= T-1 the total pressure of shot `shot` as an 8-bit grey frame [Z][X]:
 * (P - min) * (255 / (max - min)) truncated, receivers 255. frames: host
 * buffer of (T-1)/every * Z * X bytes. */
int otf_batch_frames(otf_batch *b, int every, int shot, unsigned char *frames);
/* Results of the last gradient of this batch (also after otf_multi_gradient). */
int otf_batch_last_gradient(otf_batch *b, float *grad, double *misfit, int on_device);

/* Several independent inversions -- different grids, shot counts and T --
 * as parallel branches of one CUDA graph: otf_multi_gradient computes every
 * instance's gradient in one graph launch; after otf_multi_sync read each
 * with otf_batch_last_gradient. The instances stay owned by the caller and
 * must outlive the group. No reference counterpart. */
typedef struct otf_multi otf_multi;
otf_multi *otf_multi_create(int n, otf_batch **batches);
void otf_multi_destroy(otf_multi *m);
/* chains > 0: instance i starts after instance i - chains has finished, so
 * at most `chains` instances run at once (0, the default: all at once). */
int otf_multi_set_chains(otf_multi *m, int chains);
int otf_multi_gradient(otf_multi *m, int misfit_kind);
int otf_multi_sync(otf_multi *m);

/* Stand-alone device misfit over n_traces traces [n_traces][T] (device
 * pointers, misfit [n_traces] FP64) with caller-owned scratch of at least
 * otf_misfit_scratch_bytes(kind, n_traces, T) bytes, on a cudaStream_t.
 * Kind 4 (quad_envelope) creates a cuFFT plan per (n_traces, T) on its first
 * call, which allocates: make that call outside stream capture. */
long long otf_misfit_scratch_bytes(int kind, int n_traces, int T);
int otf_misfit(int kind, const float *sim, const float *obs, float *adj, double *misfit,
               int n_traces, int T, void *scratch, long long scratch_bytes, void *stream);

/* Same as otf_misfit, but allocates nothing: no counterpart in the
 * reference. For callers that cannot allocate device memory when they need
 * a misfit -- their GPU memory is already reserved by another allocator, or
 * they cannot afford cudaMalloc/cudaFree, which may synchronise the device.
 * The scratch is a 16 MiB array built into the library (held on every GPU
 * that loads it until exit); n_traces * otf_misfit_scratch_bytes(kind, 1, T)
 * above 16 MiB is rejected with an error (returns -1). The first call in a
 * context (again after a cudaDeviceReset) looks the array's device address
 * up: make it before any stream capture. Under CUDA's default lazy module
 * loading the array is placed when the library's misfit module is first used
 * in a context (this call's first run, or an earlier otf_misfit), which needs
 * 16 MiB of free device memory at that moment; CUDA_MODULE_LOADING=EAGER
 * places it when the context is created instead. All calls share the array:
 * calls that may overlap on the GPU race, so order them on one stream.
 * Inputs and outputs are caller device memory. Kind 4 (quad_envelope) is
 * refused: its FFT plans allocate. */
int otf_misfit_noalloc(int kind, const float *sim, const float *obs, float *adj, double *misfit,
                       int n_traces, int T, void *stream);

/* ---- Part 4: learned gradient preconditioner (additive) -------------------
 * Kernels of a BF16 U-Net with FP32 accumulation, trained on the GPU. No
 * reference counterpart: the reference's inversion is plain L-BFGS-B on the
 * raw gradient (regression.py:82-88). All pointers are device pointers;
 * activations are [N][H][W][C] BF16 (void *), C a multiple of 16; conv
 * weights [9][Cout][Cin] BF16 (tap = 3*dy + dx); launches are asynchronous on
 * `stream` (a cudaStream_t). Return 0, or -1 with otf_last_error set. */

/* 3x3 convolution, zero padding: input channels [0, c0) from src0 and
 * [c0, c0+c1) from src1 (at half resolution, upsampled nearest, when up1);
 * out = bias + conv, ReLU if relu; output channels [0, split) go to dst0
 * ([..][split]) and [split, cout) to dst1 ([..][cout-split]), each zeroed
 * where its mask (same layout, optional) is <= 0. cout a multiple of 32. */
int otf_unet_conv3x3(const void *src0, int c0, const void *src1, int c1, int up1, const void *w,
                     const float *bias, int relu, void *dst0, const void *mask0, void *dst1,
                     const void *mask1, int split, int cout, int N, int H, int W, void *stream);
/* As otf_unet_conv3x3, with the weights also given packed for the tcgen05
 * kernels (wp, from otf_unet_pack_weights_tc of w): their stages then load
 * the weights by contiguous bulk copies instead of 16-byte tiled rows. */
int otf_unet_conv3x3_packed(const void *src0, int c0, const void *src1, int c1, int up1, const void *w,
                            const void *wp, const float *bias, int relu, void *dst0, const void *mask0,
                            void *dst1, const void *mask1, int split, int cout, int N, int H, int W,
                            void *stream);
/* wp [cin/8][9][cout][8] (BF16) = w [9][cout][cin] (BF16) regrouped by
 * 8-channel plane, the layout otf_unet_conv3x3_packed takes; cin a multiple
 * of 16. */
int otf_unet_pack_weights_tc(const void *w, int cout, int cin, void *wp, void *stream);
/* dw [9][cout][c0+c1] (FP32) += weight gradient for the pre-activation
 * gradient dz [N][H][W][cout] of that convolution's inputs. */
int otf_unet_conv3x3_wgrad(const void *src0, int c0, const void *src1, int c1, int up1, const void *dz,
                           int cout, float *dw, int N, int H, int W, int sm_count, void *stream);
/* Tensor-core path of the functions above: 1 = tcgen05 / UMMA kernels with
 * tensor-memory accumulators (default; the weight gradients of 16-input-
 * channel layers, of 32 -> 64 channels and of a concatenation with an
 * upsampled input into 32 channels keep the mma.sync kernel, measured faster
 * there), 2 = tcgen05 for every shape, 0 = the warp-level mma.sync kernels;
 * returns the previous setting (process-wide). */
int otf_unet_set_umma(int on);
/* Error bits of the tcgen05 kernels since the last call (1 = a bounded wait
 * timed out: that launch's results are invalid), cleared by the call; -1 if
 * the flag cannot be read. */
int otf_unet_status(void);
int otf_unet_bias_grad(const void *dz, int C, long long npix, float *db, void *stream); /* db += sum_p dz */
int otf_unet_pool2(const void *x, void *y, int N, int H, int W, int C, void *stream);  /* 2x2 mean */
/* dx += 0.25 * dy(parent) where x > 0 */
int otf_unet_pool2_bwd(const void *dy, const void *x, void *dx, int N, int H, int W, int C, void *stream);
/* dx [N][Hh][Wh][C] = (x > 0) * sum of dy over the 4 nearest-upsampling children */
int otf_unet_up2_bwd(const void *dy, const void *x, void *dx, int N, int Hh, int Wh, int C, void *stream);
/* FP32 [npix][cin] -> BF16 [npix][16], channels >= cin zero */
int otf_unet_pack_input(const float *x, int cin, long long npix, void *y, void *stream);
/* out[p] = b + sum_c x[p][c] w[c], x [npix][32] BF16, FP32 out */
int otf_unet_head(const void *x, const float *w, const float *b, long long npix, float *out, void *stream);
/* dx = dout * w * (x > 0) (BF16); dw += sum_p dout x; db += sum_p dout */
int otf_unet_head_bwd(const void *x, const float *w, const float *dout, long long npix, void *dx, float *dw,
                      float *db, void *stream);
/* loss += sum w (out - target)^2 * inv_norm; dout = 2 w (out - target) inv_norm (weight optional) */
int otf_unet_mse(const float *out, const float *target, const float *weight, long long n, float inv_norm,
                 float *dout, float *loss, void *stream);
/* Adam with bias correction (step counts from 1) and L2 weight decay on FP32 parameters */
int otf_unet_adam(float *p, const float *g, float *m, float *v, long long n, float lr, float b1, float b2,
                  float eps, int step, float weight_decay, void *stream);
/* BF16 copies of FP32 weights [9][cout][cin]: wf (same layout) and wb
 * [8 - tap][cin][cout] (the input-gradient convolution), wb optional */
int otf_unet_pack_weights(const float *w, int cout, int cin, void *wf, void *wb, void *stream);

#ifdef __cplusplus
}
#endif
#endif
