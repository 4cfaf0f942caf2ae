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
 * idx_source == -1 fires every source, otherwise only source idx_source. */
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

#ifdef __cplusplus
}
#endif
#endif
