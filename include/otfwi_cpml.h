/*
 * otfwi_cpml.h -- C ABI of the second-order CPML forward library
 * (lib/cuda_regression_CPML.so), the exact symbols and signatures of the
 * reference's simulator/src/regression_CPML.cu (built by the reference into
 * simulator/bin/cuda_regression_CPML.so). Citations are to that file.
 *
 * Conventions kept from the reference: plain pointers, process-global state,
 * single-threaded use; the library owns the pinned buffer returned through
 * rec, valid until the next init_memory_sim; functions return void and a
 * failure is recorded, read with otf_last_status() / otf_last_error().
 * Deliberate differences: no cudaDeviceReset() in init_memory_sim (:362);
 * sources outside 4 <= x < X-4, 4 <= z < Z-4 are an error; en_out (video) is
 * accepted and ignored. Environment: OTFWI_PRECISION=1 selects FP32
 * staggered sums (default 0: the reference's arithmetic).
 */
#ifndef OTFWI_CPML_H
#define OTFWI_CPML_H

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces def_python_adj, regression_CPML.cu:43-47 (stored by the reference, unused). */
void def_python_adj(void *fn);

/* Replaces init_memory_sim, regression_CPML.cu:351-431: grid, sources and
 * receivers, dx, dz, dt, dt^2, the source factor (4 pi), c^2 and kappa
 * [Z*X], densities (rho unused, half-point densities along x and z [Z*X]),
 * CPML profiles d, K, alpha, a, b along x [X] and z [Z] at the integer and
 * half points (only K, a, b are used, as in the reference), source
 * waveforms [ns*T], the initial pressure P(0), P(1) [2*Z*X]; *rec receives a
 * pinned buffer [nm*T] that cuda_simulate2 fills. ppe: pixels per element
 * (1: idx_source selects one source). */
void init_memory_sim(int x, int z, int t, int ns, int nm, int ppe, int *ps_x, int *ps_z, int *pm_x, int *pm_z,
                     float dx_h, float dz_h, float dt_h, float dt2_h, float qtpi_h, float *cq, float *kp_unr,
                     float *rho_h, float *rho_hx_h, float *rho_hz_h, float *d_x_h, float *K_x_h,
                     float *alpha_x_h, float *a_x_h, float *b_x_h, float *d_x_half_h, float *K_x_half_h,
                     float *alpha_x_half_h, float *a_x_half_h, float *b_x_half_h, float *d_z_h, float *K_z_h,
                     float *alpha_z_h, float *a_z_h, float *b_z_h, float *d_z_half_h, float *K_z_half_h,
                     float *alpha_z_half_h, float *a_z_half_h, float *b_z_half_h, float *src, float *init,
                     float **rec);

/* Replaces setCquad, regression_CPML.cu:434-438: c^2 [Z*X] (scales the source term). */
void setCquad(float *cq);

/* Replaces set_source, regression_CPML.cu:441-448: source positions (at most
 * the count init_memory_sim received waveforms for). */
void set_source(int ns, int *ps_x, int *ps_z);

/* Replaces cuda_simulate2, regression_CPML.cu:451-531: the time loop, traces
 * of every receiver from t = 0 into the buffer returned by init_memory_sim. */
void cuda_simulate2(int en_out, int idx_source);

/* Every source as its own shot (one pixel per element), all shots advanced
 * by one launch per step (no counterpart in the reference, which runs one
 * cuda_simulate2 per source): traces [ns][nm][T] (host), each identical to
 * that of cuda_simulate2(0, s). Returns 0, or -1 with otf_last_error set. */
int otf_cpml_simulate_all(float *traces);

/* Exact discrete adjoint of the forward map (no counterpart in the
 * reference, which has no CPML gradient): grad_kappa [Z*X] = dL/dkappa for
 * dL/dtraces = g [nm*T] (host arrays), kappa = rho c^2 the Laplacian's
 * coefficient (the source term's c^2 held fixed). The forward is recomputed
 * with the state kept every checkpoint_every steps (sqrt(T) minimises
 * memory). Returns 0, or -1 with otf_last_error set. */
int otf_cpml_gradient(const float *g, float *grad_kappa, int checkpoint_every, int idx_source);

/* Status (additive; no reference counterpart) and release of every buffer. */
int otf_last_status(void);
const char *otf_last_error(void);
void otf_clear_error(void);
void otf_cpml_release(void);

#ifdef __cplusplus
}
#endif
#endif
