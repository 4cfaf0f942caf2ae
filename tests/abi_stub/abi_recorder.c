/* Test infrastructure: a stand-in library with the reference simulator's C
 * ABI (regression_PML_single.cu:39-43, 102-105, 229-230, 253-254, 618-619,
 * 704-705, and the set_source export cuda_interface_pml.py:183 calls) that
 * computes nothing: every call appends one line to the file named by
 * OTFWI_ABI_LOG with the call's name, its scalar arguments and an FNV-1a
 * digest of every array argument (over the lengths the reference library
 * reads), and returns deterministic traces, gradients and callback inputs.
 * Two wrappers that drive it with identical logs make identical calls into
 * any library with this ABI. */
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static int gX, gZ, gT, g_nsrc, g_nsen, g_nrev;
static float *g_rec, *g_grad, *g_sim, *g_adj;

static uint64_t fnv(const void *p, size_t n)
{
    const unsigned char *b = (const unsigned char *)p;
    uint64_t h = 1469598103934665603ull;
    for (size_t i = 0; i < n; i++) {
        h ^= b[i];
        h *= 1099511628211ull;
    }
    return h;
}

static void logf_(const char *fmt, ...)
{
    const char *path = getenv("OTFWI_ABI_LOG");
    if (!path)
        return;
    FILE *f = fopen(path, "a");
    if (!f)
        return;
    va_list ap;
    va_start(ap, fmt);
    vfprintf(f, fmt, ap);
    va_end(ap);
    fputc('\n', f);
    fclose(f);
}

static float value(int seed, int i) { return (float)((seed * 7919 + i * 104729) % 2003) / 1001.0f - 1.0f; }

void init_memory_sim(int X, int Z, int T, float *cquad, float *constvec, float *d_x, float *d_z, int n_source,
                     int *src_x, int *src_z, int n_sensor, int *sen_x, int *sen_z, float *source, float *initial,
                     float **rec_out)
{
    size_t n = (size_t)X * Z;
    gX = X;
    gZ = Z;
    gT = T;
    g_nsrc = n_source;
    g_nsen = n_sensor;
    logf_("init_memory_sim %d %d %d cquad=%016llx constvec=%016llx d_x=%016llx d_z=%016llx n_source=%d "
          "src_x=%016llx src_z=%016llx n_sensor=%d sen_x=%016llx sen_z=%016llx source=%016llx",
          X, Z, T, (unsigned long long)fnv(cquad, 4 * n), (unsigned long long)fnv(constvec, 12),
          (unsigned long long)fnv(d_x, 4 * n), (unsigned long long)fnv(d_z, 4 * n), n_source,
          (unsigned long long)fnv(src_x, 4 * (size_t)n_source), (unsigned long long)fnv(src_z, 4 * (size_t)n_source),
          n_sensor, (unsigned long long)fnv(sen_x, 4 * (size_t)n_sensor),
          (unsigned long long)fnv(sen_z, 4 * (size_t)n_sensor),
          (unsigned long long)fnv(source, 4 * (size_t)n_source * T));
    (void)initial; /* read by neither library */
    free(g_rec);
    free(g_sim);
    free(g_adj);
    g_rec = (float *)calloc((size_t)n_sensor * T, 4);
    g_sim = (float *)calloc((size_t)n_sensor * T, 4);
    g_adj = (float *)calloc((size_t)n_sensor * T, 4);
    *rec_out = g_rec;
}

void init_memory_reg(float *observed, float **grad_out, int *rev_x, int *rev_z, int n_revert)
{
    g_nrev = n_revert;
    logf_("init_memory_reg observed=%016llx rev_x=%016llx rev_z=%016llx n_revert=%d",
          (unsigned long long)fnv(observed, 4 * (size_t)gT * g_nsrc),
          (unsigned long long)fnv(rev_x, 4 * (size_t)n_revert), (unsigned long long)fnv(rev_z, 4 * (size_t)n_revert),
          n_revert);
    free(g_grad);
    g_grad = (float *)calloc((size_t)gX * gZ, 4);
    *grad_out = g_grad;
}

void setCquad(float *cquad)
{
    logf_("setCquad cquad=%016llx", (unsigned long long)fnv(cquad, 4 * (size_t)gX * gZ));
}

void set_source(int n_source, int *src_x, int *src_z, float *source)
{
    g_nsrc = n_source;
    logf_("set_source %d src_x=%016llx src_z=%016llx source=%016llx", n_source,
          (unsigned long long)fnv(src_x, 4 * (size_t)n_source), (unsigned long long)fnv(src_z, 4 * (size_t)n_source),
          (unsigned long long)fnv(source, 4 * (size_t)n_source * gT));
}

void cuda_simulate(int en_out, int idx_source)
{
    logf_("cuda_simulate %d %d", en_out, idx_source);
    for (int i = 0; i < g_nsen * gT; i++)
        g_rec[i] = value(idx_source + 11, i);
}

void cuda_grad_ext(float *mse_out, void (*adj)(float *, float *), int idx_source)
{
    for (int i = 0; i < g_nsen * gT; i++)
        g_sim[i] = value(idx_source + 23, i);
    memset(g_adj, 0, 4 * (size_t)g_nsen * gT);
    adj(g_sim, g_adj);
    logf_("cuda_grad_ext mse_in=%.9g idx=%d adj=%016llx", (double)mse_out[0], idx_source,
          (unsigned long long)fnv(g_adj, 4 * (size_t)g_nsen * gT));
    for (int i = 0; i < gX * gZ; i++)
        g_grad[i] = value(idx_source + 37, i);
    mse_out[0] = 0.0f;
}

void def_python_adj(void *fn) { (void)fn; }

void hilbert(float *signal, float *signal90, float *envelope, int N)
{
    (void)signal;
    (void)signal90;
    (void)envelope;
    (void)N;
}
