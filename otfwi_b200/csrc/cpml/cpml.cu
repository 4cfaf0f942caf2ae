// Second-order acoustic CPML forward path and the reference's CPML C ABI
// (lib/cuda_regression_CPML.so; the reference builds the same ABI from
// simulator/src/regression_CPML.cu into bin/cuda_regression_CPML.so).
//
// One fused launch per time step replaces the reference's two frame kernels
// (regression_CPML.cu:49-207): a CTA owns a 32 x 16 tile, stages P(t-1) with
// an 8-cell halo, computes the first staggered derivatives, their CPML
// memory variables and the density division on the tile plus a 4-cell halo
// (halo recomputed, not exchanged), then the second derivatives, their
// memory variables and P(t) = 2 P(t-1) - P(t-2) + lap dt^2 kappa on the
// owned cells; the CTA then adds the sources (:210-231) and records the
// receivers (:238-246) that lie in its tile, so a step is one launch (the
// reference's are four). The forward time loop is replayed as one CUDA graph. Fields keep the reference's
// layout: P in four time slots [4][Z][X] (so cells outside the update region
// hold what the reference's would), memory variables of the first
// derivatives in two slots (the halo recompute reads t-1 while owners write
// t), those of the second derivatives in place.
//
// Numerics: faithful (default) restates the reference's arithmetic: 8-tap
// staggered sums in FP64 (leading product rounded, seven FMAs), FP32 updates
// with the contractions fma(b, m, a*v) and fma(lap*dt2, kappa, 2 P1 - P2),
// IEEE divisions; fast uses the FP32 antisymmetric-pair staggered sums.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include "../otf_common.cuh"
#include "../../../include/otfwi_cpml.h"

namespace otf {
namespace cpml {

constexpr int TX = 32, TZ = 16, NTH = 256;
constexpr int SW = TX + 16, SH = TZ + 16;  // P(t-1) tile with an 8-cell halo
constexpr int VW = TX + 8, VH = TZ + 8;    // first-derivative region (4-cell halo)

constexpr double kC0 = 1.196289e+00, kC1 = 7.975260e-02, kC2 = 9.570313e-03, kC3 = 6.975446e-04;

struct Coef {
    const float *Kx, *ax, *bx, *Kxh, *axh, *bxh;  // [X]
    const float *Kz, *az, *bz, *Kzh, *azh, *bzh;  // [Z]
    const float *kappa, *rho_hx, *rho_hz;         // [Z][X]
    float dx, dz, dt2;
    // Divisions the step may skip without changing a bit: by a power-of-two
    // spacing (multiplication by its exact reciprocal rounds the same) and by
    // a K profile that is 1 everywhere (k_max = 1, the usual CPML).
    float inv_dx, inv_dz;  // 0 when the spacing is not a power of two
    int k_one;             // bit 0 Kx, 1 Kxh, 2 Kz, 3 Kzh all exactly 1
};

// v / d, IEEE-rounded, as a product when d is a power of two (inv != 0)
__device__ __forceinline__ float div_sp(float v, float d, float inv)
{
    return inv != 0.f ? __fmul_rn(v, inv) : __fdiv_rn(v, d);
}

struct StepArgs {
    int X, Z, t;
    const float *P1, *P2;  // P(t-1), P(t-2)
    float *Pn;             // P(t)
    const float *mx_in, *mz_in;
    float *mx_out, *mz_out;
    float *mxx, *mzz;      // in place
    float *lap;            // optional: lap(t) of every owned cell (adjoint recompute)
    Coef c;
    // point work of the step, done by the CTA owning the cell after its
    // P(t): sources (somaFonte) then, when rec is set, the receivers
    int T, ns, nm, ppe;
    const int *idx_dev, *sx, *sz, *pmx, *pmz;
    const float *cquad, *src;
    float qtpi;
    float *rec;
    // batched shots (blockIdx.z = shot s, which fires source s alone): field
    // pointers are shot 0's, shot_stride floats apart; rec is [shot][nm][T]
    size_t shot_stride;
    int batch;
};

__device__ __forceinline__ bool inb(int X, int Z, int x, int z) { return x >= 4 && z >= 4 && x < X - 4 && z < Z - 4; }

// derivPMLdx / dz (deriv_macros.h:85-108) from w[0..7] = m[c-3-off .. c+4-off]
template <bool FAITHFUL>
__device__ __forceinline__ float stag(const float *w, int stride)
{
    if (FAITHFUL) {
        double s = -kC3 * (double)w[7 * stride];
        s = fma(kC2, (double)w[6 * stride], s);
        s = fma(-kC1, (double)w[5 * stride], s);
        s = fma(kC0, (double)w[4 * stride], s);
        s = fma(-kC0, (double)w[3 * stride], s);
        s = fma(kC1, (double)w[2 * stride], s);
        s = fma(-kC2, (double)w[1 * stride], s);
        s = fma(kC3, (double)w[0], s);
        return (float)s;
    } else {
        constexpr float c0h = (float)kC0, c0l = (float)(kC0 - (double)(float)kC0);
        const float d0 = __fsub_rn(w[4 * stride], w[3 * stride]);
        const float d1 = __fsub_rn(w[5 * stride], w[2 * stride]);
        const float d2 = __fsub_rn(w[6 * stride], w[1 * stride]);
        const float d3 = __fsub_rn(w[7 * stride], w[0]);
        float s = __fmul_rn(-(float)kC3, d3);
        s = __fmaf_rn((float)kC2, d2, s);
        s = __fmaf_rn(-(float)kC1, d1, s);
        s = __fmaf_rn(c0l, d0, s);
        return __fmaf_rn(c0h, d0, s);
    }
}

template <bool FAITHFUL>
__global__ void __launch_bounds__(NTH) k_cpml_step(const StepArgs a)
{
    __shared__ float sP[SH][SW];
    __shared__ float sVx[VH][VW], sVz[VH][VW];
    const int X = a.X, Z = a.Z;
    const int x0 = blockIdx.x * TX, z0 = blockIdx.y * TZ;
    const size_t so = (size_t)blockIdx.z * a.shot_stride;
    const float *__restrict__ P1 = a.P1 + so;
    const float *__restrict__ P2 = a.P2 + so;
    float *__restrict__ Pn = a.Pn + so;
    const float *__restrict__ mx_in = a.mx_in + so;
    const float *__restrict__ mz_in = a.mz_in + so;
    float *__restrict__ mx_out = a.mx_out + so;
    float *__restrict__ mz_out = a.mz_out + so;
    float *__restrict__ mxxp = a.mxx + so;
    float *__restrict__ mzzp = a.mzz + so;
    float *rec = a.rec ? a.rec + (size_t)blockIdx.z * a.nm * a.T : nullptr;
    for (int k = threadIdx.x; k < SW * SH; k += NTH) {
        const int zz = k / SW, xx = k - zz * SW;
        const int x = x0 - 8 + xx, z = z0 - 8 + zz;
        sP[zz][xx] = inb(X, Z, x, z) ? P1[(size_t)z * X + x] : 0.f;
    }
    __syncthreads();
    // first derivatives, memory variables and density division on the tile + 4-cell halo
    for (int k = threadIdx.x; k < VW * VH; k += NTH) {
        const int ez = k / VW, ex = k - ez * VW;
        const int x = x0 - 4 + ex, z = z0 - 4 + ez;
        float vx = 0.f, vz = 0.f;
        if (inb(X, Z, x, z)) {
            const size_t i = (size_t)z * X + x;
            // offset 0: taps x-3 .. x+4 (tile column of x is ex + 4)
            const float v0x = div_sp(stag<FAITHFUL>(&sP[ez + 4][ex + 1], 1), a.c.dx, a.c.inv_dx);
            const float mx = __fmaf_rn(a.c.bxh[x], mx_in[i], __fmul_rn(a.c.axh[x], v0x));
            const float kx = (a.c.k_one & 2) ? v0x : __fdiv_rn(v0x, a.c.Kxh[x]);
            vx = __fdiv_rn(__fadd_rn(kx, mx), a.c.rho_hx[i]);
            const float v0z = div_sp(stag<FAITHFUL>(&sP[ez + 1][ex + 4], SW), a.c.dz, a.c.inv_dz);
            const float mz = __fmaf_rn(a.c.bzh[z], mz_in[i], __fmul_rn(a.c.azh[z], v0z));
            const float kz = (a.c.k_one & 8) ? v0z : __fdiv_rn(v0z, a.c.Kzh[z]);
            vz = __fdiv_rn(__fadd_rn(kz, mz), a.c.rho_hz[i]);
            if (ex >= 4 && ex < TX + 4 && ez >= 4 && ez < TZ + 4) {
                mx_out[i] = mx;
                mz_out[i] = mz;
            }
        }
        sVx[ez][ex] = vx;
        sVz[ez][ex] = vz;
    }
    __syncthreads();
    // second derivatives, memory variables and P(t) on the owned cells
    for (int k = threadIdx.x; k < TX * TZ; k += NTH) {
        const int oz = k / TX, ox = k - oz * TX;
        const int x = x0 + ox, z = z0 + oz;
        if (!inb(X, Z, x, z))
            continue;
        const size_t i = (size_t)z * X + x;
        // offset 1: taps x-4 .. x+3 (region column of x is ox + 4)
        const float vxx0 = div_sp(stag<FAITHFUL>(&sVx[oz + 4][ox], 1), a.c.dx, a.c.inv_dx);
        const float mxx = __fmaf_rn(a.c.bx[x], mxxp[i], __fmul_rn(a.c.ax[x], vxx0));
        mxxp[i] = mxx;
        const float vxx1 = __fadd_rn((a.c.k_one & 1) ? vxx0 : __fdiv_rn(vxx0, a.c.Kx[x]), mxx);
        const float vzz0 = div_sp(stag<FAITHFUL>(&sVz[oz][ox + 4], VW), a.c.dz, a.c.inv_dz);
        const float mzz = __fmaf_rn(a.c.bz[z], mzzp[i], __fmul_rn(a.c.az[z], vzz0));
        mzzp[i] = mzz;
        const float vzz1 = __fadd_rn((a.c.k_one & 4) ? vzz0 : __fdiv_rn(vzz0, a.c.Kz[z]), mzz);
        const float lap = __fadd_rn(vxx1, vzz1);
        Pn[i] = __fmaf_rn(__fmul_rn(lap, a.c.dt2), a.c.kappa[i], __fmaf_rn(2.f, P1[i], -P2[i]));
        if (a.lap)  // single-shot launches only
            a.lap[i] = lap;
    }
    if (a.ns == 0 && !rec)
        return;
    // sources in this tile (somaFonte, regression_CPML.cu:210-231), then the
    // receivers in it (:238-246), by the first warp: lanes test 32 points at
    // a time, lane 0 applies the sources in source order (as a sequential
    // loop would) and __syncwarp orders them before the recording reads
    __syncthreads();
    if (threadIdx.x >= 32)
        return;
    const int lane = threadIdx.x;
    auto mine = [&](int px, int pz) { return px >= x0 && px < x0 + TX && pz >= z0 && pz < z0 + TZ; };
    const int idx = a.batch ? (int)blockIdx.z : (a.ns > 0 ? *a.idx_dev : -1);
    for (int base = 0; base < a.ns; base += 32) {
        const int n = base + lane;
        const bool hit = n < a.ns && !(a.ppe == 1 && idx != -1 && idx != n) && mine(a.sx[n], a.sz[n]);
        unsigned m = __ballot_sync(0xffffffffu, hit);
        if (lane == 0)
            while (m) {
                const int k = base + __ffs(m) - 1;
                m &= m - 1;
                const size_t i = (size_t)a.sz[k] * X + a.sx[k];
                const float sv = __fmul_rn(__fmul_rn(a.qtpi, a.cquad[i]), a.src[(size_t)k * a.T + a.t]);
                Pn[i] = __fmaf_rn(sv, a.c.dt2, Pn[i]);
            }
        __syncwarp();
    }
    if (rec)
        for (int n = lane; n < a.nm; n += 32)
            if (mine(a.pmx[n], a.pmz[n]))
                rec[(size_t)n * a.T + a.t] = Pn[(size_t)a.pmz[n] * X + a.pmx[n]];
}

// gravaBufferSensores2ordem (regression_CPML.cu:238-246)
__global__ void k_cpml_record(const float *Pn, int X, int T, int t, int nm, const int *mx, const int *mz,
                              float *rec)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < nm)
        rec[(size_t)n * T + t] = Pn[(size_t)mz[n] * X + mx[n]];
}

// ---- exact discrete adjoint (dL/dkappa), the transposed step in three passes.
// W[k + 3], k = -3..4: weight of m[c + k - off] in derivPMLdx(m, off, c).
__constant__ float kW[8] = {(float)kC3, -(float)kC2, (float)kC1, -(float)kC0,
                            (float)kC0, -(float)kC1, (float)kC2, -(float)kC3};

// transpose of the staggered gather: sum_k W[k+3] a[j - (k - off) d] over inbounds sources
__device__ __forceinline__ float stagT(const float *a, int X, int Z, int x, int z, int ddx, int ddz, int off)
{
    float s = 0.f;
#pragma unroll
    for (int k = -3; k <= 4; k++) {
        const int xx = x - (k - off) * ddx, zz = z - (k - off) * ddz;
        if (inb(X, Z, xx, zz))
            s = fmaf(kW[k + 3], a[(size_t)zz * X + xx], s);
    }
    return s;
}

struct AdjArgs {
    int X, Z;
    float *LA, *LB, *LC;            // adjoint of P(t), partial adjoints of P(t-1), P(t-2)
    float *lmx, *lmz, *lmxx, *lmzz; // adjoints carried by the memory variables
    float *a0x, *a0z, *l0x, *l0z;   // adjoints of the second / first derivatives
    const float *lap;               // lap(t)
    float *grad;                    // dL/dkappa
    Coef c;
};

// P(t) = 2 P(t-1) - P(t-2) + dt2 kappa (vxx0/Kx + mxx(t) + vzz0/Kz + mzz(t))
__global__ void k_cpml_adj_a(const AdjArgs a)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)a.X * a.Z)
        return;
    const int z = (int)(i / a.X), x = (int)(i - (int64_t)z * a.X);
    if (!inb(a.X, a.Z, x, z)) {
        a.a0x[i] = a.a0z[i] = 0.f;
        a.LC[i] = 0.f;
        return;
    }
    const float la = a.LA[i];
    a.grad[i] = fmaf(la * a.c.dt2, a.lap[i], a.grad[i]);
    const float gl = a.c.dt2 * a.c.kappa[i] * la;
    a.LB[i] = fmaf(2.f, la, a.LB[i]);
    a.LC[i] = -la;
    const float tx = a.lmxx[i] + gl;
    a.a0x[i] = gl / a.c.Kx[x] + a.c.ax[x] * tx;
    a.lmxx[i] = a.c.bx[x] * tx;
    const float tz = a.lmzz[i] + gl;
    a.a0z[i] = gl / a.c.Kz[z] + a.c.az[z] * tz;
    a.lmzz[i] = a.c.bz[z] * tz;
}

// vxx0 = D(v1x, off 1)/dx; v1x = (v0x/Kxh + mx(t))/rho_hx, mx(t) = bxh mx(t-1) + axh v0x
__global__ void k_cpml_adj_b(const AdjArgs a)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)a.X * a.Z)
        return;
    const int z = (int)(i / a.X), x = (int)(i - (int64_t)z * a.X);
    if (!inb(a.X, a.Z, x, z)) {
        a.l0x[i] = a.l0z[i] = 0.f;
        return;
    }
    const float lv1x = stagT(a.a0x, a.X, a.Z, x, z, 1, 0, 1) / a.c.dx;
    const float tx = a.lmx[i] + lv1x / a.c.rho_hx[i];
    a.l0x[i] = lv1x / (a.c.Kxh[x] * a.c.rho_hx[i]) + a.c.axh[x] * tx;
    a.lmx[i] = a.c.bxh[x] * tx;
    const float lv1z = stagT(a.a0z, a.X, a.Z, x, z, 0, 1, 1) / a.c.dz;
    const float tz = a.lmz[i] + lv1z / a.c.rho_hz[i];
    a.l0z[i] = lv1z / (a.c.Kzh[z] * a.c.rho_hz[i]) + a.c.azh[z] * tz;
    a.lmz[i] = a.c.bzh[z] * tz;
}

// v0x = D(P(t-1), off 0)/dx into the adjoint of P(t-1)
__global__ void k_cpml_adj_c(const AdjArgs a)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)a.X * a.Z)
        return;
    const int z = (int)(i / a.X), x = (int)(i - (int64_t)z * a.X);
    if (!inb(a.X, a.Z, x, z))
        return;
    a.LB[i] += stagT(a.l0x, a.X, a.Z, x, z, 1, 0, 0) / a.c.dx + stagT(a.l0z, a.X, a.Z, x, z, 0, 1, 0) / a.c.dz;
}

// the loss gradient of the traces at step t enters the adjoint of P(t)
__global__ void k_cpml_adj_g(float *LA, const float *g, int X, int Z, int T, int t, int nm, const int *mx,
                             const int *mz)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < nm && inb(X, Z, mx[n], mz[n]))
        atomicAdd(LA + (size_t)mz[n] * X + mx[n], g[(size_t)n * T + t]);
}

struct State {
    int X = 0, Z = 0, T = 0, ns = 0, nm = 0, ppe = 1;
    float dx = 1.f, dz = 1.f, dt = 1.f, dt2 = 1.f, qtpi = 1.f;
    int precision = 0;
    cudaStream_t st = nullptr;
    float *P = nullptr, *mx = nullptr, *mz = nullptr, *mxx = nullptr, *mzz = nullptr;
    float *cquad = nullptr, *kappa = nullptr, *rho_hx = nullptr, *rho_hz = nullptr;
    float *cx = nullptr;  // K a b, K_half a_half b_half along x: [6][X]
    float *cz = nullptr;  // the same along z: [6][Z]
    float *src = nullptr, *init = nullptr, *rec_d = nullptr, *rec_h = nullptr;
    int *sx = nullptr, *sz = nullptr, *pmx = nullptr, *pmz = nullptr;
    int cap_src = 0;
    int *idx_dev = nullptr, *idx_h = nullptr;  // idx_source of the current call (device / pinned host)
    // the forward time loop captured as a CUDA graph, for the source count it
    // was captured with (set_source may change it)
    cudaGraphExec_t sim_graph = nullptr;
    int sim_graph_ns = -1;
    float inv_dx = 0.f, inv_dz = 0.f;  // exact reciprocals of power-of-two spacings, else 0
    int k_one = 0;                     // K profiles that are exactly 1 (bits Kx, Kxh, Kz, Kzh)
    float *gbuf = nullptr;  // gradient work buffers, kept between calls
    size_t gbuf_floats = 0;
    // every source as its own shot in one launch per step: per shot P [4]
    // slots, mx, mz [2], mxx, mzz (10 fields of Z*X), traces [shot][nm][T]
    float *bfields = nullptr, *brec = nullptr;
    int b_shots = 0;
    cudaGraphExec_t batch_graph = nullptr;

    void release()
    {
        if (batch_graph)
            cudaGraphExecDestroy(batch_graph);
        if (bfields)
            cudaFree(bfields);
        if (brec)
            cudaFree(brec);
        if (gbuf)
            cudaFree(gbuf);
        if (sim_graph)
            cudaGraphExecDestroy(sim_graph);
        if (idx_dev)
            cudaFree(idx_dev);
        if (idx_h)
            cudaFreeHost(idx_h);
        float *f[] = {P, mx, mz, mxx, mzz, cquad, kappa, rho_hx, rho_hz, cx, cz, src, init, rec_d};
        for (float *p : f)
            if (p)
                cudaFree(p);
        int *ip[] = {sx, sz, pmx, pmz};
        for (int *p : ip)
            if (p)
                cudaFree(p);
        if (rec_h)
            cudaFreeHost(rec_h);
        if (st)
            cudaStreamDestroy(st);
        *this = State();
        (void)cudaGetLastError();
    }
};

static State g;

static int env_int(const char *name, int dflt)
{
    const char *v = std::getenv(name);
    return v && *v ? std::atoi(v) : dflt;
}

static bool valid_points(int n, const int *x, const int *z, int X, int Z, bool interior)
{
    for (int k = 0; k < n; k++) {
        if (x[k] < 0 || z[k] < 0 || x[k] >= X || z[k] >= Z)
            return false;
        if (interior && !(x[k] >= 4 && z[k] >= 4 && x[k] < X - 4 && z[k] < Z - 4))
            return false;
    }
    return true;
}

static int init(int X, int Z, int T, int ns, int nm, int ppe, const int *ps_x, const int *ps_z, const int *pm_x,
                const int *pm_z, float dx, float dz, float dt, float dt2, float qtpi, const float *cq,
                const float *kp, const float *rhx, const float *rhz, const float *const *cx6,
                const float *const *cz6, const float *src, const float *init_h)
{
    g.release();
    clear_error();
    OTF_CHECK(X >= 9 && Z >= 9 && T >= 1, 1, "cpml init_memory_sim: grid or T too small");
    OTF_CHECK(ns >= 0 && nm >= 0, 1, "cpml init_memory_sim: negative point count");
    OTF_CHECK(valid_points(ns, ps_x, ps_z, X, Z, true), 1,
              "cpml init_memory_sim: sources must lie in 4 <= x < X-4, 4 <= z < Z-4");
    OTF_CHECK(valid_points(nm, pm_x, pm_z, X, Z, false), 1, "cpml init_memory_sim: receiver outside the grid");
    g.X = X;
    g.Z = Z;
    g.T = T;
    g.ns = ns;
    g.nm = nm;
    g.ppe = ppe;
    g.dx = dx;
    g.dz = dz;
    g.dt = dt;
    g.dt2 = dt2;
    g.qtpi = qtpi;
    g.precision = env_int("OTFWI_PRECISION", 0);
    const size_t XZ = (size_t)X * Z;
    OTF_CUDA(cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking));
    OTF_CUDA(cudaMalloc(&g.P, 4 * XZ * sizeof(float)));
    OTF_CUDA(cudaMalloc(&g.mx, 2 * XZ * sizeof(float)));
    OTF_CUDA(cudaMalloc(&g.mz, 2 * XZ * sizeof(float)));
    OTF_CUDA(cudaMalloc(&g.mxx, XZ * sizeof(float)));
    OTF_CUDA(cudaMalloc(&g.mzz, XZ * sizeof(float)));
    OTF_CUDA(cudaMalloc(&g.cquad, XZ * sizeof(float)));
    OTF_CUDA(cudaMalloc(&g.kappa, XZ * sizeof(float)));
    OTF_CUDA(cudaMalloc(&g.rho_hx, XZ * sizeof(float)));
    OTF_CUDA(cudaMalloc(&g.rho_hz, XZ * sizeof(float)));
    OTF_CUDA(cudaMalloc(&g.cx, 6 * (size_t)X * sizeof(float)));
    OTF_CUDA(cudaMalloc(&g.cz, 6 * (size_t)Z * sizeof(float)));
    OTF_CUDA(cudaMalloc(&g.init, 2 * XZ * sizeof(float)));
    OTF_CUDA(cudaMalloc(&g.rec_d, std::max<size_t>(1, (size_t)nm * T) * sizeof(float)));
    OTF_CUDA(cudaMallocHost(&g.rec_h, std::max<size_t>(1, (size_t)nm * T) * sizeof(float)));
    g.cap_src = std::max(ns, 1);
    OTF_CUDA(cudaMalloc(&g.src, (size_t)g.cap_src * T * sizeof(float)));
    OTF_CUDA(cudaMalloc(&g.sx, g.cap_src * sizeof(int)));
    OTF_CUDA(cudaMalloc(&g.sz, g.cap_src * sizeof(int)));
    OTF_CUDA(cudaMalloc(&g.idx_dev, sizeof(int)));
    OTF_CUDA(cudaMallocHost(&g.idx_h, sizeof(int)));
    OTF_CUDA(cudaMalloc(&g.pmx, std::max(nm, 1) * sizeof(int)));
    OTF_CUDA(cudaMalloc(&g.pmz, std::max(nm, 1) * sizeof(int)));
    OTF_CUDA(cudaMemcpy(g.cquad, cq, XZ * sizeof(float), cudaMemcpyHostToDevice));
    OTF_CUDA(cudaMemcpy(g.kappa, kp, XZ * sizeof(float), cudaMemcpyHostToDevice));
    OTF_CUDA(cudaMemcpy(g.rho_hx, rhx, XZ * sizeof(float), cudaMemcpyHostToDevice));
    OTF_CUDA(cudaMemcpy(g.rho_hz, rhz, XZ * sizeof(float), cudaMemcpyHostToDevice));
    for (int k = 0; k < 6; k++) {
        OTF_CUDA(cudaMemcpy(g.cx + (size_t)k * X, cx6[k], X * sizeof(float), cudaMemcpyHostToDevice));
        OTF_CUDA(cudaMemcpy(g.cz + (size_t)k * Z, cz6[k], Z * sizeof(float), cudaMemcpyHostToDevice));
    }
    if (ns > 0) {
        OTF_CUDA(cudaMemcpy(g.src, src, (size_t)ns * T * sizeof(float), cudaMemcpyHostToDevice));
        OTF_CUDA(cudaMemcpy(g.sx, ps_x, ns * sizeof(int), cudaMemcpyHostToDevice));
        OTF_CUDA(cudaMemcpy(g.sz, ps_z, ns * sizeof(int), cudaMemcpyHostToDevice));
    }
    if (nm > 0) {
        OTF_CUDA(cudaMemcpy(g.pmx, pm_x, nm * sizeof(int), cudaMemcpyHostToDevice));
        OTF_CUDA(cudaMemcpy(g.pmz, pm_z, nm * sizeof(int), cudaMemcpyHostToDevice));
    }
    // divisions the step may replace exactly (see Coef)
    auto pow2_inv = [](float d) {
        int e = 0;
        const float m = std::frexp(d, &e);
        return (d > 0.f && m == 0.5f) ? std::ldexp(1.f, 1 - e) : 0.f;
    };
    g.inv_dx = pow2_inv(dx);
    g.inv_dz = pow2_inv(dz);
    auto all_one = [](const float *v, int n) {
        for (int k = 0; k < n; k++)
            if (v[k] != 1.f)
                return false;
        return true;
    };
    g.k_one = (all_one(cx6[0], X) ? 1 : 0) | (all_one(cx6[3], X) ? 2 : 0) | (all_one(cz6[0], Z) ? 4 : 0) |
              (all_one(cz6[3], Z) ? 8 : 0);
    if (init_h)
        OTF_CUDA(cudaMemcpy(g.init, init_h, 2 * XZ * sizeof(float), cudaMemcpyHostToDevice));
    else
        OTF_CUDA(cudaMemset(g.init, 0, 2 * XZ * sizeof(float)));
    return 0;
}

static void fill_args(StepArgs &a)
{
    const int X = g.X, Z = g.Z;
    a.X = X;
    a.Z = Z;
    a.c.Kx = g.cx;
    a.c.ax = g.cx + X;
    a.c.bx = g.cx + 2 * X;
    a.c.Kxh = g.cx + 3 * X;
    a.c.axh = g.cx + 4 * X;
    a.c.bxh = g.cx + 5 * X;
    a.c.Kz = g.cz;
    a.c.az = g.cz + Z;
    a.c.bz = g.cz + 2 * Z;
    a.c.Kzh = g.cz + 3 * Z;
    a.c.azh = g.cz + 4 * Z;
    a.c.bzh = g.cz + 5 * Z;
    a.c.kappa = g.kappa;
    a.c.rho_hx = g.rho_hx;
    a.c.rho_hz = g.rho_hz;
    a.c.dx = g.dx;
    a.c.dz = g.dz;
    a.c.inv_dx = g.inv_dx;
    a.c.inv_dz = g.inv_dz;
    a.c.k_one = g.k_one;
    a.c.dt2 = g.dt2;
    a.mxx = g.mxx;
    a.mzz = g.mzz;
    a.lap = nullptr;
    a.T = g.T;
    a.ns = g.ns;
    a.nm = g.nm;
    a.ppe = g.ppe;
    a.idx_dev = g.idx_dev;
    a.sx = g.sx;
    a.sz = g.sz;
    a.pmx = g.pmx;
    a.pmz = g.pmz;
    a.cquad = g.cquad;
    a.src = g.src;
    a.qtpi = g.qtpi;
    a.rec = nullptr;
    a.shot_stride = 0;
    a.batch = 0;
}

// P(0), P(1) from the initial field, every other slot and memory variable zero
static int reset_state()
{
    const size_t XZ = (size_t)g.X * g.Z;
    cudaStream_t st = g.st;
    OTF_CUDA(cudaMemsetAsync(g.P, 0, 4 * XZ * sizeof(float), st));
    OTF_CUDA(cudaMemcpyAsync(g.P, g.init, 2 * XZ * sizeof(float), cudaMemcpyDeviceToDevice, st));
    OTF_CUDA(cudaMemsetAsync(g.mx, 0, 2 * XZ * sizeof(float), st));
    OTF_CUDA(cudaMemsetAsync(g.mz, 0, 2 * XZ * sizeof(float), st));
    OTF_CUDA(cudaMemsetAsync(g.mxx, 0, XZ * sizeof(float), st));
    OTF_CUDA(cudaMemsetAsync(g.mzz, 0, XZ * sizeof(float), st));
    return 0;
}

// idx_source of the next launches, read by the step kernel from the device
static int set_idx(int idx)
{
    *g.idx_h = idx;
    OTF_CUDA(cudaMemcpyAsync(g.idx_dev, g.idx_h, sizeof(int), cudaMemcpyHostToDevice, g.st));
    return 0;
}

// one time step t >= 2: one launch computes P(t), adds the sources and, with
// rec, records the receivers (lap optional)
static void step(StepArgs &a, int t, float *lap, float *rec = nullptr)
{
    const size_t XZ = (size_t)g.X * g.Z;
    float *Pn = g.P + (size_t)(t % 4) * XZ;
    a.t = t;
    a.P1 = g.P + (size_t)((t + 3) % 4) * XZ;
    a.P2 = g.P + (size_t)((t + 2) % 4) * XZ;
    a.Pn = Pn;
    a.mx_in = g.mx + (size_t)((t + 1) % 2) * XZ;
    a.mz_in = g.mz + (size_t)((t + 1) % 2) * XZ;
    a.mx_out = g.mx + (size_t)(t % 2) * XZ;
    a.mz_out = g.mz + (size_t)(t % 2) * XZ;
    a.lap = lap;
    a.rec = rec;
    const dim3 grid((g.X + TX - 1) / TX, (g.Z + TZ - 1) / TZ);
    if (g.precision == 1)
        k_cpml_step<false><<<grid, NTH, 0, g.st>>>(a);
    else
        k_cpml_step<true><<<grid, NTH, 0, g.st>>>(a);
}

// the forward time loop: state reset, T-2 steps, the recording of every step
static int emit_forward()
{
    const int X = g.X, T = g.T;
    const size_t XZ = (size_t)X * g.Z;
    if (reset_state())
        return -1;
    StepArgs a;
    fill_args(a);
    for (int t = 0; t < T; t++) {
        if (t > 1)
            step(a, t, nullptr, g.nm > 0 ? g.rec_d : nullptr);
        else if (g.nm > 0)  // the initial field
            k_cpml_record<<<(g.nm + 127) / 128, 128, 0, g.st>>>(g.P + (size_t)(t % 4) * XZ, X, T, t, g.nm, g.pmx,
                                                                g.pmz, g.rec_d);
    }
    OTF_CUDA(cudaGetLastError());
    return 0;
}

// The forward loop is captured once (per source count) as a CUDA graph and
// replayed: three small launches per step on a 2D field are launch-bound
// when issued one by one.
static int simulate(int idx)
{
    OTF_CHECK(g.P != nullptr, 2, "cpml cuda_simulate2 called before init_memory_sim");
    const int T = g.T;
    cudaStream_t st = g.st;
    if (set_idx(idx))
        return -1;
    if (!g.sim_graph || g.sim_graph_ns != g.ns) {
        if (g.sim_graph)
            cudaGraphExecDestroy(g.sim_graph);
        g.sim_graph = nullptr;
        cudaGraph_t graph = nullptr;
        OTF_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        const int rc = emit_forward();
        const cudaError_t ec = cudaStreamEndCapture(st, &graph);
        if (rc) {
            if (graph)
                cudaGraphDestroy(graph);
            return -1;
        }
        OTF_CUDA(ec);
        const cudaError_t ei = cudaGraphInstantiate(&g.sim_graph, graph, 0);
        cudaGraphDestroy(graph);
        OTF_CUDA(ei);
        g.sim_graph_ns = g.ns;
    }
    OTF_CUDA(cudaGraphLaunch(g.sim_graph, st));
    if (g.nm > 0)
        OTF_CUDA(cudaMemcpyAsync(g.rec_h, g.rec_d, (size_t)g.nm * T * sizeof(float), cudaMemcpyDeviceToHost, st));
    OTF_CUDA(cudaStreamSynchronize(st));
    return 0;
}

// Every source as its own shot (ppe = 1), all shots in one launch per step
// (grid z = shot): the traces of cuda_simulate2(0, s) for every s, bit for
// bit, into rec_h [ns][nm][T]. The time loop is one graph, as in simulate.
static int simulate_all(float *rec_h)
{
    OTF_CHECK(g.P != nullptr, 2, "cpml simulate_all called before init_memory_sim");
    OTF_CHECK(g.ppe == 1, 1, "cpml simulate_all: one pixel per element only (each source its own shot)");
    OTF_CHECK(g.ns > 0, 1, "cpml simulate_all: no sources");
    const int X = g.X, T = g.T, S = g.ns;
    const size_t XZ = (size_t)X * g.Z, stride = 10 * XZ;
    cudaStream_t st = g.st;
    if (g.b_shots != S) {
        if (g.batch_graph)
            cudaGraphExecDestroy(g.batch_graph);
        g.batch_graph = nullptr;
        if (g.bfields)
            cudaFree(g.bfields);
        if (g.brec)
            cudaFree(g.brec);
        g.bfields = g.brec = nullptr;
        g.b_shots = 0;
        OTF_CUDA(cudaMalloc(&g.bfields, stride * S * sizeof(float)));
        OTF_CUDA(cudaMalloc(&g.brec, std::max<size_t>(1, (size_t)S * g.nm * T) * sizeof(float)));
        g.b_shots = S;
    }
    if (!g.batch_graph) {
        cudaGraph_t graph = nullptr;
        OTF_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        int rc = 0;
        // shot layout: P slots 0-3 | mx 0-1 | mz 0-1 | mxx | mzz
        float *P = g.bfields, *mx = P + 4 * XZ, *mz = mx + 2 * XZ, *mxx = mz + 2 * XZ, *mzz = mxx + XZ;
        for (int sh = 0; sh < S && rc == 0; sh++) {
            float *b = g.bfields + (size_t)sh * stride;
            if (cudaMemsetAsync(b, 0, stride * sizeof(float), st) != cudaSuccess ||
                cudaMemcpyAsync(b, g.init, 2 * XZ * sizeof(float), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
                rc = -1;
        }
        StepArgs a;
        fill_args(a);
        a.shot_stride = stride;
        a.batch = 1;
        a.mxx = mxx;
        a.mzz = mzz;
        const dim3 grid((X + TX - 1) / TX, (g.Z + TZ - 1) / TZ, S);
        for (int t = 0; t < T && rc == 0; t++) {
            if (t <= 1) {
                for (int sh = 0; sh < S && g.nm > 0; sh++)
                    k_cpml_record<<<(g.nm + 127) / 128, 128, 0, st>>>(
                        P + (size_t)sh * stride + (size_t)(t % 4) * XZ, X, T, t, g.nm, g.pmx, g.pmz,
                        g.brec + (size_t)sh * g.nm * T);
                continue;
            }
            a.t = t;
            a.P1 = P + (size_t)((t + 3) % 4) * XZ;
            a.P2 = P + (size_t)((t + 2) % 4) * XZ;
            a.Pn = P + (size_t)(t % 4) * XZ;
            a.mx_in = mx + (size_t)((t + 1) % 2) * XZ;
            a.mz_in = mz + (size_t)((t + 1) % 2) * XZ;
            a.mx_out = mx + (size_t)(t % 2) * XZ;
            a.mz_out = mz + (size_t)(t % 2) * XZ;
            a.rec = g.nm > 0 ? g.brec : nullptr;
            if (g.precision == 1)
                k_cpml_step<false><<<grid, NTH, 0, st>>>(a);
            else
                k_cpml_step<true><<<grid, NTH, 0, st>>>(a);
        }
        const cudaError_t el = cudaGetLastError();
        const cudaError_t ec = cudaStreamEndCapture(st, &graph);
        if (rc || el != cudaSuccess) {
            if (graph)
                cudaGraphDestroy(graph);
            OTF_CUDA(el);
            return -1;
        }
        OTF_CUDA(ec);
        const cudaError_t ei = cudaGraphInstantiate(&g.batch_graph, graph, 0);
        cudaGraphDestroy(graph);
        OTF_CUDA(ei);
    }
    OTF_CUDA(cudaGraphLaunch(g.batch_graph, st));
    if (g.nm > 0)
        OTF_CUDA(cudaMemcpyAsync(rec_h, g.brec, (size_t)S * g.nm * T * sizeof(float), cudaMemcpyDeviceToHost, st));
    OTF_CUDA(cudaStreamSynchronize(st));
    return 0;
}

// dL/dkappa of the forward map for dL/dtraces = g_h [nm][T]: forward keeping
// the full state after steps 1, 1+k, 1+2k, ...; then, per segment from the
// last, the forward recomputed from its checkpoint keeping lap(t), and the
// transposed steps backwards. The gradient is the exact adjoint of the
// forward the library computes (its FP32 Laplacians), summed in FP32.
static int gradient(int idx, int every, const float *g_h, float *grad_h)
{
    OTF_CHECK(g.P != nullptr, 2, "cpml gradient called before init_memory_sim");
    OTF_CHECK(every >= 1, 1, "cpml gradient: checkpoint interval must be >= 1");
    OTF_CHECK(g.T >= 3, 1, "cpml gradient: T must be at least 3");
    const int X = g.X, Z = g.Z, T = g.T;
    const size_t XZ = (size_t)X * Z;
    cudaStream_t st = g.st;
    const int n_ck = (T - 2 + every - 1) / every + 1;  // checkpoints at 1 + j*every <= T-1
    // work buffers carved from one allocation kept between calls (grown when
    // a call needs more): a per-call cudaMalloc / cudaFree of the checkpoints
    // costs more than the adjoint itself on small grids
    const size_t n_trace = std::max<size_t>(1, (size_t)g.nm * T);
    const size_t need = (size_t)n_ck * 6 * XZ + (size_t)every * XZ + 13 * XZ + n_trace;
    if (need > g.gbuf_floats) {
        if (g.gbuf)
            cudaFree(g.gbuf);
        g.gbuf = nullptr;
        g.gbuf_floats = 0;
        OTF_CUDA(cudaMalloc(&g.gbuf, need * sizeof(float)));
        g.gbuf_floats = need;
    }
    auto done = [&](int rc) { return rc; };
    float *cur = g.gbuf;
    auto carve = [&](size_t n) {
        float *p = cur;
        cur += n;
        return p;
    };
    float *ck = carve((size_t)n_ck * 6 * XZ), *lapb = carve((size_t)every * XZ);
    float *LA = carve(XZ), *LB = carve(XZ), *LC = carve(XZ), *lmx = carve(XZ), *lmz = carve(XZ);
    float *lmxx = carve(XZ), *lmzz = carve(XZ), *a0x = carve(XZ), *a0z = carve(XZ), *l0x = carve(XZ);
    float *l0z = carve(XZ), *grad = carve(XZ), *gd = carve(n_trace);
    if (set_idx(idx))
        return -1;
    auto save = [&](int j, int c) -> int {
        float *d = ck + (size_t)j * 6 * XZ;
        const float *src[6] = {g.P + (size_t)(c % 4) * XZ, g.P + (size_t)((c + 3) % 4) * XZ,
                               g.mx + (size_t)(c % 2) * XZ, g.mz + (size_t)(c % 2) * XZ, g.mxx, g.mzz};
        for (int k = 0; k < 6; k++)
            OTF_CUDA(cudaMemcpyAsync(d + k * XZ, src[k], XZ * sizeof(float), cudaMemcpyDeviceToDevice, st));
        return 0;
    };
    auto restore = [&](int j, int c) -> int {
        const float *s = ck + (size_t)j * 6 * XZ;
        float *dst[6] = {g.P + (size_t)(c % 4) * XZ, g.P + (size_t)((c + 3) % 4) * XZ,
                         g.mx + (size_t)(c % 2) * XZ, g.mz + (size_t)(c % 2) * XZ, g.mxx, g.mzz};
        for (int k = 0; k < 6; k++)
            OTF_CUDA(cudaMemcpyAsync(dst[k], s + k * XZ, XZ * sizeof(float), cudaMemcpyDeviceToDevice, st));
        return 0;
    };
    if (reset_state())
        return done(-1);
    StepArgs a;
    fill_args(a);
    for (int t = 1; t < T; t++) {
        if (t > 1)
            step(a, t, nullptr);
        if ((t - 1) % every == 0 && save((t - 1) / every, t))
            return done(-1);
    }
    if (g.nm > 0)
        OTF_CUDA(cudaMemcpyAsync(gd, g_h, (size_t)g.nm * T * sizeof(float), cudaMemcpyHostToDevice, st));
    for (float *p : {LA, LB, LC, lmx, lmz, lmxx, lmzz, grad})
        OTF_CUDA(cudaMemsetAsync(p, 0, XZ * sizeof(float), st));
    AdjArgs ad;
    ad.X = X;
    ad.Z = Z;
    ad.lmx = lmx;
    ad.lmz = lmz;
    ad.lmxx = lmxx;
    ad.lmzz = lmzz;
    ad.a0x = a0x;
    ad.a0z = a0z;
    ad.l0x = l0x;
    ad.l0z = l0z;
    ad.grad = grad;
    ad.c = a.c;
    const unsigned nb = (unsigned)((XZ + 255) / 256);
    for (int j = n_ck - 1; j >= 0; j--) {
        const int c = 1 + j * every, end = std::min(c + every, T - 1);
        if (end <= c)
            continue;
        if (restore(j, c))
            return done(-1);
        for (int t = c + 1; t <= end; t++)
            step(a, t, lapb + (size_t)(t - c - 1) * XZ);
        for (int t = end; t > c; t--) {
            if (g.nm > 0)
                k_cpml_adj_g<<<(g.nm + 127) / 128, 128, 0, st>>>(LA, gd, X, Z, T, t, g.nm, g.pmx, g.pmz);
            ad.LA = LA;
            ad.LB = LB;
            ad.LC = LC;
            ad.lap = lapb + (size_t)(t - c - 1) * XZ;
            k_cpml_adj_a<<<nb, 256, 0, st>>>(ad);
            k_cpml_adj_b<<<nb, 256, 0, st>>>(ad);
            k_cpml_adj_c<<<nb, 256, 0, st>>>(ad);
            float *tmp = LA;  // P(t-1) becomes the current state
            LA = LB;
            LB = LC;
            LC = tmp;
        }
    }
    OTF_CUDA(cudaGetLastError());
    OTF_CUDA(cudaMemcpyAsync(grad_h, grad, XZ * sizeof(float), cudaMemcpyDeviceToHost, st));
    OTF_CUDA(cudaStreamSynchronize(st));
    return done(0);
}

}  // namespace cpml
}  // namespace otf

using otf::cpml::g;

extern "C" {

void def_python_adj(void *fn) { (void)fn; }

void init_memory_sim(int x, int z, int t, int ns, int nm, int ppe, int *ps_x, int *ps_z, int *pm_x, int *pm_z,
                     float dx_h, float dz_h, float dt_h, float dt2_h, float qtpi_h, float *cq, float *kp_unr,
                     float *rho_h, float *rho_hx_h, float *rho_hz_h, float *d_x_h, float *K_x_h,
                     float *alpha_x_h, float *a_x_h, float *b_x_h, float *d_x_half_h, float *K_x_half_h,
                     float *alpha_x_half_h, float *a_x_half_h, float *b_x_half_h, float *d_z_h, float *K_z_h,
                     float *alpha_z_h, float *a_z_h, float *b_z_h, float *d_z_half_h, float *K_z_half_h,
                     float *alpha_z_half_h, float *a_z_half_h, float *b_z_half_h, float *src, float *init,
                     float **rec)
{
    (void)rho_h;
    (void)d_x_h;
    (void)alpha_x_h;
    (void)d_x_half_h;
    (void)alpha_x_half_h;
    (void)d_z_h;
    (void)alpha_z_h;
    (void)d_z_half_h;
    (void)alpha_z_half_h;
    const float *cx6[6] = {K_x_h, a_x_h, b_x_h, K_x_half_h, a_x_half_h, b_x_half_h};
    const float *cz6[6] = {K_z_h, a_z_h, b_z_h, K_z_half_h, a_z_half_h, b_z_half_h};
    if (otf::cpml::init(x, z, t, ns, nm, ppe, ps_x, ps_z, pm_x, pm_z, dx_h, dz_h, dt_h, dt2_h, qtpi_h, cq, kp_unr,
                        rho_hx_h, rho_hz_h, cx6, cz6, src, init) == 0 &&
        rec)
        *rec = g.rec_h;
}

void setCquad(float *cq)
{
    if (!g.cquad) {
        otf::set_error_msg(2, "cpml setCquad called before init_memory_sim");
        return;
    }
    const cudaError_t e = cudaMemcpy(g.cquad, cq, (size_t)g.X * g.Z * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess)
        otf::set_error((int)e, "cpml setCquad", __FILE__, __LINE__);
}

void set_source(int ns, int *ps_x, int *ps_z)
{
    if (!g.sx) {
        otf::set_error_msg(2, "cpml set_source called before init_memory_sim");
        return;
    }
    if (ns < 0 || ns > g.cap_src) {
        otf::set_error_msg(1, "cpml set_source: more sources than init_memory_sim allocated waveforms for");
        return;
    }
    if (!otf::cpml::valid_points(ns, ps_x, ps_z, g.X, g.Z, true)) {
        otf::set_error_msg(1, "cpml set_source: sources must lie in 4 <= x < X-4, 4 <= z < Z-4");
        return;
    }
    g.ns = ns;
    if (g.batch_graph) {  // captured for the previous source set
        cudaGraphExecDestroy(g.batch_graph);
        g.batch_graph = nullptr;
    }
    if (ns > 0 && (cudaMemcpy(g.sx, ps_x, ns * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
                   cudaMemcpy(g.sz, ps_z, ns * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess))
        otf::set_error_msg(2, "cpml set_source: copy failed");
}

void cuda_simulate2(int en_out, int idx_source)
{
    (void)en_out;
    otf::cpml::simulate(idx_source);
}

int otf_last_status(void) { return otf::last_status(); }
const char *otf_last_error(void) { return otf::last_error(); }
void otf_clear_error(void) { otf::clear_error(); }
void otf_cpml_release(void) { g.release(); }

int otf_cpml_simulate_all(float *traces)
{
    otf::clear_error();
    return otf::cpml::simulate_all(traces);
}

int otf_cpml_gradient(const float *g_traces, float *grad_kappa, int checkpoint_every, int idx_source)
{
    otf::clear_error();
    return otf::cpml::gradient(idx_source, checkpoint_every, g_traces, grad_kappa);
}

}  // extern "C"
