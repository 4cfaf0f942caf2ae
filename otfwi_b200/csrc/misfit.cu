// Trace misfits and adjoint sources on the GPU, one CTA per trace.
//
//  kind 0  L2           adjoint_functions.py:8-11   J = sum r^2, adj = r = sim - obs
//  kind 1  Wasserstein  adjoint_functions.py:25-67  shift + rectangle normalisation,
//                       trapezoid CDFs, linear inverse CDFs (scipy 1.18 interp1d
//                       semantics, extrapolating; a non-monotone CDF is sorted
//                       stably first), W2 = sum (F^-1(t) - G^-1(t))^2,
//                       adj = 2 cumtrapz(t - G^-1(F(t))) - (its last value)
//  kind 2  Wasserstein on softplus-normalised traces (no reference counterpart):
//                       p = phi(f)/Z, phi = s softplus(./s), s = 0.1 max|obs|,
//                       same W2 and potential, adjoint through phi and Z
//  kind 3  wasserstein_quad  adjoint_functions.py:70-104 (squared traces)
//  kind 5  wasserstein_pm    adjoint_functions.py:144-223 with its negative-part
//                       CDFs built from the negative parts (the reference's
//                       lines 179-180 take the positive ones): positive and
//                       negative parts as two densities, W2 and transport
//                       potentials summed over both
//
// The reference evaluates kinds 0/1 in FP64 on the host. Here every
// accumulation (normalisation sums, the two CDF scans, the misfit sum, the
// potential scan) is a compensated FP32 "float-float" (hi + lo, about 44
// significant bits) block scan built from warp shuffles, which keeps the
// inverse-CDF positions at FP64-class accuracy without FP64 arithmetic.
// The CDF arrays live in a caller-provided scratch buffer in global memory.
#include <cuda_runtime.h>
#include <cstdint>
#include "otf_common.cuh"
#include "misfit.h"

namespace otf {
namespace {

constexpr int MT = 256;  // threads per trace CTA

struct FF {
    float hi, lo;
};

__device__ __forceinline__ FF ff(float a) { return {a, 0.f}; }
__device__ __forceinline__ FF ffd(double a)
{
    const float h = __double2float_rn(a);
    return {h, __double2float_rn(a - (double)h)};
}
__device__ __forceinline__ double ff2d(FF a) { return (double)a.hi + (double)a.lo; }
__device__ __forceinline__ FF two_sum(float a, float b)
{
    const float s = __fadd_rn(a, b);
    const float bb = __fsub_rn(s, a);
    const float e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
    return {s, e};
}
__device__ __forceinline__ FF quick_two_sum(float a, float b)
{
    const float s = __fadd_rn(a, b);
    return {s, __fsub_rn(b, __fsub_rn(s, a))};
}
__device__ __forceinline__ FF add(FF a, FF b)
{
    FF s = two_sum(a.hi, b.hi);
    FF t = two_sum(a.lo, b.lo);
    s.lo = __fadd_rn(s.lo, t.hi);
    s = quick_two_sum(s.hi, s.lo);
    s.lo = __fadd_rn(s.lo, t.lo);
    return quick_two_sum(s.hi, s.lo);
}
__device__ __forceinline__ FF neg(FF a) { return {-a.hi, -a.lo}; }
__device__ __forceinline__ FF sub(FF a, FF b) { return add(a, neg(b)); }
__device__ __forceinline__ FF mul(FF a, FF b)
{
    const float p = __fmul_rn(a.hi, b.hi);
    float e = __fmaf_rn(a.hi, b.hi, -p);
    e = __fmaf_rn(a.hi, b.lo, e);
    e = __fmaf_rn(a.lo, b.hi, e);
    return quick_two_sum(p, e);
}
__device__ __forceinline__ FF mulf(FF a, float b) { return mul(a, ff(b)); }
__device__ __forceinline__ FF div(FF a, FF b)
{
    const float q1 = __fdiv_rn(a.hi, b.hi);
    const FF r = sub(a, mulf(b, q1));
    const float q2 = __fdiv_rn(r.hi, b.hi);
    const FF r2 = sub(r, mulf(b, q2));
    const float q3 = __fdiv_rn(r2.hi, b.hi);
    FF q = quick_two_sum(q1, q2);
    return add(q, ff(q3));
}
__device__ __forceinline__ bool lt(FF a, FF b) { return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo); }

__device__ __forceinline__ FF shfl_up(FF v, int d)
{
    return {__shfl_up_sync(0xffffffffu, v.hi, d), __shfl_up_sync(0xffffffffu, v.lo, d)};
}
__device__ __forceinline__ FF shfl_xor(FF v, int d)
{
    return {__shfl_xor_sync(0xffffffffu, v.hi, d), __shfl_xor_sync(0xffffffffu, v.lo, d)};
}

// Compensated block sum; every thread gets the total.
__device__ FF block_sum(FF v, FF *red)
{
    for (int d = 16; d > 0; d >>= 1)
        v = add(v, shfl_xor(v, d));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0)
        red[w] = v;
    __syncthreads();
    FF t = l < (MT / 32) ? red[l] : FF{0.f, 0.f};
    for (int d = 16; d > 0; d >>= 1)
        t = add(t, shfl_xor(t, d));
    return t;
}

__device__ float block_minmax(float v, bool is_max, float *red)
{
    for (int d = 16; d > 0; d >>= 1) {
        const float o = __shfl_xor_sync(0xffffffffu, v, d);
        v = is_max ? fmaxf(v, o) : fminf(v, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0)
        red[w] = v;
    __syncthreads();
    float t = l < (MT / 32) ? red[l] : red[0];
    for (int d = 16; d > 0; d >>= 1) {
        const float o = __shfl_xor_sync(0xffffffffu, t, d);
        t = is_max ? fmaxf(t, o) : fminf(t, o);
    }
    return t;
}

// Inclusive compensated scan in place over out[0..T): thread k owns the
// contiguous chunk [k*C, min((k+1)*C, T)); term(i) gives the i-th summand.
template <class Term>
__device__ void block_scan(FF *out, int T, Term term, FF *red)
{
    const int C = (T + MT - 1) / MT;
    const int b = threadIdx.x * C, e = min(b + C, T);
    FF acc{0.f, 0.f};
    for (int i = b; i < e; i++) {
        acc = add(acc, term(i));
        out[i] = acc;
    }
    // warp-level inclusive scan of the chunk totals
    FF inc = acc;
    const int l = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int d = 1; d < 32; d <<= 1) {
        const FF o = shfl_up(inc, d);
        if (l >= d)
            inc = add(inc, o);
    }
    __syncthreads();
    if (l == 31)
        red[w] = inc;
    __syncthreads();
    FF off{0.f, 0.f};
    for (int k = 0; k < w; k++)
        off = add(off, red[k]);
    off = add(off, sub(inc, acc));  // exclusive prefix of this thread
    for (int i = b; i < e; i++)
        out[i] = add(out[i], off);
    __syncthreads();
}

// first j with x[j] >= q (numpy searchsorted 'left'), clipped to [1, T-1]
__device__ __forceinline__ int search_left(const FF *x, int T, FF q)
{
    int lo = 0, hi = T;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (lt(x[mid], q))
            lo = mid + 1;
        else
            hi = mid;
    }
    return min(max(lo, 1), T - 1);
}

// linear interpolation of y over x at q, interp1d's formula
__device__ __forceinline__ FF lerp(FF q, FF xlo, FF xhi, FF ylo, FF yhi)
{
    const FF den = sub(xhi, xlo);
    return add(mul(div(sub(q, xlo), den), yhi), mul(div(sub(xhi, q), den), ylo));
}

__device__ __forceinline__ double tval(int i, int T, double step)
{
    return i == T - 1 ? 1.0 : (double)i * step;  // numpy linspace(0, 1, T)
}

// log(1 + exp(y)) without overflow
__device__ __forceinline__ double softplus_unit(double y)
{
    return fmax(y, 0.0) + log1p(exp(-fabs(y)));
}

// Stable ascending sort of (key, index) pairs of length n (padded to a power
// of two with +inf keys) in global scratch, bitonic with index tie-break.
__device__ void block_sort(FF *key, int *idx, int n)
{
    int P = 1;
    while (P < n)
        P <<= 1;
    for (int i = n + threadIdx.x; i < P; i += MT) {
        key[i] = FF{__int_as_float(0x7f800000), 0.f};
        idx[i] = i;
    }
    __syncthreads();
    for (int k = 2; k <= P; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < P; i += MT) {
                const int p = i ^ j;
                if (p > i) {
                    const bool up = (i & k) == 0;
                    const FF a = key[i], b = key[p];
                    const bool a_gt = lt(b, a) || (!lt(a, b) && idx[i] > idx[p]);
                    if (a_gt == up) {
                        key[i] = b;
                        key[p] = a;
                        const int t = idx[i];
                        idx[i] = idx[p];
                        idx[p] = t;
                    }
                }
            }
            __syncthreads();
        }
    }
}

template <int KIND>
__global__ void __launch_bounds__(MT) k_wasserstein(const float *__restrict__ sim,
                                                     const float *__restrict__ obs,
                                                     float *__restrict__ adj,
                                                     double *__restrict__ misfit, char *scratch,
                                                     int T, int64_t per_trace)
{
    __shared__ FF red[MT / 32];
    __shared__ float redf[MT / 32];
    __shared__ int s_mono;
    const int tr = blockIdx.x;
    const float *f = sim + (int64_t)tr * T;
    const float *g = obs + (int64_t)tr * T;
    char *base = scratch + per_trace * tr;
    FF *Fs = reinterpret_cast<FF *>(base);
    FF *Gs = Fs + T;
    FF *Ws = Gs + T;
    int P = 1;
    while (P < T)
        P <<= 1;
    FF *Ks = Ws + T;
    int *Is = reinterpret_cast<int *>(Ks + P);

    const double step = 1.0 / (double)(T - 1);
    // per-trace transform parameters, from the observed trace only
    double c = 0.0, s = 1.0;
    float scale = 1.f;
    {
        float mn = __int_as_float(0x7f800000), mx = -mn, am = 0.f, af = 0.f;
        for (int i = threadIdx.x; i < T; i += MT) {
            mn = fminf(mn, g[i]);
            mx = fmaxf(mx, g[i]);
            am = fmaxf(am, fabsf(g[i]));
            af = fmaxf(af, fabsf(f[i]));
        }
        mn = block_minmax(mn, false, redf);
        mx = block_minmax(mx, true, redf);
        am = block_minmax(am, true, redf);
        af = block_minmax(af, true, redf);
        c = fmax(-1.1 * (double)mn, 0.1 * (double)mx);  // adjoint_functions.py:38-39
        s = am > 0.f ? 0.1 * (double)am : 1.0;
        if (KIND == 3)  // c = 0.05 max(obs^2) in FP32 (adjoint_functions.py:79)
            c = (double)__fmul_rn(__fmul_rn(am, am), 0.05f);
        // The normalisation p = f / sum(f dt) is scale-free, so the shifted
        // traces are brought to unit magnitude by an exact power of two:
        // float-float keeps FP64-class precision only for normal magnitudes.
        const double m = fmax(fmax((double)am, (double)af), fabs(c));
        if (m > 0.0 && m < 1e30)
            scale = ldexpf(1.f, -ilogb(m));
    }
    // densities up to a constant factor (scale for kind 1, 1/s for kind 2,
    // scale^2 for kind 3, whose observed density is the reference's FP32
    // obs^2 + c, adjoint_functions.py:76-82)
    const double cs = c * (double)scale;
    const float sc2 = scale * scale, c32 = (float)c;
    auto pf = [&](int i) -> FF {
        if (KIND == 3) {
            const FF x = ff(__fmul_rn(f[i], scale));
            return add(mul(x, x), ff(__fmul_rn(c32, sc2)));
        }
        return KIND == 1 ? add(ff(__fmul_rn(f[i], scale)), ffd(cs)) : ffd(softplus_unit((double)f[i] / s));
    };
    auto pg = [&](int i) -> FF {
        if (KIND == 3)
            return ff(__fmul_rn(__fadd_rn(__fmul_rn(g[i], g[i]), c32), sc2));
        return KIND == 1 ? add(ff(__fmul_rn(g[i], scale)), ffd(cs)) : ffd(softplus_unit((double)g[i] / s));
    };
    // normalisation: divide by sum(p * dt) (adjoint_functions.py:43-44)
    FF sf{0.f, 0.f}, sg{0.f, 0.f};
    for (int i = threadIdx.x; i < T; i += MT) {
        sf = add(sf, pf(i));
        sg = add(sg, pg(i));
    }
    const FF dtf = ffd(step);
    const FF Zf = mul(block_sum(sf, red), dtf);
    const FF Zg = mul(block_sum(sg, red), dtf);
    if (KIND == 3) {
        // rectangle CDFs cumsum(p dt); the observed density is normalised in
        // place in FP32 by the reference (adjoint_functions.py:82-86)
        block_scan(Gs, T, [&](int i) -> FF {
            return mul(ff(__double2float_rn(ff2d(div(pg(i), Zg)))), dtf);
        }, red);
        block_scan(Fs, T, [&](int i) -> FF { return mul(div(pf(i), Zf), dtf); }, red);
    } else {
        // trapezoid CDFs with x = t (cumulative_trapezoid(., t, initial=0))
        auto dti = [&](int i) { return ffd(tval(i, T, step) - tval(i - 1, T, step)); };
        block_scan(Gs, T, [&](int i) -> FF {
            if (i == 0) return FF{0.f, 0.f};
            return mulf(mul(dti(i), add(div(pg(i), Zg), div(pg(i - 1), Zg))), 0.5f);
        }, red);
        block_scan(Fs, T, [&](int i) -> FF {
            if (i == 0) return FF{0.f, 0.f};
            return mulf(mul(dti(i), add(div(pf(i), Zf), div(pf(i - 1), Zf))), 0.5f);
        }, red);
    }
    // F may be non-monotone (shifted simulated trace below zero): interp1d
    // then interpolates over the stably sorted (F, t) pairs
    if (threadIdx.x == 0)
        s_mono = 1;
    __syncthreads();
    for (int i = 1 + threadIdx.x; i < T; i += MT)
        if (lt(Fs[i], Fs[i - 1]))
            s_mono = 0;
    __syncthreads();
    const bool mono = s_mono != 0;
    if (!mono) {
        for (int i = threadIdx.x; i < T; i += MT) {
            Ks[i] = Fs[i];
            Is[i] = i;
        }
        __syncthreads();
        block_sort(Ks, Is, T);
    }
    const FF *Fx = mono ? Fs : Ks;
    // quantile differences, transport map and the misfit sum
    FF w2{0.f, 0.f};
    for (int i = threadIdx.x; i < T; i += MT) {
        const FF ti = ffd(tval(i, T, step));
        int j = search_left(Gs, T, ti);
        const FF g1 = lerp(ti, Gs[j - 1], Gs[j], ffd(tval(j - 1, T, step)), ffd(tval(j, T, step)));
        j = search_left(Fx, T, ti);
        const int jl = mono ? j - 1 : Is[j - 1], jh = mono ? j : Is[j];
        const FF f1 = lerp(ti, Fx[j - 1], Fx[j], ffd(tval(jl, T, step)), ffd(tval(jh, T, step)));
        const FF d = sub(f1, g1);
        w2 = add(w2, mul(d, d));
        j = search_left(Gs, T, Fs[i]);
        const FF gf = lerp(Fs[i], Gs[j - 1], Gs[j], ffd(tval(j - 1, T, step)), ffd(tval(j, T, step)));
        Ws[i] = sub(ti, gf);
    }
    w2 = block_sum(w2, red);
    __syncthreads();
    // potential: 2 * cumulative_trapezoid(v, initial=0) with unit spacing
    // (kind 3: 2 * cumsum(v) * dt, adjoint_functions.py:97)
    block_scan(Fs, T, [&](int i) -> FF {
        if (KIND == 3) return mul(mulf(Ws[i], 2.f), dtf);
        if (i == 0) return FF{0.f, 0.f};
        return add(Ws[i], Ws[i - 1]);  // 2 * (v_i + v_{i-1}) / 2
    }, red);
    const FF last = Fs[T - 1];
    float *a = adj + (int64_t)tr * T;
    if (KIND == 1 || KIND == 3) {
        for (int i = threadIdx.x; i < T; i += MT)
            a[i] = __double2float_rn(ff2d(sub(Fs[i], last)));
    } else {
        // centring under p and the chain rule through phi and Z
        FF m{0.f, 0.f};
        for (int i = threadIdx.x; i < T; i += MT)
            m = add(m, mul(sub(Fs[i], last), div(pf(i), Zf)));
        m = mul(block_sum(m, red), dtf);
        // Zf holds Z / s (densities were built as softplus(f/s))
        for (int i = threadIdx.x; i < T; i += MT) {
            const double sig = 0.5 * (1.0 + tanh(0.5 * (double)f[i] / s));
            a[i] = __double2float_rn(sig / (s * ff2d(Zf)) * ff2d(sub(sub(Fs[i], last), m)));
        }
    }
    if (threadIdx.x == 0)
        misfit[tr] = ff2d(w2);
}

// wasserstein_pm (kind 5): per part (positive, negative) the observed
// density max(0, +-obs) + c (c = 1% of the observed part's maximum, FP32 as
// NumPy keeps float32 * Python float) normalised in place in FP32, the
// simulated one max(0, +-sim) + c in FP64 class; rectangle CDFs cumsum(p dt);
// W2 = sum (F^-1(t) - G^-1(t))^2 over both parts; adjoint = the summed
// potentials cumsum(t - G^-1(F(t))) dt, less their last value. Every CDF is
// strictly increasing (c > 0), so no sort is needed.
__global__ void __launch_bounds__(MT) k_wasserstein_pm(const float *__restrict__ sim, const float *__restrict__ obs,
                                                       float *__restrict__ adj, double *__restrict__ misfit,
                                                       char *scratch, int T, int64_t per_trace)
{
    __shared__ FF red[MT / 32];
    __shared__ float redf[MT / 32];
    const int tr = blockIdx.x;
    const float *f = sim + (int64_t)tr * T;
    const float *g = obs + (int64_t)tr * T;
    FF *Fp = reinterpret_cast<FF *>(scratch + per_trace * tr);
    FF *Gp = Fp + T, *Fn = Gp + T, *Gn = Fn + T, *V = Gn + T;
    const double step = 1.0 / (double)(T - 1);
    float mp = 0.f, mn = 0.f, af = 0.f;
    for (int i = threadIdx.x; i < T; i += MT) {
        mp = fmaxf(mp, g[i]);
        mn = fmaxf(mn, -g[i]);
        af = fmaxf(af, fabsf(f[i]));
    }
    mp = block_minmax(mp, true, redf);
    mn = block_minmax(mn, true, redf);
    af = block_minmax(af, true, redf);
    const float cp = __fmul_rn(mp, 0.01f), cn = __fmul_rn(mn, 0.01f);
    // exact power-of-two scaling to unit magnitude (the densities are
    // normalised, so it cancels; float-float needs normal magnitudes)
    float scale = 1.f;
    {
        const double m = fmax(fmax((double)mp, (double)mn), (double)af);
        if (m > 0.0 && m < 1e30)
            scale = ldexpf(1.f, -ilogb(m));
    }
    const float cps = __fmul_rn(cp, scale), cns = __fmul_rn(cn, scale);
    auto gpv = [&](int i) { return __fmul_rn(__fadd_rn(fmaxf(g[i], 0.f), cp), scale); };
    auto gnv = [&](int i) { return __fmul_rn(__fadd_rn(fmaxf(-g[i], 0.f), cn), scale); };
    auto fpv = [&](int i) { return add(ff(__fmul_rn(fmaxf(f[i], 0.f), scale)), ff(cps)); };
    auto fnv = [&](int i) { return add(ff(__fmul_rn(fmaxf(-f[i], 0.f), scale)), ff(cns)); };
    FF sgp{0.f, 0.f}, sgn{0.f, 0.f}, sfp{0.f, 0.f}, sfn{0.f, 0.f};
    for (int i = threadIdx.x; i < T; i += MT) {
        sgp = add(sgp, ff(gpv(i)));
        sgn = add(sgn, ff(gnv(i)));
        sfp = add(sfp, fpv(i));
        sfn = add(sfn, fnv(i));
    }
    const FF dtf = ffd(step);
    const FF Zgp = mul(block_sum(sgp, red), dtf), Zgn = mul(block_sum(sgn, red), dtf);
    const FF Zfp = mul(block_sum(sfp, red), dtf), Zfn = mul(block_sum(sfn, red), dtf);
    block_scan(Gp, T, [&](int i) -> FF { return mul(ff(__double2float_rn(ff2d(div(ff(gpv(i)), Zgp)))), dtf); },
               red);
    block_scan(Gn, T, [&](int i) -> FF { return mul(ff(__double2float_rn(ff2d(div(ff(gnv(i)), Zgn)))), dtf); },
               red);
    block_scan(Fp, T, [&](int i) -> FF { return mul(div(fpv(i), Zfp), dtf); }, red);
    block_scan(Fn, T, [&](int i) -> FF { return mul(div(fnv(i), Zfn), dtf); }, red);
    auto inv = [&](const FF *C, FF q) {  // interp1d(C, t) at q
        const int j = search_left(C, T, q);
        return lerp(q, C[j - 1], C[j], ffd(tval(j - 1, T, step)), ffd(tval(j, T, step)));
    };
    FF w2p{0.f, 0.f}, w2n{0.f, 0.f};
    for (int i = threadIdx.x; i < T; i += MT) {
        const FF ti = ffd(tval(i, T, step));
        const FF dp = sub(inv(Fp, ti), inv(Gp, ti));
        const FF dn = sub(inv(Fn, ti), inv(Gn, ti));
        w2p = add(w2p, mul(dp, dp));
        w2n = add(w2n, mul(dn, dn));
        V[i] = add(sub(ti, inv(Gp, Fp[i])), sub(ti, inv(Gn, Fn[i])));
    }
    w2p = block_sum(w2p, red);
    w2n = block_sum(w2n, red);
    __syncthreads();
    block_scan(V, T, [&](int i) -> FF { return mul(V[i], dtf); }, red);
    const FF last = V[T - 1];
    float *a = adj + (int64_t)tr * T;
    for (int i = threadIdx.x; i < T; i += MT)
        a[i] = __double2float_rn(ff2d(sub(V[i], last)));
    if (threadIdx.x == 0)
        misfit[tr] = ff2d(w2p) + ff2d(w2n);
}

// L2: adj = sim - obs in FP64 rounded to FP32 (the reference's float64
// residual written into the FP32 adjoint buffer); misfit = sum r^2 in FP64.
__global__ void __launch_bounds__(MT) k_l2(const float *__restrict__ sim, const float *__restrict__ obs,
                                           float *__restrict__ adj, double *__restrict__ misfit, int T)
{
    __shared__ double red[MT / 32];
    const int tr = blockIdx.x;
    const float *f = sim + (int64_t)tr * T;
    const float *g = obs + (int64_t)tr * T;
    float *a = adj + (int64_t)tr * T;
    double acc = 0.0;
    for (int i = threadIdx.x; i < T; i += MT) {
        const double r = (double)f[i] - (double)g[i];
        a[i] = __double2float_rn(r);
        acc += r * r;
    }
    for (int d = 16; d > 0; d >>= 1)
        acc += __shfl_xor_sync(0xffffffffu, acc, d);
    if ((threadIdx.x & 31) == 0)
        red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < MT / 32; k++)
            s += red[k];
        misfit[tr] = s;
    }
}

}  // namespace

int64_t misfit_scratch_per_trace(int kind, int T)
{
    if (kind == kMisfitL2)
        return 0;
    if (kind == kMisfitQuadEnvelope)
        return envelope_scratch_per_trace(T);
    if (kind == kMisfitWassersteinPM)
        return ((int64_t)sizeof(FF) * 5 * T + 255) / 256 * 256;
    int64_t P = 1;
    while (P < T)
        P <<= 1;
    const int64_t bytes = (int64_t)sizeof(FF) * (3 * (int64_t)T + P) + (int64_t)sizeof(int) * P;
    return (bytes + 255) / 256 * 256;
}

int launch_misfit(int kind, const float *sim, const float *obs, float *adj, double *misfit,
                  int n_traces, int T, void *scratch, int64_t scratch_bytes, cudaStream_t st)
{
    OTF_CHECK(T >= 2, 1, "misfit: T must be at least 2");
    OTF_CHECK(n_traces >= 0, 1, "misfit: negative trace count");
    if (n_traces == 0)
        return 0;
    const int64_t per = misfit_scratch_per_trace(kind, T);
    OTF_CHECK(per * n_traces <= scratch_bytes, 1, "misfit: scratch buffer too small");
    switch (kind) {
    case kMisfitL2:
        k_l2<<<n_traces, MT, 0, st>>>(sim, obs, adj, misfit, T);
        break;
    case kMisfitWasserstein:
        k_wasserstein<1><<<n_traces, MT, 0, st>>>(sim, obs, adj, misfit, (char *)scratch, T, per);
        break;
    case kMisfitWassersteinSoftplus:
        k_wasserstein<2><<<n_traces, MT, 0, st>>>(sim, obs, adj, misfit, (char *)scratch, T, per);
        break;
    case kMisfitQuadEnvelope:
        return launch_envelope(sim, obs, adj, misfit, n_traces, T, scratch, st);
    case kMisfitWassersteinQuad:
        k_wasserstein<3><<<n_traces, MT, 0, st>>>(sim, obs, adj, misfit, (char *)scratch, T, per);
        break;
    case kMisfitWassersteinPM:
        k_wasserstein_pm<<<n_traces, MT, 0, st>>>(sim, obs, adj, misfit, (char *)scratch, T, per);
        break;
    default:
        OTF_CHECK(false, 1, "misfit: unknown kind");
    }
    OTF_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace otf

// ---------------------------------------------------------------------------
// Misfit without any device allocation.
//
// Some callers cannot allocate device memory at the moment they need a
// misfit: a host whose GPU memory is already fully reserved by another
// allocator (a framework that preallocates most of the device, so cudaMalloc
// fails), or a time-critical loop that must not pay for cudaMalloc/cudaFree,
// which can synchronise the whole device and stall other streams. For them
// the CDF scratch of the misfit kernel lives in the fixed array below,
// compiled into the library: every GPU that loads the library holds these
// 16 MiB until the process exits.
//
// Host code cannot use the array's name as a device address (in host code it
// names a host-side stand-in), so its device address is looked up with
// cudaGetSymbolAddress, with the device current, and remembered per device
// together with the id of the context it was looked up in: a context that
// was destroyed and made again (cudaDeviceReset, which the reference's own
// init_memory_sim calls) reloads the module and may place the array
// elsewhere, so a changed context id triggers a new lookup. The lookup is
// done by the first otf_misfit_noalloc call in each context; make that call
// before any stream capture. Under CUDA's default lazy module loading, the
// first use of this file's kernels or of the array in a context (this entry
// point's first call, or an earlier otf_misfit call) loads the module and
// places the 16 MiB array then: at that moment the device needs 16 MiB free
// (CUDA_MODULE_LOADING=EAGER places it when the context is created). All
// calls share the one array and it keeps whatever the last call left there;
// the kernel writes every scratch element it reads, so nothing has to be
// cleared between calls. Calls whose kernels may run at the same time on the
// GPU (different streams without ordering between them) race on the array:
// serialise them.
#include <cuda.h>
#include <mutex>
#include <string>

namespace {
constexpr long long kNoAllocScratchBytes = 16ll << 20;
static __device__ __align__(256) char g_noalloc_misfit_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
struct NoAllocSlot {
    unsigned long long ctx_id;
    void *addr;
};
NoAllocSlot g_noalloc_slot[kMaxDevices] = {};

// the driver's context queries, through the runtime (the library does not
// link the driver library itself, so that it loads on hosts without one)
int context_id(unsigned long long *id)
{
    using GetCurrent = CUresult (*)(CUcontext *);
    using GetId = CUresult (*)(CUcontext, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    if (!get_current || !get_id) {
        void *p = nullptr, *q = nullptr;
        cudaDriverEntryPointQueryResult r1, r2;
        OTF_CUDA(cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &r1));
        OTF_CUDA(cudaGetDriverEntryPoint("cuCtxGetId", &q, cudaEnableDefault, &r2));
        OTF_CHECK(p && q && r1 == cudaDriverEntryPointSuccess && r2 == cudaDriverEntryPointSuccess, 1,
                  "otf_misfit_noalloc: driver context queries unavailable");
        get_current = reinterpret_cast<GetCurrent>(p);
        get_id = reinterpret_cast<GetId>(q);
    }
    CUcontext ctx = nullptr;
    OTF_CHECK(get_current(&ctx) == CUDA_SUCCESS && ctx != nullptr, 1, "otf_misfit_noalloc: no current CUDA context");
    OTF_CHECK(get_id(ctx, id) == CUDA_SUCCESS, 1, "otf_misfit_noalloc: context id lookup failed");
    return 0;
}

// device address of the scratch array in the current context
int noalloc_scratch(void **out)
{
    int dev = -1;
    OTF_CUDA(cudaGetDevice(&dev));
    OTF_CHECK(dev >= 0 && dev < kMaxDevices, 1, "otf_misfit_noalloc: device index out of range");
    // make the device's primary context current (created if need be)
    OTF_CUDA(cudaSetDevice(dev));
    unsigned long long id = 0;
    if (context_id(&id))
        return -1;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoAllocSlot &s = g_noalloc_slot[dev];
    if (!s.addr || s.ctx_id != id) {
        void *p = nullptr;
        OTF_CUDA(cudaGetSymbolAddress(&p, g_noalloc_misfit_scratch));
        OTF_CHECK(p != nullptr, 1, "otf_misfit_noalloc: scratch address lookup returned null");
        s.addr = p;
        s.ctx_id = id;
    }
    *out = s.addr;
    return 0;
}
}  // namespace

extern "C" int otf_misfit_noalloc(int kind, const float *sim, const float *obs, float *adj,
                                  double *misfit, int n_traces, int T, void *stream)
{
    OTF_CHECK(T >= 2, 1, "otf_misfit_noalloc: T must be at least 2");
    OTF_CHECK(n_traces >= 0, 1, "otf_misfit_noalloc: negative trace count");
    OTF_CHECK(kind != otf::kMisfitQuadEnvelope, 1,
              "otf_misfit_noalloc: quad_envelope needs FFT plans, whose creation allocates; use otf_misfit");
    const long long need = (long long)otf::misfit_scratch_per_trace(kind, T) * n_traces;
    OTF_CHECK(need <= kNoAllocScratchBytes, 1,
              "otf_misfit_noalloc: " + std::to_string(n_traces) + " traces of " + std::to_string(T) +
                  " samples need " + std::to_string(need) +
                  " bytes of scratch, more than the built-in 16 MiB; split the traces over several "
                  "calls or use otf_misfit with your own scratch");
    void *scratch = nullptr;
    if (noalloc_scratch(&scratch))
        return -1;
    return otf::launch_misfit(kind, sim, obs, adj, misfit, n_traces, T, scratch,
                              kNoAllocScratchBytes, (cudaStream_t)stream);
}
