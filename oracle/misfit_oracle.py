"""CPU oracle for the trace misfits and their adjoint sources.

TEST INFRASTRUCTURE ONLY: the parity tests, smoke() and bench.py's
cpu_baseline / reference legs use it as the checker; the product path never
imports it.

Restates the reference's ``adjoint_functions.py`` (Otfwi project root):
  * ``L2``          adjoint_functions.py:8-11
  * ``wasserstein`` adjoint_functions.py:25-67 (the misfit regression.py:42 uses)
  * ``wasserstein_quad`` adjoint_functions.py:70-104, ``wasserstein_pm``
    adjoint_functions.py:144-223 (as written, and with its G_n / F_n lines
    taking the negative parts), ``quad_envelope`` adjoint_functions.py:14-22

The reference computes through two scipy routines that are not part of the
reference tree (scipy 1.18.1 is the version installed beside it). Their
published algorithms are restated here so the same arithmetic can be mirrored
on the GPU:
  * ``scipy.integrate.cumulative_trapezoid(y, x, initial=0)``:
        res = cumsum(diff(x) * (y[1:] + y[:-1]) / 2.0), prefixed by 0;
        with no x the spacing is the scalar 1.0;
  * ``scipy.interpolate.interp1d(x, y, kind='linear',
        fill_value='extrapolate')``: x is stably sorted (mergesort argsort);
        an evaluation point xn takes i = searchsorted(x, xn, 'left') clipped to
        [1, n-1], lo = i-1, hi = i, and returns
        ((xn - x_lo)/(x_hi - x_lo))*y_hi + ((x_hi - xn)/(x_hi - x_lo))*y_lo,
        extrapolating with the first / last segment.
The operations and their order are the reference's, so on the same inputs
this oracle reproduces the reference bit for bit (pinned by
tests/golden/misfit_*.npz, generated from the reference itself).
"""
import numpy as np


def cumtrapz0(y, x=None):
    """cumulative_trapezoid(y, x, initial=0) in float64."""
    y = np.asarray(y, dtype=np.float64)
    d = np.diff(np.asarray(x, dtype=np.float64)) if x is not None else 1.0
    res = np.cumsum(d * (y[1:] + y[:-1]) / 2.0)
    return np.concatenate((np.zeros(1, dtype=res.dtype), res))


class Interp1dLinear:
    """interp1d(x, y, kind='linear', fill_value='extrapolate', assume_sorted=False)."""

    def __init__(self, x, y):
        x = np.array(x, dtype=np.float64)
        y = np.array(y, dtype=np.float64)
        ind = np.argsort(x, kind="mergesort")
        self.x = x[ind]
        self.y = y[ind]

    def __call__(self, xn):
        xn = np.asarray(xn, dtype=np.float64)
        idx = np.searchsorted(self.x, xn).clip(1, len(self.x) - 1).astype(int)
        lo = idx - 1
        hi = idx
        x_lo = self.x[lo]
        x_hi = self.x[hi]
        y_lo = self.y[lo]
        y_hi = self.y[hi]
        return ((xn - x_lo) / (x_hi - x_lo)) * y_hi + ((x_hi - xn) / (x_hi - x_lo)) * y_lo


def L2(sim, obs):
    """adjoint_functions.py:8-11: J = sum (sim-obs)^2, adjoint = sim - obs."""
    resid = np.asarray(sim, dtype=np.float64) - obs
    mse = np.sum(resid ** 2)
    return mse, resid


def wasserstein_trace(sim_s, obs_s, t, dt):
    """One trace of adjoint_functions.py:33-64; returns (W2 term, adjoint row)."""
    f_gate = np.concatenate([np.zeros(0), np.asarray(sim_s)])
    g_gate = np.concatenate([np.zeros(0), np.asarray(obs_s)])
    c = -1.1 * np.min(g_gate)
    c = np.maximum(c, 0.1 * np.max(g_gate))
    g = g_gate + c
    f = f_gate + c
    g /= np.sum(g * dt)
    f /= np.sum(f * dt)
    G = cumtrapz0(g, t)
    F = cumtrapz0(f, t)
    F_i = Interp1dLinear(t, F)
    F_1 = Interp1dLinear(F, t)
    G_1 = Interp1dLinear(G, t)
    dist = Interp1dLinear(t, 2 * cumtrapz0(t - G_1(F_i(t))))
    adj = dist(t) - dist(1)
    w2 = sum(np.abs(F_1(t) - G_1(t)) ** 2)
    return w2, adj


def wasserstein(sim, obs):
    """adjoint_functions.py:25-67: per-trace quadratic Wasserstein misfit of
    shifted, rectangle-normalised traces and its adjoint source."""
    sim = np.asarray(sim)
    obs = np.asarray(obs)
    n_sens, T = sim.shape
    t = np.linspace(0, 1, T)
    dt = t[1] - t[0]
    W2 = 0
    s_W2 = np.zeros((n_sens, T))
    for s in range(n_sens):
        w2, adj = wasserstein_trace(sim[s], obs[s], t, dt)
        s_W2[s, :] = adj
        W2 += w2
    return W2, s_W2


def softplus_scale(obs_s):
    """Per-trace softplus width: one tenth of the observed trace's peak
    magnitude (the reference shift's 0.1*max(obs) scale); 1 for a zero trace."""
    m = float(np.max(np.abs(obs_s)))
    return 0.1 * m if m > 0 else 1.0


def softplus(x, s):
    """s * log(1 + exp(x / s)), overflow-safe."""
    y = np.asarray(x, np.float64) / s
    return s * (np.maximum(y, 0) + np.log1p(np.exp(-np.abs(y))))


def wasserstein_softplus_trace(sim_s, obs_s, t, dt):
    """Quadratic Wasserstein misfit of softplus-normalised traces (no
    counterpart in the reference, which shifts by a constant instead).

    Densities p = phi(f)/Z_f, q = phi(g)/Z_g with phi = softplus of width
    s = softplus_scale(obs); Z = sum(phi * dt). CDFs, inverse CDFs, the misfit
    sum((F^-1(t) - G^-1(t))^2) and the transport potential
    Phi = 2*cumtrapz(t - G^-1(F(t))) (unit spacing), Phi -= Phi[-1], follow
    the reference recipe (wasserstein_trace above). The adjoint source is the
    chain rule of p through the normalisation and phi:
        adj_i = phi'(f_i)/Z_f * (Phi_i - sum_k Phi_k p_k dt),
    phi'(x) = sigmoid(x / s)."""
    s = softplus_scale(obs_s)
    f_in = np.asarray(sim_s, np.float64)
    pf = softplus(f_in, s)
    pg = softplus(np.asarray(obs_s, np.float64), s)
    Zf = np.sum(pf * dt)
    Zg = np.sum(pg * dt)
    p = pf / Zf
    q = pg / Zg
    G = cumtrapz0(q, t)
    F = cumtrapz0(p, t)
    F_1 = Interp1dLinear(F, t)
    G_1 = Interp1dLinear(G, t)
    phi = 2 * cumtrapz0(t - G_1(F))
    phi = phi - phi[-1]
    w2 = sum(np.abs(F_1(t) - G_1(t)) ** 2)
    sig = 0.5 * (1.0 + np.tanh(0.5 * f_in / s))
    adj = sig / Zf * (phi - np.sum(phi * p * dt))
    return w2, adj


def wasserstein_softplus(sim, obs):
    """Per-trace softplus-normalised W2 over [n_traces, T]."""
    sim = np.asarray(sim)
    obs = np.asarray(obs)
    n_sens, T = sim.shape
    t = np.linspace(0, 1, T)
    dt = t[1] - t[0]
    W2 = 0.0
    out = np.zeros((n_sens, T))
    for s in range(n_sens):
        w2, adj = wasserstein_softplus_trace(sim[s], obs[s], t, dt)
        out[s] = adj
        W2 += w2
    return W2, out


def wasserstein_quad_trace(sim_s, obs_s, t, dt):
    """One trace of adjoint_functions.py:70-108 (wasserstein_quad): densities
    sim^2 + c and obs^2 + c with c = 0.05 max(obs^2), each keeping its input
    dtype as in the reference (the callback passes float64 sim and float32
    obs), rectangle-normalised, rectangle-rule CDFs (cumsum * dt); returns
    (W2 term, adjoint row)."""
    g = np.asarray(obs_s) ** 2
    f = np.asarray(sim_s) ** 2
    c = np.max(g) * 0.05
    g += c
    f += c
    g /= np.sum(g * dt)
    f /= np.sum(f * dt)
    G = np.cumsum(g * dt)
    F = np.cumsum(f * dt)
    F_i = Interp1dLinear(t, F)
    F_1 = Interp1dLinear(F, t)
    G_1 = Interp1dLinear(G, t)
    dist = Interp1dLinear(t, 2 * np.cumsum(t - G_1(F_i(t))) * dt)
    adj = dist(t) - dist(1)
    w2 = sum(np.abs(F_1(t) - G_1(t)) ** 2)
    return w2, adj


def wasserstein_quad(sim, obs):
    """adjoint_functions.py:70-108: Wasserstein misfit of squared traces."""
    sim = np.asarray(sim)
    obs = np.asarray(obs)
    n_sens, T = sim.shape
    t = np.linspace(0, 1, T)
    dt = t[1] - t[0]
    W2 = 0
    s_W2 = np.zeros((n_sens, T))
    for s in range(n_sens):
        w2, adj = wasserstein_quad_trace(sim[s], obs[s], t, dt)
        s_W2[s, :] = adj
        W2 += w2
    return W2, s_W2


def analytic_signal(x):
    """scipy.signal.hilbert(x) along the last axis: FFT, one-sided spectrum
    weights h (h[0] = 1, 2 on positive frequencies, h[N/2] = 1 for even N,
    0 on negative frequencies), inverse FFT."""
    x = np.asarray(x, dtype=np.float64)
    N = x.shape[-1]
    h = np.zeros(N)
    if N % 2 == 0:
        h[0] = h[N // 2] = 1
        h[1:N // 2] = 2
    else:
        h[0] = 1
        h[1:(N + 1) // 2] = 2
    return np.fft.ifft(np.fft.fft(x, axis=-1) * h, axis=-1)


def quad_envelope(sim, obs):
    """adjoint_functions.py:14-22: misfit sum((|H sim|^2 - |H obs|^2)^2) and
    adjoint sim * e - Im(H(e * Im(H sim))), e = |H sim|^2 - |H obs|^2, H the
    analytic signal."""
    hs = analytic_signal(sim)
    ho = analytic_signal(obs)
    e = np.abs(hs) ** 2 - np.abs(ho) ** 2
    adj = np.asarray(sim, np.float64) * e - np.imag(analytic_signal(e * np.imag(hs)))
    return np.sum(e ** 2), adj


def wasserstein_pm_trace(sim_s, obs_s, t, dt, fixed=True):
    """One trace of adjoint_functions.py:144-223 (wasserstein_pm): the positive
    and the negative parts of each trace as two densities, each shifted by 1%
    of the observed part's maximum, rectangle-normalised, rectangle-rule CDFs;
    misfit sum (F_p^-1 - G_p^-1)^2 + sum (F_n^-1 - G_n^-1)^2, adjoint the
    sum of the two transport potentials cumsum(t - G^-1(F(t))) dt, less its
    last value. The reference builds G_n and F_n from the POSITIVE parts
    (adjoint_functions.py:179-180), which makes the negative part vanish from
    the result; ``fixed=False`` reproduces that line as written, ``fixed=True``
    (the device misfit) uses the negative parts. Each operation keeps the
    reference's dtype: the observed parts are float32 and normalised in
    place, the simulated ones float64; the two misfit sums are Python sums."""
    g_p = np.maximum(0, obs_s)
    f_p = np.maximum(0, sim_s)
    g_n = -np.minimum(0, obs_s)
    f_n = -np.minimum(0, sim_s)
    c_p = np.max(g_p) * 0.01
    c_n = np.max(g_n) * 0.01
    g_p += c_p
    f_p += c_p
    g_n += c_n
    f_n += c_n
    mass_gp = np.sum(g_p * dt)
    mass_gn = np.sum(g_n * dt)
    mass_fp = np.sum(f_p * dt)
    mass_fn = np.sum(f_n * dt)
    g_p /= mass_gp
    g_n /= mass_gn
    f_p /= mass_fp
    f_n /= mass_fn
    G_p = np.cumsum(g_p * dt)
    F_p = np.cumsum(f_p * dt)
    G_n = np.cumsum((g_n if fixed else g_p) * dt)
    F_n = np.cumsum((f_n if fixed else f_p) * dt)
    F_ip = Interp1dLinear(t, F_p)
    G_1p = Interp1dLinear(G_p, t)
    F_1p = Interp1dLinear(F_p, t)
    F_in = Interp1dLinear(t, F_n)
    G_1n = Interp1dLinear(G_n, t)
    F_1n = Interp1dLinear(F_n, t)
    dist = Interp1dLinear(t, np.cumsum(t - G_1p(F_ip(t))) * dt + np.cumsum(t - G_1n(F_in(t))) * dt)
    adj = dist(t) - dist(t[-1])
    w2 = sum(np.abs(F_1p(t) - G_1p(t)) ** 2) + sum(np.abs(F_1n(t) - G_1n(t)) ** 2)
    return w2, adj


def wasserstein_pm(sim, obs, fixed=True):
    """adjoint_functions.py:144-223 over every trace (see wasserstein_pm_trace)."""
    sim = np.asarray(sim)
    obs = np.asarray(obs)
    n_sens, T = sim.shape
    t = np.linspace(0, 1, T)
    dt = t[1] - t[0]
    W2 = 0
    s_W2 = np.zeros((n_sens, T))
    for s in range(n_sens):
        w2, adj = wasserstein_pm_trace(sim[s].copy(), obs[s].copy(), t, dt, fixed)
        s_W2[s, :] = adj
        W2 += w2
    return W2, s_W2
