"""Seeded synthetic ultrasonic-NDT scenarios in the reference's conventions.

The reference configures runs through module globals in setups/setup*_OCNDT.py
(grid, PML, nondimensional velocity c*dt/dx, source and receiver masks, source
waveforms [n_src, T]). A ``Scenario`` carries the same quantities. Velocities
are nondimensionalised with CFL 0.4: dt = 0.4*dx/c_max, so c_nd = 0.4*c/c_max.
No external data is used; every model, waveform and array is generated from a
seed.
"""
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Scenario:
    X: int
    Z: int
    T: int
    PML: int
    c_true: np.ndarray          # nondimensional velocity [Z, X]
    c_start: np.ndarray         # starting model [Z, X]
    src_mask: np.ndarray        # bool [Z, X]
    rec_mask: np.ndarray        # bool [Z, X]
    source: np.ndarray          # [n_src, T] float32, rows in np.where(src_mask) order
    dx: float = 5e-5
    c_max: float = 5900.0
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def n_src(self):
        return int(self.src_mask.sum())

    @property
    def n_rec(self):
        return int(self.rec_mask.sum())

    @property
    def dt(self):
        return 0.4 * self.dx / self.c_max

    def to_mps(self, c_nd):
        return np.asarray(c_nd) * self.c_max / 0.4

    def src_xz(self):
        z, x = np.where(self.src_mask)
        return x.astype(np.int32), z.astype(np.int32)

    def rec_xz(self):
        z, x = np.where(self.rec_mask)
        return x.astype(np.int32), z.astype(np.int32)


def ricker(T, f0_per_sample, t0_samples):
    """Ricker wavelet (1 - 2 a) exp(-a), a = (pi f0 (t - t0))^2, t in samples."""
    t = np.arange(T, dtype=np.float64)
    a = (np.pi * f0_per_sample * (t - t0_samples)) ** 2
    return (1.0 - 2.0 * a) * np.exp(-a)


def circle_defects(X, Z, c_bg, c_def, n_def, rmin, rmax, lo, hi, rng):
    c = np.full((Z, X), float(c_bg))
    zz, xx = np.mgrid[0:Z, 0:X]
    for _ in range(n_def):
        r = rng.integers(rmin, rmax + 1)
        cx = rng.uniform(lo, hi)
        cz = rng.uniform(lo, hi)
        c[(xx - cx) ** 2 + (zz - cz) ** 2 <= r * r] = c_def
    return c


def gaussian_smooth(a, sigma):
    """Separable Gaussian filter (truncated at 4 sigma, reflected edges)."""
    r = int(4 * sigma + 0.5)
    k = np.exp(-0.5 * (np.arange(-r, r + 1) / sigma) ** 2)
    k /= k.sum()
    out = np.asarray(a, np.float64)
    for ax in (0, 1):
        pad = [(0, 0), (0, 0)]
        pad[ax] = (r, r)
        p = np.pad(out, pad, mode="reflect")
        out = sum(k[i] * np.take(p, np.arange(i, i + out.shape[ax]), axis=ax) for i in range(2 * r + 1))
    return out


def heterogeneous_defects(X, Z, rng, n_def=8, c_bg=5900.0, v_lo=4000.0, v_hi=6300.0, amin=4, amax=14,
                          lo=None, hi=None, hetero=0.03, sigma=4.0):
    """Velocity model in m/s: background c_bg with Gaussian-smoothed random
    heterogeneity (sigma cells, +-hetero relative, peak-normalised) and n_def
    elliptical defects (semi-axes amin..amax cells, random orientation,
    velocities uniform in [v_lo, v_hi]) with centres uniform in [lo, hi]^2."""
    lo = 0.25 * min(X, Z) if lo is None else lo
    hi = 0.75 * min(X, Z) if hi is None else hi
    h = gaussian_smooth(rng.standard_normal((Z, X)), sigma)
    c = c_bg * (1.0 + hetero * h / np.abs(h).max())
    zz, xx = np.mgrid[0:Z, 0:X]
    for _ in range(n_def):
        a, b = rng.uniform(amin, amax, size=2)
        th = rng.uniform(0, np.pi)
        cx, cz = rng.uniform(lo, hi, size=2)
        u = (xx - cx) * np.cos(th) + (zz - cz) * np.sin(th)
        v = -(xx - cx) * np.sin(th) + (zz - cz) * np.cos(th)
        c[(u / a) ** 2 + (v / b) ** 2 <= 1.0] = rng.uniform(v_lo, v_hi)
    return c


def _array_masks(X, Z, xs, z, src_idx=None):
    rec = np.zeros((Z, X), dtype=bool)
    rec[z, xs] = True
    src = np.zeros((Z, X), dtype=bool)
    if src_idx is None:
        src[z, xs] = True
    else:
        src[z, np.asarray(xs)[src_idx]] = True
    return src, rec


def plain_single_shot(X=256, Z=256, T=1500, PML=20, n_rec=32, pitch=8, seed=0, f0_hz=5e6):
    """Plain single-shot forward + gradient case (256^2, T=1500, 1 source at
    the top-surface centre, 32 receivers at pitch 8, 3 circular defects at
    3000 m/s in 5900 m/s)."""
    rng = np.random.default_rng(seed)
    dx, c_max = 5e-5, 5900.0
    dt = 0.4 * dx / c_max
    lo, hi = PML + 25, min(X, Z) - PML - 25
    c = circle_defects(X, Z, 5900.0, 3000.0, 3, 5, 15, lo, hi, rng)
    zrow = PML + 6
    xs = 4 + pitch * np.arange(n_rec)
    xs = xs[xs < X]
    rec = np.zeros((Z, X), dtype=bool)
    rec[zrow, xs] = True
    src = np.zeros((Z, X), dtype=bool)
    src[zrow, X // 2] = True
    f0 = f0_hz * dt
    w = ricker(T, f0, 1.2 / f0)
    return Scenario(X, Z, T, PML, 0.4 * c / c_max, np.full((Z, X), 0.4), src, rec,
                    w[None, :].astype(np.float32), dx, c_max, "plain_single_shot")


def fmc(X=512, Z=512, T=4000, PML=20, n_elem=64, pitch=6, x_first=67, seed=0, f0_hz=5e6):
    """Full-matrix capture: a linear array at the top surface, every element
    both fires (one shot each) and receives (512^2, T=4000, 64 elements at
    pitch 6)."""
    rng = np.random.default_rng(seed)
    dx, c_max = 5e-5, 5900.0
    dt = 0.4 * dx / c_max
    lo, hi = PML + 25, min(X, Z) - PML - 25
    c = circle_defects(X, Z, 5900.0, 3000.0, 3, 5, 15, lo, hi, rng)
    zrow = PML + 6
    xs = x_first + pitch * np.arange(n_elem)
    src, rec = _array_masks(X, Z, xs, zrow)
    f0 = f0_hz * dt
    w = ricker(T, f0, 1.2 / f0).astype(np.float32)
    return Scenario(X, Z, T, PML, 0.4 * c / c_max, np.full((Z, X), 0.4), src, rec,
                    np.repeat(w[None, :], n_elem, axis=0), dx, c_max, "fmc")


def small(X=96, Z=80, T=400, PML=20, n_src=2, n_rec=8, seed=1, f0=0.04):
    """Small seeded case for parity tests (oracle runs it in about a second)."""
    rng = np.random.default_rng(seed)
    c = np.full((Z, X), 0.4)
    zz, xx = np.mgrid[0:Z, 0:X]
    for _ in range(2):
        cx, cz, r = rng.uniform(PML + 8, X - PML - 8), rng.uniform(PML + 12, Z - PML - 6), rng.uniform(3, 7)
        c[(xx - cx) ** 2 + (zz - cz) ** 2 <= r * r] = rng.uniform(0.2, 0.3)
    zrow = PML + 6
    xs = np.linspace(PML + 2, X - PML - 3, n_rec).round().astype(int)
    rec = np.zeros((Z, X), dtype=bool)
    rec[zrow, xs] = True
    src = np.zeros((Z, X), dtype=bool)
    sxs = np.linspace(PML + 8, X - PML - 9, n_src).round().astype(int)
    src[zrow + 1, sxs] = True
    w = np.stack([ricker(T, f0, 1.3 / f0 + 7 * i) for i in range(n_src)]).astype(np.float32)
    return Scenario(X, Z, T, PML, c, np.full((Z, X), 0.4), src, rec, w, name="small")
