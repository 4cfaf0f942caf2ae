"""FWI outer loop on the GPU.

The reference drives the inversion from regression.py:45-96: an objective
``objfun(c) = (1e3 * mse, grad_scale * gmask * grad)`` over
``Cuda_interface_PML.calc_grad`` (per-shot loop, host misfit), minimised by
scipy's L-BFGS-B with bounds [vmin, vmax], with the model misfit
``|c - c_true|^2 / (Nz*Nx)`` recorded per iteration. Here:

- ``Problem`` holds the acquisition, the true model (for synthetic observed
  data and error tracking) and one ``ShotBatch`` per frequency band; every
  gradient is one CUDA-graph replay of all shots with the misfit on the GPU;
- ``objfun`` / ``lbfgsb`` are the reference's objective and optimiser over
  that batch (one D2H of the gradient per evaluation instead of per shot);
- ``descent`` is gradient descent with a bracketing parabolic line search,
  the model, gradient and update staying on the GPU; each line-search trial
  is a forward-only evaluation (``ShotBatch.objective``);
- ``descent`` with a ``proposer`` (the learned preconditioner) first tries
  the proposed update and keeps it only if the misfit decreases, otherwise
  it takes the plain line-search step from the same gradient;
- with a process group of several ranks (one per GPU), each band's shots
  are split over the ranks (``distributed.ShardedShots``): every rank models
  and back-propagates its own block of shots, and one all-reduce per
  gradient (and per line-search evaluation) gives every rank the same
  gradient and misfit, so the model updates stay identical on all ranks.
Models are nondimensional velocities c*dt/dx, as the reference's ABI takes.
"""
import time
from dataclasses import dataclass, field

import numpy as np

from .batch import ShotBatch
from .scenarios import ricker


@dataclass
class Band:
    f0_hz: float
    iters: int


@dataclass
class History:
    """Per accepted iterate: wall time since start (s), total misfit, RMS
    velocity error (m/s), forward-equivalent evaluations, and whether the
    learned proposal was accepted."""
    t: list = field(default_factory=list)
    misfit: list = field(default_factory=list)
    rms: list = field(default_factory=list)
    evals: list = field(default_factory=list)
    learned: list = field(default_factory=list)
    band: list = field(default_factory=list)

    def time_to(self, rms_target):
        """First wall time at which the RMS error is <= rms_target (None if never)."""
        for t, r in zip(self.t, self.rms):
            if r <= rms_target:
                return t
        return None


class Problem:
    """One inversion: scenario (grid, array, true and starting model), bands,
    misfit, gradient mask and bounds. Observed data of every band are modelled
    on the GPU from the true model (synthetic, noise-free)."""

    def __init__(self, sc, bands, misfit="wasserstein", shots=None, precision=1, gmask=None, vmin=None,
                 vmax=None, illum_every=8, group=None):
        import torch
        from .distributed import world_of
        self.torch = torch
        self.group = group
        self.world, self.rank = world_of(group)
        self.sc, self.bands, self.misfit = sc, list(bands), misfit
        self.shots, self.precision, self.illum_every = shots, precision, illum_every
        c_lo = float(min(sc.c_true.min(), sc.c_start.min()))
        c_hi = float(max(sc.c_true.max(), sc.c_start.max()))
        self.vmin = 0.9 * c_lo if vmin is None else vmin
        self.vmax = 1.1 * c_hi if vmax is None else vmax
        if gmask is None:
            gmask = default_gmask(sc)
        self.gmask = torch.as_tensor(np.asarray(gmask, np.float32)).cuda()
        self.c_true = torch.as_tensor(np.asarray(sc.c_true, np.float32)).cuda()
        self._batches = {}
        self._illum = {}

    def wavelets(self, f0_hz):
        sc = self.sc
        f0 = f0_hz * sc.dt
        w = ricker(sc.T, f0, 1.2 / f0).astype(np.float32)
        return np.repeat(w[None, :], sc.n_src, axis=0)

    def batch(self, b):
        """ShotBatch of band b with its observed data set (with several
        ranks: this rank's block of the shots behind a ShardedShots)."""
        if b not in self._batches:
            sc = self.sc
            wav = self.wavelets(self.bands[b].f0_hz)
            if self.world > 1:
                from .batch import fmc_shots
                from .distributed import ShardedShots
                ptr, srcs = self.shots if self.shots is not None else fmc_shots(sc.n_src)
                sb = ShardedShots(lambda shots: ShotBatch(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, wav,
                                                          shots=shots, precision=self.precision),
                                  ptr, srcs, (sc.Z, sc.X), group=self.group,
                                  device=self.torch.device("cuda", self.torch.cuda.current_device()))
                n_local = sb.n_local
                n_rec = int(sc.n_rec)
            else:
                sb = ShotBatch(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, wav, shots=self.shots,
                               precision=self.precision)
                n_local, n_rec = sb.n_shots, sb.n_rec
            sb.set_model(self.c_true)
            obs = self.torch.empty((n_local, n_rec, sc.T), dtype=self.torch.float32, device="cuda")
            if n_local > 0:
                sb.forward(out=obs)
                sb.set_observed(obs)
            sb._obs_dev = obs
            self._batches[b] = sb
        return self._batches[b]

    def illumination(self, b, c):
        """Source illumination of band b at model c (computed once per band)."""
        if b not in self._illum:
            sb = self.batch(b)
            sb.set_model(c)
            out = self.torch.empty((self.sc.Z, self.sc.X), dtype=self.torch.float32, device="cuda")
            sb.illumination(self.illum_every, out=out)
            self._illum[b] = out
        return self._illum[b]

    def gradient(self, b, c):
        """(shot-mean gradient [Z, X] device, total misfit float) at model c."""
        torch = self.torch
        sb = self.batch(b)
        sb.set_model(c)
        g = torch.empty((self.sc.Z, self.sc.X), dtype=torch.float32, device="cuda")
        m = torch.empty(1, dtype=torch.float64, device="cuda")
        sb.gradient(self.misfit, grad=g, misfit_out=m)
        return g, float(m.item())

    def objective(self, b, c):
        sb = self.batch(b)
        sb.set_model(c)
        return sb.objective(self.misfit)

    def rms(self, c):
        """RMS velocity error in m/s over the inverted region (gmask > 0)."""
        d = (c - self.c_true) * float(self.sc.c_max / 0.4) * self.gmask
        return float(self.torch.sqrt(self.torch.sum(d * d) / self.gmask.sum()).item())

    def clip(self, c):
        return self.torch.clamp(c, self.vmin, self.vmax)


def default_gmask(sc):
    """1 on the central rectangle of half the grid's height and width, 0
    elsewhere, as the reference's setups draw it
    (setups/setup1_OCNDT.py:82-84)."""
    m = np.zeros((sc.Z, sc.X), np.float32)
    m[sc.Z // 4:sc.Z - sc.Z // 4, sc.X // 4:sc.X - sc.X // 4] = 1.0
    return m


def line_search(prob, b, c, d, J0, alpha0, max_evals=6):
    """Bracketing parabolic line search along direction d (device, max|d| = 1)
    from J(c) = J0: expand / shrink from alpha0 until a decrease is bracketed,
    then one parabolic step. Returns (alpha, J, evals); alpha 0 when no
    decrease was found."""
    pts = [(0.0, J0)]

    def f(a):
        return prob.objective(b, prob.clip(c + a * d))

    a1 = alpha0
    J1 = f(a1)
    pts.append((a1, J1))
    evals = 1
    if J1 < J0:
        a2 = 2 * a1
        J2 = f(a2)
        evals += 1
        pts.append((a2, J2))
        while J2 < J1 and evals < max_evals:
            a1, J1 = a2, J2
            a2 = 2 * a1
            J2 = f(a2)
            evals += 1
            pts.append((a2, J2))
        lo, mid, hi = (a1 / 2 if a1 > alpha0 else 0.0), a1, a2
    else:
        a2 = a1
        while J1 >= J0 and evals < max_evals:
            a2 = a1
            a1 = a1 / 2
            J1 = f(a1)
            evals += 1
            pts.append((a1, J1))
        if J1 >= J0:
            return 0.0, J0, evals
        lo, mid, hi = 0.0, a1, a2
    Jd = dict(pts)
    flo, fmid, fhi = Jd.get(lo, J0), Jd[mid], Jd[hi]
    den = (mid - lo) * (fmid - fhi) - (mid - hi) * (fmid - flo)
    best_a, best_J = min(pts, key=lambda p: p[1])
    if den != 0:
        a_star = mid - 0.5 * ((mid - lo) ** 2 * (fmid - fhi) - (mid - hi) ** 2 * (fmid - flo)) / den
        if lo < a_star < hi and abs(a_star - best_a) > 1e-3 * best_a:
            Js = f(a_star)
            evals += 1
            if Js < best_J:
                best_a, best_J = a_star, Js
    return best_a, best_J, evals


def descent(prob, c0, proposer=None, alpha0=None, on_step=None, on_iter=None, proposal_scales=(1.0, 0.5)):
    """Gradient descent with line search over the bands (the model stays on
    the GPU). With ``proposer(prob, band, c, g, J)`` -> update (device) the
    proposal is tried first, at each of ``proposal_scales`` in turn, and
    accepted only if the misfit decreases; the plain step is the fallback. ``on_step(b, it, c, g, J)`` is called with
    every gradient, ``on_iter(b, it, c_new, g, J_old, J_new)`` after every
    accepted step. Returns (c, History); timing is wall clock with the device
    synchronised at every accepted iterate."""
    torch = prob.torch
    c = prob.clip(torch.as_tensor(np.asarray(c0, np.float32)).cuda().clone())
    h = History()
    # the library's calls wait for their own stream; the model updates run on
    # this thread's torch stream: waiting for that one times an iterate
    # without stalling inversions that other threads run concurrently
    torch.cuda.current_stream().synchronize()
    t0 = time.perf_counter()
    evals_total = 0.0
    c_ref = float(c.mean().item())
    h.t.append(0.0)
    h.misfit.append(float("nan"))
    h.rms.append(prob.rms(c))
    h.evals.append(0.0)
    h.learned.append(False)
    h.band.append(0)
    for b, band in enumerate(prob.bands):
        alpha = alpha0 if alpha0 is not None else 0.05 * c_ref
        if proposer is not None:
            prob.illumination(b, c)
        for it in range(band.iters):
            g, J0 = prob.gradient(b, c)
            evals_total += 92.0 / 28.0  # a gradient costs 92/28 forward modellings
            if on_step is not None:
                on_step(b, it, c, g, J0)
            used_learned = False
            if proposer is not None:
                dc = proposer(prob, b, c, g, J0)
                for scale in proposal_scales:
                    cand = prob.clip(c + scale * dc)
                    Jc = prob.objective(b, cand)
                    evals_total += 1
                    if Jc < J0:
                        c, J_new, used_learned = cand, Jc, True
                        break
            if not used_learned:
                d = -g * prob.gmask
                gm = float(d.abs().max().item())
                if gm == 0:
                    break
                d = d / gm
                a, J_new, ne = line_search(prob, b, c, d, J0, alpha)
                evals_total += ne
                if a == 0.0:
                    alpha *= 0.25
                    continue
                c = prob.clip(c + a * d)
                alpha = a
            torch.cuda.current_stream().synchronize()
            h.t.append(time.perf_counter() - t0)
            h.misfit.append(J_new)
            h.rms.append(prob.rms(c))
            h.evals.append(evals_total)
            h.learned.append(used_learned)
            h.band.append(b)
            if on_iter is not None:
                on_iter(b, it, c, g, J0, J_new)
    return c, h


def objfun(prob, b, c_flat, grad_scale=1e-2):
    """regression.py:45-49 over the batched GPU gradient: (1e3 * mse, grad),
    mse = mean over shots of the per-shot misfit, grad = grad_scale * gmask *
    shot-mean gradient (host float64 for scipy)."""
    torch = prob.torch
    c = torch.as_tensor(np.asarray(c_flat, np.float32).reshape(prob.sc.Z, prob.sc.X)).cuda()
    g, J = prob.gradient(b, c)
    n_shots = prob.batch(b).n_shots
    grad = (grad_scale * prob.gmask * g).double().cpu().numpy().ravel()
    return 1e3 * J / n_shots, grad


def lbfgsb(prob, c0, b=0, maxiter=200, grad_scale=1e-2, callback=None):
    """scipy L-BFGS-B with bounds [vmin, vmax] and the reference's options
    (regression.py:82-87); returns (result, model misfit per iteration)."""
    from scipy.optimize import Bounds, minimize
    torch = prob.torch
    ct = prob.c_true.double().cpu().numpy()
    model_misfit = []

    def cb(x):
        model_misfit.append(float(np.linalg.norm(x.reshape(ct.shape) - ct) ** 2 / ct.size))
        if callback is not None:
            callback(x)

    opt = {"gtol": 1e-8, "ftol": 1e-8, "maxiter": maxiter, "maxcor": 20, "maxls": 10}
    r = minimize(lambda x: objfun(prob, b, x, grad_scale), np.asarray(c0, np.float64).ravel(), jac=True,
                 method="L-BFGS-B", bounds=Bounds(prob.vmin, prob.vmax), options=opt, callback=cb)
    return r, model_misfit
