"""The reference's inversion result file.

After the optimiser, the reference's driver (regression.py:89-96) simulates
the recovered model once more, takes its L2 misfit against the observed data
(adjoint_functions.py:8-11, ``sum((sim - obs)**2)`` in the traces' FP32) and
pickles the list

    [recording, model, true model, xzm, xzs, vmin, vmax, fun, mseL2, model_misfit]

to ``output/regression_<name>.pickle``: the recording of every shot
([n_source, n_sensor, T] float32 with the multishot wrapper), the model
[Nz, Nx], the true model, the receiver and source masks, the bounds, the
final objective, that misfit and the per-iteration model misfit. ``save`` /
``load`` write and read that layout; ``finish`` does the driver's closing
steps for a ``fwi.Problem`` on the GPU (one batched forward of every shot).
"""
import os
import pickle

import numpy as np

FIELDS = ("recording", "model", "true_model", "xzm", "xzs", "vmin", "vmax", "fun", "mseL2", "model_misfit")


def save(path, recording, model, true_model, xzm, xzs, vmin, vmax, fun, mseL2, model_misfit):
    """Pickle the result list in the reference's order (regression.py:95-96)."""
    d = os.path.dirname(os.path.abspath(path))
    os.makedirs(d, exist_ok=True)
    with open(path, "wb") as f:
        pickle.dump([recording, model, true_model, xzm, xzs, vmin, vmax, fun, mseL2, model_misfit], f)


def load(path):
    """The result list of a reference or of this package as a dict keyed by FIELDS.

    The format is a pickle, as the reference writes it, and unpickling runs
    whatever the file tells it to: load only result files you trust."""
    with open(path, "rb") as f:
        r = pickle.load(f)
    if not isinstance(r, list) or len(r) != len(FIELDS):
        raise ValueError(f"{path}: not a regression result list of {len(FIELDS)} items")
    return dict(zip(FIELDS, r))


def l2(sim, obs):
    """adjoint_functions.L2's misfit: sum of squared residuals, in the dtype of the traces."""
    resid = sim - obs
    return np.sum(resid ** 2)


def finish(prob, x, fun, model_misfit, path, b=-1):
    """regression.py:89-96 for a fwi.Problem: forward of every shot of band b
    (default: the last) at the model x (flat or [Z, X], nondimensional),
    mseL2 against that band's observed data, and the pickle. Returns the
    dict that ``load`` would return."""
    import torch
    sc = prob.sc
    b = b % len(prob.bands)
    sb = prob.batch(b)
    model = np.asarray(x, np.float64).reshape(sc.Z, sc.X)
    sb.set_model(torch.as_tensor(model, dtype=torch.float32).cuda())
    recording = np.asarray(sb.forward(), np.float32)
    obs = sb._obs_dev.cpu().numpy()
    mse = l2(recording, obs)
    true_model = np.asarray(sc.c_true, np.float64)
    save(path, recording, model, true_model, sc.rec_mask, sc.src_mask, prob.vmin, prob.vmax, fun, mse,
         list(model_misfit))
    return dict(zip(FIELDS, [recording, model, true_model, sc.rec_mask, sc.src_mask, prob.vmin, prob.vmax, fun,
                             mse, list(model_misfit)]))
