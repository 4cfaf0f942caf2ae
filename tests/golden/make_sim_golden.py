"""Generate tests/golden/sim_*.npz by running the reference simulator itself.

Runs oracle/_ref/cuda_regression_PML_single.so -- the reference's
regression_PML_single.cu compiled from its own sources by oracle/Makefile --
on a CUDA GPU, through its C ABI in the call sequence the reference wrapper
uses (tests/abi_driver.py). It must run in a process of its own: the
reference calls cudaDeviceReset() in init_memory_sim.

Cases are small seeded problems, plus the plain single-shot benchmark
configuration at its full size (256 x 256, T = 1500; ``c1``), all with X a
multiple of 32, which keeps the reference's unguarded somaFrames / calcGrad2
writes inside each row. Each
file holds the inputs and the reference's outputs:
  traces_all / traces_s<k>  cuda_simulate(0, -1) / cuda_simulate(0, k)
  grad_s<k>                 cuda_grad_ext, L2 adjoint source against data
                            from the true model, at the start model
  sim_s<k>                  the traces the reference handed to the callback

    python tests/golden/make_sim_golden.py --out /tmp/golden [--cases c1]
"""
import argparse
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from otfwi_b200 import scenarios  # noqa: E402
from otfwi_b200._lib import _declare  # noqa: E402
from otfwi_b200.cuda_interface_pml import pml_damping, ring_mask  # noqa: E402
from abi_driver import run_abi  # noqa: E402


def case_inputs(sc, d_x, d_z, constvec):
    sx, sz = sc.src_xz()
    mx, mz = sc.rec_xz()
    rz, rx = np.where(ring_mask(sc.X, sc.Z, sc.PML, np.where(sc.src_mask), 4))
    return dict(X=sc.X, Z=sc.Z, T=sc.T, PML=sc.PML, c_true=sc.c_true.astype(np.float32),
                c_start=sc.c_start.astype(np.float32), d_x=np.asarray(d_x, np.float32),
                d_z=np.asarray(d_z, np.float32), constvec=np.asarray(constvec, np.float32),
                src_x=sx, src_z=sz, source=sc.source, rec_x=mx, rec_z=mz,
                ring_x=rx.astype(np.int32), ring_z=rz.astype(np.int32))


def cases():
    out = {}
    sc = scenarios.small()
    out["small"] = case_inputs(sc, *pml_damping(sc.X, sc.Z, sc.PML), np.ones(3))
    sc = scenarios.small(X=128, Z=96, T=500, n_src=3, n_rec=12, seed=7, f0=0.03)
    out["medium"] = case_inputs(sc, *pml_damping(sc.X, sc.Z, sc.PML), np.ones(3))
    # general ABI inputs the wrapper never produces: dt != 1 and damping that
    # varies along rows and columns
    sc = scenarios.small(X=96, Z=72, T=300, n_src=1, n_rec=6, seed=11, f0=0.05)
    sc.c_true = sc.c_true * 1.2
    sc.c_start = sc.c_start * 1.2
    rng = np.random.default_rng(5)
    dxp, dzp = pml_damping(sc.X, sc.Z, sc.PML)
    dxp = dxp * (1 + 0.2 * rng.random(dxp.shape))
    dzp = dzp * (1 + 0.2 * rng.random(dzp.shape))
    out["general"] = case_inputs(sc, dxp, dzp, [1.0, 1.0, 0.8])
    return out


def benchmark_cases():
    """The plain single-shot configuration at its full size: 256 x 256, 20-cell
    PML, T = 1500, one 5 MHz Ricker source at the top-surface centre, 32
    receivers at pitch 8 on the same row, three seeded 3000 m/s circular
    defects in 5900 m/s, gradient at the homogeneous 5900 m/s start."""
    sc = scenarios.plain_single_shot()
    return {"c1": case_inputs(sc, *pml_damping(sc.X, sc.Z, sc.PML), np.ones(3))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--lib", default=os.path.join(ROOT, "oracle", "_ref", "cuda_regression_PML_single.so"))
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--cases", default="all", help="comma-separated case names (default: every case)")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    lib = _declare(ctypes.CDLL(os.path.abspath(args.lib)))
    todo = dict(cases(), **benchmark_cases())
    if args.cases != "all":
        todo = {k: todo[k] for k in args.cases.split(",")}
    for name, inp in todo.items():
        res = run_abi(lib, **inp)
        path = os.path.join(args.out, f"sim_{name}.npz")
        np.savez_compressed(path, **inp, **res)
        print(path, float(np.abs(res["traces_all"]).max()), float(np.abs(res["grad_s0"]).max()))


if __name__ == "__main__":
    main()
