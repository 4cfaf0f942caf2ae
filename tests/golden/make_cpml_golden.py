"""Generate tests/golden/cpml_*.npz from the reference's own CPML library.

Runs on a machine with a GPU and oracle/_ref/cuda_regression_CPML.so (built
from the reference's simulator/src/regression_CPML.cu by `make -C oracle
ref`). Each case runs in its own process: the reference's init_memory_sim
calls cudaDeviceReset(). Inputs are seeded synthetic models and Ricker
sources; the library is driven through otfwi_b200.cpml.CPMLSimulator, the
same caller the tests use for this package's library.

    python tests/golden/make_cpml_golden.py
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "cuda_regression_CPML.so")

CASES = {
    # name: (X, Z, T, n_src, n_rec, seed, idx_source, ppe, initial field)
    "cpml_small": (96, 80, 400, 2, 8, 5, -1, 1, False),
    "cpml_shot1": (128, 96, 350, 3, 10, 6, 1, 1, False),
    "cpml_odd": (101, 77, 300, 2, 6, 7, -1, 2, True),
}


def case_sim(name, lib):
    sys.path.insert(0, ROOT)
    from otfwi_b200 import scenarios
    from otfwi_b200.cpml import CPMLSimulator
    X, Z, T, ns, nr, seed, idx, ppe, with_init = CASES[name]
    sc = scenarios.small(X=X, Z=Z, T=T, n_src=ns, n_rec=nr, seed=seed, f0=0.04)
    rng = np.random.default_rng(seed)
    rho = 1.0 + 0.5 * rng.random((Z, X))
    init = None
    if with_init:
        zz, xx = np.mgrid[0:Z, 0:X]
        bump = np.exp(-((xx - X / 2) ** 2 + (zz - Z / 2) ** 2) / 30.0)
        init = np.stack([bump, 0.98 * bump]).astype(np.float32)
    sim = CPMLSimulator(X, Z, T, sc.PML, sc.c_true, sc.src_mask, sc.rec_mask, sc.source, rho=rho, f0=0.04,
                        ppe=ppe, init=init, lib=lib)
    return sim, idx, ppe


def run_case(name, out):
    sim, idx, ppe = case_sim(name, REF_LIB)
    rec = sim.simulate(idx)
    X, Z, T = sim.X, sim.Z, sim.T
    np.savez_compressed(out, traces=rec, X=X, Z=Z, T=T, idx=idx, ppe=ppe, **sim.inputs)
    print(out, rec.shape, float(np.abs(rec).max()))


def main():
    if len(sys.argv) > 2 and sys.argv[1] == "--case":
        run_case(sys.argv[2], os.path.join(HERE, sys.argv[2] + ".npz"))
        return
    for name in CASES:
        subprocess.run([sys.executable, os.path.abspath(__file__), "--case", name], check=True)


if __name__ == "__main__":
    main()
