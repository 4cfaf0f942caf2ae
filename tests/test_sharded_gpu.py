"""GPU tests of the shot sharding used with several GPUs
(distributed.ShardedShots): one acquisition's shot table split into
contiguous blocks, each block run as its own batched gradient, the local
shot means weighted by their shot counts and summed.

This run has one GPU, so the ranks' blocks run one after the other in one
process (no process group); the all-reduce itself is covered by the gloo
tests (tests/test_distributed.py)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scenario():
    from otfwi_b200 import scenarios
    return scenarios.fmc(X=256, Z=160, T=300, n_elem=12, pitch=12, x_first=50, seed=6)


def _gradient(sc, shots):
    from otfwi_b200.batch import ShotBatch
    b = ShotBatch(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, sc.source, prec_deriv=4, precision=1,
                  shots=shots)
    try:
        b.set_model(sc.c_true)
        b.set_observed(b.forward())
        b.set_model(sc.c_start)
        g, m = b.gradient("wasserstein_softplus")
        return g.copy(), m, b.n_shots
    finally:
        b.close()


@pytest.mark.parametrize("world", [2, 3, 5])
def test_rank_blocks_sum_to_full_acquisition(lib, world):
    from otfwi_b200.distributed import shard_block
    sc = _scenario()
    g_full, m_full, n = _gradient(sc, None)
    g = np.zeros_like(g_full, dtype=np.float64)
    m = 0.0
    for r in range(world):
        lo, hi = shard_block(n, world, r)
        gr, mr, nr = _gradient(sc, (np.arange(hi - lo + 1), np.arange(lo, hi)))
        assert nr == hi - lo
        g += gr.astype(np.float64) * (nr / n)
        m += mr
    assert np.abs(g - g_full).max() <= 1e-6 * np.abs(g_full).max()
    assert abs(m - m_full) <= 1e-12 * abs(m_full)


def test_single_rank_sharded_shots_is_the_batch(lib):
    """Without a process group ShardedShots is the whole batch: identical
    gradient, misfit and line-search objective."""
    import torch
    from otfwi_b200.batch import ShotBatch, fmc_shots
    from otfwi_b200.distributed import ShardedShots
    sc = _scenario()
    g_full, m_full, n = _gradient(sc, None)
    ptr, srcs = fmc_shots(sc.n_src)
    sh = ShardedShots(lambda shots: ShotBatch(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, sc.source,
                                              prec_deriv=4, precision=1, shots=shots),
                      ptr, srcs, (sc.Z, sc.X), device="cuda")
    try:
        assert (sh.lo, sh.hi, sh.n_shots) == (0, n, n)
        sh.set_model(sc.c_true)
        obs = torch.empty((n, sc.n_rec, sc.T), dtype=torch.float32, device="cuda")
        sh.forward(out=obs)
        sh.set_observed(obs)
        sh.set_model(sc.c_start)
        g, m = sh.gradient("wasserstein_softplus")
        assert np.array_equal(g.cpu().numpy(), g_full)
        assert float(m.item()) == m_full
        j = sh.objective("wasserstein_softplus")
        assert j == m_full
    finally:
        sh.close()
