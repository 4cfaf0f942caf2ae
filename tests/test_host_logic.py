"""CPU tests of host-side logic around the kernels: the uneven batch's
instance generator and wave packing, the autotuner's candidate set and cache
key, and the bench's reading of the committed ncu summaries."""
import importlib.util
import os

import pytest

from conftest import ROOT


def test_uneven_instances_record_a_transmission():
    """Every seeded instance's T covers the travel time between its arrays
    (an all-zero observed trace makes the Wasserstein misfit 0/0)."""
    from otfwi_b200 import uneven
    specs = uneven.instance_specs(48)
    assert len(specs) == 48
    for s in specs:
        assert s["T"] >= uneven.min_steps(s["Z"])
        assert s["X"] % 32 == 0 and s["Z"] % 32 == 0
        assert 8 <= s["shots"] <= 64 and s["shots"] % 2 == 0
    assert uneven.instance_specs(48) == specs  # seeded


def test_uneven_waves_respect_the_budget():
    from otfwi_b200 import uneven
    specs = uneven.instance_specs(48)
    budget = 40e9
    waves = uneven.waves(specs, budget)
    assert sorted(i for w in waves for i in w) == list(range(48))
    for w in waves:
        assert len(w) == 1 or sum(uneven.device_bytes(specs[i]) for i in w) <= budget


def test_autotune_candidates_and_cache_key():
    from otfwi_b200 import autotune
    fast, faithful = autotune.candidates(1), autotune.candidates(0)
    assert (4, 4) in fast and (2, 4) in fast and all(k in (0, 1) for k, _ in faithful)
    k1 = autotune._key(512, 512, 64, 64, 1, "B200", fast)
    k2 = autotune._key(512, 512, 64, 64, 1, "B200", fast[:2])
    assert k1 != k2  # a different candidate set is a different cache entry
    assert all(t in autotune.TILES for _, t in fast + faithful)


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("kernel", [2, 4])
def test_bench_reads_the_committed_traffic_summaries(kernel):
    b = _bench()
    v = b.profile_traffic(kernel)
    assert v is not None and 20.0 < v < 100.0
    if kernel == 4:
        share = b.profile_value(4, "a_rev_share_of_step")
        assert 0.3 < share < 0.9
