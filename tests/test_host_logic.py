"""CPU tests of host-side logic around the kernels: the uneven batch's
instance generator and wave packing, the autotuner's candidate set and cache
key, the bench's reading of the committed ncu summaries, and the FWI loop's
line search, history and gradient mask, and that the integration guide names
only what the package has."""
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


def test_autotune_cache_round_trip_and_unwritable_location(tmp_path, monkeypatch):
    """The cache survives a store/load round trip with no temporary file left
    behind; an unreadable or unwritable location degrades to an empty cache
    instead of an error; a torn file reads as empty."""
    from otfwi_b200 import autotune
    p = tmp_path / "tune" / "tune.json"
    monkeypatch.setenv("OTFWI_TUNE_CACHE", str(p))
    entry = {"k": {"kernel": 4, "tile": 4, "table": {"4/4": 118.1}}}
    autotune._store(entry)
    assert autotune._load() == entry
    assert [f.name for f in p.parent.iterdir()] == ["tune.json"]
    p.write_text('{"k": {"kernel"')
    assert autotune._load() == {}
    blocker = tmp_path / "file"
    blocker.write_text("")
    monkeypatch.setenv("OTFWI_TUNE_CACHE", str(blocker / "sub" / "tune.json"))
    autotune._store(entry)  # the directory cannot be made: silently skipped
    assert autotune._load() == {}


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


class _Quadratic:
    """A stand-in for fwi.Problem along one direction: J(c) = (c - c_min)^2 + J_min
    on a scalar model, clipped to [vmin, vmax]; counts evaluations."""

    def __init__(self, c_min, J_min=0.0, vmin=-1e9, vmax=1e9):
        self.c_min, self.J_min, self.vmin, self.vmax = c_min, J_min, vmin, vmax
        self.calls = 0

    def objective(self, b, c):
        self.calls += 1
        return float((c - self.c_min) ** 2 + self.J_min)

    def clip(self, c):
        return min(max(c, self.vmin), self.vmax)


@pytest.mark.parametrize("alpha0", [0.25, 1.0, 16.0, 100.0])
def test_line_search_brackets_and_lands_on_a_quadratic_minimum(alpha0):
    """Expanding from a short first step or shrinking from a long one, the
    bracket's parabolic step lands on the minimum of a quadratic (the
    three-point vertex is exact for a parabola); the evaluation count it
    reports is the number of objective calls."""
    from otfwi_b200.fwi import line_search
    prob = _Quadratic(3.0)
    J0 = prob.objective(0, 0.0)
    prob.calls = 0
    a, J, evals = line_search(prob, 0, 0.0, 1.0, J0, alpha0, max_evals=12)
    assert evals == prob.calls
    assert abs(a - 3.0) < 1e-9 and J < 1e-12


def test_line_search_reports_no_step_uphill():
    """Along an ascent direction no trial decreases the misfit: step 0, the
    starting misfit, and no more than max_evals trials."""
    from otfwi_b200.fwi import line_search
    prob = _Quadratic(0.0, J_min=1.0)
    a, J, evals = line_search(prob, 0, 0.0, 1.0, 1.0, 0.5, max_evals=6)
    assert (a, J) == (0.0, 1.0) and evals == 6 == prob.calls


def test_line_search_respects_the_bounds():
    """Trial models are clipped to [vmin, vmax]: a minimum beyond the upper
    bound gives a step that reaches the bound and never a misfit below the
    bound's."""
    from otfwi_b200.fwi import line_search
    prob = _Quadratic(10.0, vmax=4.0)
    J0 = prob.objective(0, 0.0)
    a, J, _ = line_search(prob, 0, 0.0, 1.0, J0, 1.0, max_evals=8)
    assert prob.clip(a) == 4.0 and J == prob.objective(0, 4.0)


def test_history_time_to_and_default_gmask():
    from otfwi_b200 import scenarios
    from otfwi_b200.fwi import History, default_gmask
    h = History(t=[0.0, 1.5, 3.0], rms=[100.0, 80.0, 60.0])
    assert h.time_to(80.0) == 1.5 and h.time_to(59.0) is None and h.time_to(1e9) == 0.0
    sc = scenarios.small(X=96, Z=80, T=50, n_src=1, n_rec=4, seed=1)
    m = default_gmask(sc)
    assert m.shape == (80, 96) and m.sum() == (80 - 2 * 20) * (96 - 2 * 24)
    assert m[20, 24] == 1 and m[19, 24] == 0 and m[20, 23] == 0 and m[59, 71] == 1 and m[60, 71] == 0


def test_integration_guide_names_exist():
    """Every package name the integration guide's examples use exists, so the
    guide cannot drift from the API."""
    import re
    import importlib
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    used = set(re.findall(r"from (otfwi_b200(?:\.\w+)?) import ([\w, ]+)", text))
    assert used
    for mod, names in used:
        m = importlib.import_module(mod)
        for n in (x.split(" as ")[0].strip() for x in names.split(",")):
            assert hasattr(m, n) or importlib.util.find_spec(f"{mod}.{n}") is not None, (mod, n)
    for mod, attr in re.findall(r"\b(fwi|learned|results|autotune)\.(\w+)\(", text):
        assert hasattr(importlib.import_module(f"otfwi_b200.{mod}"), attr), (mod, attr)
    for cls, meth in (("ShotBatch", "frames"), ("ShotBatch", "objective"), ("ShotBatch", "illumination"),
                      ("MultiBatch", "gradient")):
        assert hasattr(getattr(importlib.import_module("otfwi_b200.batch"), cls), meth)
