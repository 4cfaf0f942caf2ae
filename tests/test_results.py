"""CPU tests of the result file (regression.py:89-96 layout)."""
import pickle

import numpy as np
import pytest

from otfwi_b200 import results


def test_result_file_layout_roundtrip(tmp_path):
    rng = np.random.default_rng(0)
    rec = rng.standard_normal((3, 5, 40)).astype(np.float32)
    obs = rng.standard_normal((3, 5, 40)).astype(np.float32)
    model = rng.random((8, 12))
    xzm = np.zeros((8, 12), bool)
    xzm[2, 3:8] = True
    xzs = np.zeros((8, 12), bool)
    xzs[2, [3, 7]] = True
    mse = results.l2(rec, obs)
    assert mse.dtype == np.float32 and mse == np.sum((rec - obs) ** 2)
    p = tmp_path / "output" / "regression_case.pickle"
    results.save(str(p), rec, model, model * 2, xzm, xzs, 0.3, 0.5, 1.25, mse, [0.1, 0.05])
    # the reference's reader unpickles a plain list in this order
    with open(p, "rb") as f:
        raw = pickle.load(f)
    assert isinstance(raw, list) and len(raw) == 10
    assert np.array_equal(raw[0], rec) and np.array_equal(raw[1], model) and np.array_equal(raw[3], xzm)
    assert raw[5:8] == [0.3, 0.5, 1.25] and raw[9] == [0.1, 0.05]
    d = results.load(str(p))
    assert list(d) == list(results.FIELDS)
    assert np.array_equal(d["xzs"], xzs) and d["mseL2"] == mse


def test_load_rejects_other_pickles(tmp_path):
    p = tmp_path / "x.pickle"
    with open(p, "wb") as f:
        pickle.dump({"a": 1}, f)
    with pytest.raises(ValueError):
        results.load(str(p))
