"""CPU tests of the video-frame oracle (cuda_simulate with en_out = 1).

The oracle's frames are pinned to the reference twice: the FP32 pressure it
quantises equals, at every receiver, the reference library's own recorded
traces (tests/golden/sim_*.npz, bit for bit), and its bytes equal an
independent numpy restatement of writeFramePipe (utils.cu:94-113) applied to
that pressure."""
import glob
import os

import numpy as np
import pytest

import pml_oracle as po
from conftest import GOLDEN


def quantise(p, rec_x, rec_z):
    """writeFramePipe in numpy FP32: offset = -min, scale = 255 / (max - min),
    byte = (p + offset) * scale truncated, receivers 255."""
    p = np.asarray(p, np.float32)
    mn, mx = p.min(), p.max()
    offset = np.float32(-mn)
    scale = np.float32(255.0) / np.float32(mx - mn)
    q = (p + offset) * scale
    assert q.dtype == np.float32
    out = np.trunc(q).astype(np.uint8)
    out[np.asarray(rec_z), np.asarray(rec_x)] = 255
    return out


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "sim_*.npz"))), ids=os.path.basename)
@pytest.mark.parametrize("every", [1, 7])
def test_frame_oracle_pinned_to_reference_traces(path, every):
    d = np.load(path)
    T = int(d["T"])
    fr, pf = po.frames(np.asarray(d["c_true"], np.float32) ** 2, d["constvec"], d["d_x"], d["d_z"], d["src_x"],
                       d["src_z"], d["source"], d["rec_x"], d["rec_z"], every=every)
    n = (T - 1) // every
    assert fr.shape == (n, int(d["Z"]), int(d["X"])) and fr.dtype == np.uint8
    ts = every * np.arange(1, n + 1)
    # the quantised pressure at the receivers is the reference's own trace sample
    at_rec = pf[:, d["rec_z"], d["rec_x"]].T
    assert np.array_equal(at_rec, d["traces_all"][:, ts])
    for f in range(0, n, max(1, n // 25)):
        assert np.array_equal(fr[f], quantise(pf[f], d["rec_x"], d["rec_z"])), f
    # the frame's maximum maps to 255 (its minimum to 0, unless a receiver mark covers it)
    assert np.all(fr.reshape(n, -1).max(axis=1) == 255)


def test_frame_oracle_single_source_matches_simulate():
    d = np.load(os.path.join(GOLDEN, "sim_medium.npz"))
    fr, pf = po.frames(np.asarray(d["c_true"], np.float32) ** 2, d["constvec"], d["d_x"], d["d_z"], d["src_x"],
                       d["src_z"], d["source"], d["rec_x"], d["rec_z"], every=3, idx_source=1)
    ts = 3 * np.arange(1, fr.shape[0] + 1)
    assert np.array_equal(pf[:, d["rec_z"], d["rec_x"]].T, d["traces_s1"][:, ts])
