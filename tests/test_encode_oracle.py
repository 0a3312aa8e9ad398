"""The oracle's edit-stream encoder against the reference's own helpers.

tests/golden/encode_cases.npz holds int32 inputs and the outputs of the
reference's encodeTo3BitBitmap and get_diff_index, run from the reference's
source (tests/golden/make_golden.py --encode).  The oracle encodes whole
fields; each case is turned into a field whose edits produce exactly that
input: every voxel edited with its counter set to the value (3-bit stream,
edit_type 0), or the listed ids edited (delta-coded ids, edit_type 1).
"""

import os

import numpy as np
import pytest

from oracle import ffi

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, "golden", "encode_cases.npz"))
LENGTHS = sorted({int(k.split("/")[1]) for k in GOLD.files})


@pytest.mark.parametrize("n", LENGTHS)
def test_pack3_matches_reference(n):
    v = GOLD[f"pack3/{n}/in"]
    f = np.linspace(0.0, 1.0, n)
    d0 = f - 0.01
    d1 = d0 - 0.001              # every voxel edited
    idx, edits, rep = ffi.encode(f, d0, d1, v.astype(np.int32), 0.02, q=4, edit_type=0)
    assert np.array_equal(idx, GOLD[f"pack3/{n}/out"])
    assert rep["index_bytes"] == (3 * n + 7) // 8
    assert rep["edited"] == n and rep["n_edits"] == int(np.count_nonzero(v == 4))


@pytest.mark.parametrize("n", LENGTHS)
def test_diff_matches_reference(n):
    ids = GOLD[f"diff/{n}/in"]
    size = int(ids.max()) + 3
    f = np.linspace(0.0, 1.0, size)
    d0 = f - 0.01
    d1 = d0.copy()
    d1[ids] -= 0.001             # exactly the listed voxels edited
    idx, edits, rep = ffi.encode(f, d0, d1, None, 0.02, edit_type=1)
    assert np.array_equal(idx.view("<i4"), GOLD[f"diff/{n}/out"])
    # Lossless edits: (f - bound) - decp at each edited voxel, in id order.
    assert np.array_equal(edits, -(d0[ids] - (f[ids] - 0.02)))


def test_counter_beyond_three_bits_rejected():
    f = np.zeros(4)
    with pytest.raises(ValueError):
        ffi.encode(f, f - 1, f - 2, np.array([0, 8, 0, 0], np.int32), 1.0, q=8, edit_type=0)


def test_psnr_follows_reference_formula():
    rng = np.random.default_rng(0)
    f = rng.normal(size=1000)
    d0 = f + rng.uniform(-1e-3, 1e-3, size=1000)
    d1 = d0.copy()
    d1[::7] -= 1e-4
    _, _, rep = ffi.encode(f, d0, d1, None, 1e-3, edit_type=1)
    rng_f = f.max() - f.min()
    want0 = -20 * np.log10(np.sqrt(np.mean((f - d0) ** 2)) / rng_f)
    want1 = -20 * np.log10(np.sqrt(np.mean((f - d1) ** 2)) / rng_f)
    assert abs(rep["psnr_before"] - want0) < 1e-9 and abs(rep["psnr_after"] - want1) < 1e-9
