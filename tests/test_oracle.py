"""The CPU oracle: golden regression, invariants and edge cases."""

import os

import numpy as np
import pytest

from extrem_z_b200 import synth
from oracle import ffi

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = np.load(os.path.join(HERE, "golden", "oracle_cases.npz"))
CASES = sorted({k.split("/")[0] for k in GOLDEN.files})
KW = dict(q=4, max_outer=500, max_cloop_rounds=100000, final_join=True)


def check_invariants(f, decp, out, eb):
    """Lowering only, and within the bound.

    The bound is the field type's bound T(eb).  A snapped voxel is set to
    f - bound computed in T (as the reference does, src/ExtreM_cuda.cu:3074),
    whose rounding can add up to one ulp of f: that is the stated tolerance.
    """
    assert out.dtype == f.dtype
    assert np.all(out <= decp)
    err = np.abs(f.astype(np.float64) - out.astype(np.float64))
    bound_t = float(f.dtype.type(eb))
    tol = bound_t + np.spacing(np.abs(f)).astype(np.float64)
    assert np.all(err <= tol)


@pytest.mark.parametrize("name", CASES)
def test_golden_regression(name):
    f, decp = GOLDEN[f"{name}/f"], GOLDEN[f"{name}/decp"]
    eb, et = GOLDEN[f"{name}/meta"][:2]
    out, rep, trace = ffi.correct(f, decp, eb, edit_type=int(et), trace_cap=200000, **KW)
    assert np.array_equal(out.view(np.uint8), GOLDEN[f"{name}/fixed"].view(np.uint8))
    assert np.array_equal(trace, GOLDEN[f"{name}/trace"])
    assert rep["status"] == 0
    check_invariants(f, decp, out, eb)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("edit_type", [0, 1])
def test_zero_mismatch_after_correction(dtype, edit_type):
    fld = synth.make_field(20, 16, 12, n_gauss=10, seed=42, rel=2e-3, dtype=dtype)
    out, rep, _ = ffi.correct(fld.f, fld.decp, fld.eb, edit_type=edit_type, **KW)
    assert rep["status"] == 0 and rep["counters"] == [0] * 11
    check_invariants(fld.f, fld.decp, out, fld.eb)
    # Critical points of the corrected field equal the original's.
    t0, _ = ffi.classify(fld.f)
    t1, _ = ffi.classify(out)
    assert np.array_equal(t0 == 4, t1 == 4) and np.array_equal(t0 == 0, t1 == 0)


def test_constant_field_bound_zero():
    f = np.full((4, 5, 6), 1.5)
    out, rep, _ = ffi.correct(f, f.copy(), 0.0, max_outer=3, max_cloop_rounds=3)
    assert np.array_equal(out, f)


@pytest.mark.parametrize("shape", [(1, 1, 1), (1, 1, 2), (2, 2, 2), (1, 7, 1), (3, 3, 3)])
def test_tiny_grids(shape):
    rng = np.random.default_rng(sum(shape))
    f = rng.standard_normal(shape)
    decp = f - 0.01 * rng.uniform(size=shape)
    out, rep, _ = ffi.correct(f, decp, 0.02, max_outer=50)
    assert rep["status"] in (0, 1)
    assert np.all(out <= decp)


def test_roots_are_extrema():
    fld = synth.make_field(12, 10, 8, n_gauss=6, seed=1, rel=1e-3)
    t, _ = ffi.classify(fld.f)
    ds, a_s = ffi.roots(fld.f)
    assert np.all(t[ds] == 4)
    assert np.all(t[a_s] == 0)


def test_two_d_slice_only_extrema_classified():
    # The reference LUT has no 2-D keys: non-extremal vertices of a slice are -1.
    fld = synth.make_field(16, 12, 1, n_gauss=4, seed=2, rel=1e-3)
    t, _ = ffi.classify(fld.f)
    assert set(np.unique(t)) <= {-1, 0, 4}
