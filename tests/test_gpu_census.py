"""Mismatch census on the GPU against the oracle's census.

The census evaluates the eleven loop-test counters once on a field, with no
edit: on the decompressed field before any correction (every counter busy),
and on the corrected field with and without the final join-saddle pass, which
edits after the loop's last test (src/ExtreM_cuda.cu:5997) and so can leave
critical-point mismatches behind.  Counts are integers: equality is exact.
"""

import numpy as np
import pytest

from extrem_z_b200 import synth

pytestmark = pytest.mark.gpu

KW = dict(q=4, edit_type=1, max_outer=500, max_cloop_rounds=100000)

CASES = [
    ("plain64_f64", lambda: synth.plain_64(np.float64)),
    ("plain64_f32", lambda: synth.plain_64(np.float32)),
    ("box_f64", lambda: synth.make_field(40, 33, 21, n_gauss=14, seed=41, rel=2e-3)),
    ("slice_f32", lambda: synth.make_field(96, 80, 1, n_gauss=12, seed=42, rel=1e-3,
                                           dtype=np.float32)),
]


def _census_gpu(f, g, thr=0.0):
    import torch
    from extrem_z_b200 import api
    tf = torch.from_numpy(np.ascontiguousarray(f)).cuda()
    tg = torch.from_numpy(np.ascontiguousarray(g)).cuda()
    before = tg.clone()
    res = api.context(0).mismatch_census(tf, tg, thr=thr)
    torch.cuda.synchronize()
    assert torch.equal(tg, before)  # the census only reads the field
    return res["counters"]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_census_matches_oracle(name, make):
    from oracle import ffi
    fld = make()
    assert _census_gpu(fld.f, fld.decp) == ffi.census(fld.f, fld.decp)
    for final_join in (True, False):
        fixed, rep, _ = ffi.correct(fld.f, fld.decp, fld.eb, final_join=final_join, **KW)
        assert rep["status"] == 0
        want = ffi.census(fld.f, fixed)
        assert _census_gpu(fld.f, fixed) == want
        if not final_join:
            # The loop ends when its counters are zero; preserve_join_tree is
            # off, so only the join-tree counters may stay busy.
            assert want[:8] == [0] * 8


@pytest.mark.parametrize("name,make", CASES[1:3], ids=[c[0] for c in CASES[1:3]])
def test_classify_and_roots_match_oracle(name, make):
    """extremz_classify: vertex types and steepest-path roots, exact."""
    import torch
    from extrem_z_b200 import api
    from oracle import ffi
    fld = make()
    for a in (fld.f, fld.decp):
        t, ds, as_ = api.context(0).classify(torch.from_numpy(np.ascontiguousarray(a)).cuda())
        t0, _ = ffi.classify(a)
        r_ds, r_as = ffi.roots(a)
        assert np.array_equal(t.cpu().numpy().reshape(-1), t0)
        assert np.array_equal(ds.cpu().numpy().reshape(-1), r_ds)
        assert np.array_equal(as_.cpu().numpy().reshape(-1), r_as)


def test_census_of_original_is_zero():
    fld = synth.make_field(30, 26, 18, n_gauss=10, seed=43, rel=1e-3)
    assert _census_gpu(fld.f, fld.f) == [0] * 11
