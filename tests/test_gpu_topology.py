"""Merge-tree persistence pairs on the GPU against the union-find oracle.

The library pairs extrema with saddles by the reference's extremum-graph
rounds (constructPersistencePairs) over the field's own critical points and
manifold labels; the oracle applies the elder rule with a union-find over
all vertices.  Both must give the same pairs, in the same order.
"""

import numpy as np
import pytest

from extrem_z_b200 import synth

pytestmark = pytest.mark.gpu

CASES = [
    ("plain64_f32", lambda: synth.plain_64(np.float32)),
    ("box_f64", lambda: synth.make_field(40, 30, 20, n_gauss=12, seed=4, rel=1e-3)),
    ("slice_f64", lambda: synth.make_field(96, 80, 1, n_gauss=16, seed=5, rel=1e-3)),
    ("thin_f32", lambda: synth.make_field(5, 70, 9, n_gauss=6, seed=6, rel=2e-3,
                                          dtype=np.float32)),
]


@pytest.mark.parametrize("name", [c[0] for c in CASES])
def test_pairs_match_union_find(name):
    import torch
    from extrem_z_b200 import api
    from oracle import ffi
    fld = dict(CASES)[name]()
    for field in (fld.f, fld.decp):
        mx, mn = api.context(0).persistence_pairs(torch.from_numpy(field).cuda())
        rmx, rmn = ffi.persistence_pairs(field)
        assert np.array_equal(mx, rmx), name
        assert np.array_equal(mn, rmn), name


def test_correction_report():
    import torch
    from extrem_z_b200 import api
    from oracle import ffi
    fld = synth.plain_64(np.float64)
    f = torch.from_numpy(fld.f).cuda()
    ctx = api.context(0)
    # Without the final join pass the loop ends at zero critical-point
    # mismatch: the same extrema, so the same number of pairs, on both sides.
    g = torch.from_numpy(fld.decp.copy()).cuda()
    ctx.correct_device(f, g, fld.eb, final_join=False)
    rep = ctx.compare_topology(f, g)
    for side in ("split", "join"):
        assert rep[side]["pairs_original"] == rep[side]["pairs_corrected"] > 0
        assert rep[side]["identical"] <= rep[side]["pairs_original"]
    # The reference's unconditional final saddle_loops_join (src/ExtreM_cuda.cu
    # :5997) edits after the last detection; on this field it removes two
    # minima, which the report shows as the oracle's classification does.
    g = torch.from_numpy(fld.decp.copy()).cuda()
    ctx.correct_device(f, g, fld.eb, final_join=True)
    rep = ctx.compare_topology(f, g)
    t, _ = ffi.classify(g.cpu().numpy())
    assert rep["join"]["pairs_corrected"] == int((t == 0).sum())
    assert rep["split"]["pairs_corrected"] == int((t == 4).sum())


@pytest.mark.parametrize("name", [c[0] for c in CASES])
def test_merge_targets_match_rounds(name):
    # Each extremum's merge target (constructPersistencePairs' largestMax)
    # against the numpy restatement of the same rounds, exactly; and the
    # branches built from them.
    import torch
    from extrem_z_b200 import api
    from oracle import merge_tree
    fld = dict(CASES)[name]()
    fv = fld.f.astype(np.float64).ravel()
    mx, mn, px, pn = api.context(0).persistence_tree(torch.from_numpy(fld.f).cuda())
    for pairs, par, split in ((mx, px, True), (mn, pn, False)):
        rpairs, rpar = merge_tree.persistence_tree(fld.f, split)
        assert np.array_equal(pairs, rpairs), name
        assert np.array_equal(par, rpar), name
        b = api.merge_tree_branches(fv, pairs, par, split=split)
        rb = api.merge_tree_branches(fv, rpairs, rpar, split=split)
        assert all(np.array_equal(x, y) for x, y in zip(b, rb)), name


def test_branch_report_of_a_correction():
    import torch
    from extrem_z_b200 import api
    fld = synth.plain_64(np.float64)
    f = torch.from_numpy(fld.f).cuda()
    g = torch.from_numpy(fld.decp.copy()).cuda()
    ctx = api.context(0)
    ctx.correct_device(f, g, fld.eb, final_join=False)
    rep = ctx.compare_topology(f, g)["split"]["branches"]
    assert rep["branches_original"] == rep["branches_corrected"] > 0
    assert 0 <= rep["identical_by_rank"] <= rep["identical_by_extremum"] <= rep["branches_original"]
    assert rep["same"] == (rep["identical_by_rank"] == rep["branches_original"])
