"""Branch decomposition of merge trees (constructMergeTree, src/ExtreM.cpp
:1863-1918) from the oracle's elder-rule pairs and parents.

The oracle's parent of an extremum is the elder survivor where it merges,
which is alive there by construction, so constructMergeTree's compression
must leave it unchanged; every branch of n extrema then lists 3n - 1 vertices
in all (each extremum, each non-global partner twice -- in its own branch and
in its parent's -- and the opposite global extremum once).
"""

import numpy as np
import pytest

from extrem_z_b200 import api, synth
from oracle import ffi, merge_tree


def test_line_field_branches():
    # x: 0  1  2   3  4 ; maxima at 0, 2 (global), 4; merge vertices 1 and 3.
    f = np.array([1.0, 0.0, 3.0, -1.0, 2.0]).reshape(1, 1, 5)
    mx, mn, px, pn = ffi.persistence_tree(f)
    assert mx.tolist() == [[1, 0], [3, 4], [3, 2]]   # (partner, maximum), ascending maxima
    assert px.tolist() == [2, 2, 2]
    br = api.merge_tree_branches(f.ravel(), mx, px, split=True)
    assert [b.tolist() for b in br] == [[0, 1], [4, 3], [2, 1, 3, 3]]


@pytest.mark.parametrize("shape,seed", [((24, 20, 16), 0), ((37, 29, 1), 3), ((40, 36, 12), 5)])
def test_oracle_tree_consistent(shape, seed):
    w, h, d = shape
    fld = synth.make_field(w, h, d, n_gauss=10, seed=seed, rel=1e-3, dtype=np.float64)
    mx, mn, px, pn = ffi.persistence_tree(fld.f)
    mx0, mn0 = ffi.persistence_pairs(fld.f)
    assert np.array_equal(mx, mx0) and np.array_equal(mn, mn0)
    fv = fld.f.ravel()
    for pairs, par, split in ((mx, px, True), (mn, pn, False)):
        n = len(pairs)
        ext = pairs[:, 1]
        rank = {int(v): k for k, v in enumerate(ext)}
        pr = np.array([rank[int(p)] for p in par])
        assert pr[-1] == n - 1                    # the global extremum is its own parent
        assert np.all(pr[:-1] > np.arange(n - 1))  # parents are older extrema
        compressed = api._compress_parents(fv, pairs, pr, split)
        assert np.array_equal(compressed, pr)     # alive at the merge: nothing to compress
        br = api.merge_tree_branches(fv, pairs, par, split=split)
        assert sum(len(b) for b in br) == 3 * n - 1
        assert all(b[0] == e for b, e in zip(br, ext))
        assert br[-1][-1] == pairs[-1, 0]         # the global branch ends at the opposite one


@pytest.mark.parametrize("shape,seed,dtype", [((24, 20, 16), 0, np.float64), ((37, 29, 1), 3, np.float64),
                                              ((5, 70, 9), 6, np.float32), ((40, 36, 12), 5, np.float64)])
def test_rounds_restatement_pairs_match_elder_rule(shape, seed, dtype):
    # The numpy restatement of constructPersistencePairs' rounds pairs every
    # extremum as the union-find elder rule does; its merge targets, once
    # compressed, differ from the elder survivors only where several extrema
    # pair at one merge vertex (the reference's order of rewriting rows).
    w, h, d = shape
    fld = synth.make_field(w, h, d, n_gauss=10, seed=seed, rel=1e-3, dtype=dtype)
    mx, mn, px, pn = ffi.persistence_tree(fld.f)
    fv = fld.f.astype(np.float64).ravel()
    for split, rp, rt in ((True, mx, px), (False, mn, pn)):
        pairs, tgt = merge_tree.persistence_tree(fld.f, split)
        assert np.array_equal(pairs, rp)
        ext = pairs[:, 1]
        idx = np.argsort(ext)
        rk = lambda v: idx[np.searchsorted(ext[idx], v)]
        comp = api._compress_parents(fv, pairs, rk(tgt), split)
        elder = rk(rt)
        for e in np.flatnonzero(comp != elder):
            assert pairs[comp[e], 0] == pairs[e, 0]   # same merge vertex: the tie case


def test_rounds_on_line_field():
    f = np.array([1.0, 0.0, 3.0, -1.0, 2.0]).reshape(1, 1, 5)
    pairs, tgt = merge_tree.persistence_tree(f, True)
    assert pairs.tolist() == [[1, 0], [3, 4], [3, 2]] and tgt.tolist() == [2, 2, 2]


def test_branch_comparison_by_rank_and_by_extremum():
    a = [np.array([5, 3, 1]), np.array([7, 2]), np.array([9, 3, 3])]
    b = [np.array([7, 2]), np.array([5, 3, 1]), np.array([9, 3, 3])]   # two maxima swapped in rank
    rep = api.compare_branches(a, b)
    assert rep["identical_by_rank"] == 1 and rep["identical_by_extremum"] == 3
    assert not rep["same"]
    assert [d["branch"] for d in rep["first_differences"]] == [0, 1]
    assert api.compare_branches(a, a)["same"]
