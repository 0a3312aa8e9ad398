"""The pairing rounds and the branch decomposition against the reference's own
constructPersistencePairs and constructMergeTree (src/ExtreM.cpp :2132-2249,
:1863-1918), compiled from its source by oracle/ref/build_ref_cpu.sh into
oracle/_ref/ref_mergetree.

Both sides get the same extremum graph (split tree), built by
oracle/merge_tree.py from seeded fields: maxima ascending, merge vertices
descending, rows of distinct maximum ranks (single-entry rows emptied, as the
rounds do after each step), and the vertex order.  The reference's pairs, its
merge targets before and after constructMergeTree, and its branches must equal
the restatement's, which the GPU's equal (tests/test_gpu_topology.py).
"""

import os
import subprocess
import tempfile

import numpy as np
import pytest

from extrem_z_b200 import api, synth
from oracle import merge_tree

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "..", "oracle", "_ref", "ref_mergetree")

pytestmark = pytest.mark.skipif(not os.path.exists(REF),
                                reason="oracle/_ref/ref_mergetree not built")


def _run_reference(gr):
    ext, sad, rows, cnt = gr["ext"], gr["sad"], gr["rows"], gr["cnt"]
    rank = gr["rank"]
    nmax, ns, n = len(ext), len(sad), len(rank)
    tri = np.zeros((ns, 46), np.int32)
    tri[:, :rows.shape[1]] = np.where(rows >= 0, rows, 0)
    tri[:, 44] = cnt
    tri[:, 45] = sad
    data = np.concatenate([np.array([nmax, ns, n, gr["opposite"]]), ext, sad, tri.ravel(),
                           rank]).astype("<i4")
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.i32"), os.path.join(d, "out.i32")
        data.tofile(fin)
        subprocess.run([REF, fin, fout], check=True, timeout=120)
        out = np.fromfile(fout, "<i4")
    k = 1
    pairs = out[k:k + 2 * nmax].reshape(-1, 2); k += 2 * nmax
    paired = out[k:k + 2 * nmax].reshape(-1, 2); k += 2 * nmax
    merged = out[k:k + 2 * nmax].reshape(-1, 2); k += 2 * nmax
    branches = []
    for _ in range(nmax):
        m = out[k]; k += 1
        branches.append(out[k:k + 2 * m].reshape(-1, 2)[:, 1].astype(np.int64)); k += 2 * m
    return pairs, paired, merged, branches


@pytest.mark.parametrize("shape,seed,dtype", [((24, 20, 16), 0, np.float64),
                                              ((37, 29, 1), 3, np.float64),
                                              ((5, 70, 9), 6, np.float32),
                                              ((40, 36, 12), 5, np.float64)])
def test_rounds_and_branches_match_reference(shape, seed, dtype):
    w, h, d = shape
    fld = synth.make_field(w, h, d, n_gauss=10, seed=seed, rel=1e-3, dtype=dtype)
    gr = merge_tree.extremum_graph(fld.f, True)
    pairs, tgt = merge_tree.persistence_tree(fld.f, True)
    rpairs, rpaired, rmerged, rbranches = _run_reference(gr)
    ext, sad = gr["ext"], gr["sad"]
    n = len(ext)
    paired = pairs[:, 0] >= 0
    # pairs[maximum] = (saddles2[largestSaddle], Maximum[maximum]); the global
    # maximum's partner is the global minimum.
    assert np.array_equal(rpairs[paired], pairs[paired])
    # maximaTriplets after the rounds: (largestSaddle, largestMax) by rank.
    idx = np.argsort(ext)
    trank = idx[np.searchsorted(ext[idx], tgt)]
    assert np.array_equal(rpaired[:-1][paired[:-1], 1], trank[:-1][paired[:-1]])
    # constructMergeTree's compression of them.
    comp = api._compress_parents(fld.f.astype(np.float64).ravel(), pairs, trank, True)
    assert np.array_equal(rmerged[:, 1], comp)
    # Branches: the reference orders vertices by the given order (here the
    # (value, id) rank), as merge_tree_branches does.
    br = api.merge_tree_branches(fld.f.astype(np.float64).ravel(), pairs, tgt, split=True)
    assert len(br) == len(rbranches) == n
    assert all(np.array_equal(a, b) for a, b in zip(br, rbranches))
