"""Extremum-graph persistence pairs and merge targets, restated with numpy.

Test infrastructure only: the oracle of ``extremz_persistence_tree``.  It
follows the reference's constructPersistencePairs (src/ExtreM.cpp:2132-2249)
round by round, on the extremum graph that the library builds from the field
itself (the same inputs the GPU pairing takes):

* order: (value, id) ascending for the split tree, the reverse for the join
  tree; -0.0 and +0.0 are equal values;
* extrema: vertices with no neighbour above them in the tree's order (of the
  14 Freudenthal neighbours in the grid);
* merge vertices: vertices whose link restricted to the neighbours above has
  two or more components (link edges join two neighbours whose offset is
  itself one of the 14 directions);
* rows: per merge vertex, in descending tree order, the distinct ranks of the
  extrema that the steepest paths of its neighbours above reach, ascending; a
  row with one entry is emptied.

Rounds (:2141-2236): every extremum but the global one takes the first
(largest) merge vertex whose row holds it; an extremum that is the smallest
entry of that row pairs with it and points to the row's largest entry (the
merge target, maximaTriplets' second element, :2187); pointers are
compressed (:2201-2215) and every row is rewritten through them, deduplicated
and emptied at one entry (:2217-2227).  The global extremum pairs with the
opposite global extremum (:2239-2240).

The elder rule (``ffi.persistence_tree``) gives the same pairs.  Its merge
target is the oldest extremum of the components that meet at the partner
vertex.  The rounds' target can differ from it when several extrema pair at
one merge vertex: an extremum can pair before a row entry has been rewritten
to the older extremum that entry already merged into, so it points to a
younger one, and constructMergeTree's compression (:1869-1885) does not move
it because both share the merge vertex.
"""

from __future__ import annotations

import numpy as np

from . import ffi

DIRS = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1), (-1, 1, 0),
        (1, -1, 0), (0, 1, 1), (0, -1, -1), (-1, 0, 1), (1, 0, -1), (-1, 1, 1), (1, -1, -1)]


def _link_components_table() -> np.ndarray:
    adj = []
    for a in DIRS:
        m = 0
        for b, db in enumerate(DIRS):
            if db != a and (db[0] - a[0], db[1] - a[1], db[2] - a[2]) in DIRS:
                m |= 1 << b
        adj.append(m)
    table = np.zeros(1 << 14, np.int8)
    for nodes in range(1 << 14):
        comps, left = 0, nodes
        while left:
            comp = left & -left
            while True:
                grow = comp
                for d in range(14):
                    if comp >> d & 1:
                        grow |= adj[d] & nodes
                if grow == comp:
                    break
                comp = grow
            left &= ~comp
            comps += 1
        table[nodes] = comps
    return table


_TABLE = None


def _rows_sorted_unique(e: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Per row of e (entries >= 0, -1 empty): distinct entries ascending, and
    their count; a row with one entry is emptied."""
    big = np.iinfo(np.int64).max
    r = np.where(e >= 0, e, big)
    r.sort(axis=1)
    dup = np.zeros_like(r, dtype=bool)
    dup[:, 1:] = r[:, 1:] == r[:, :-1]
    r[dup] = big
    r.sort(axis=1)
    cnt = (r != big).sum(axis=1)
    cnt[cnt == 1] = 0
    r[np.arange(r.shape[1])[None, :] >= cnt[:, None]] = -1
    return r, cnt


def extremum_graph(f: np.ndarray, split: bool = True) -> dict:
    """The extremum graph of one tree: rank (every vertex's position in the
    tree's order), ext (extrema, ascending), sad (merge vertices,
    descending), rows / cnt (per merge vertex, distinct extremum ranks
    ascending, -1 padded; single-entry rows emptied) and opposite (the
    vertex first in the tree's order)."""
    global _TABLE
    if _TABLE is None:
        _TABLE = _link_components_table()
    f = np.ascontiguousarray(f)
    D, H, W = f.shape
    N = f.size
    vals = f.astype(np.float64).ravel()
    ids = np.arange(N)
    asc = np.lexsort((ids, vals))
    rank = np.empty(N, np.int64)
    rank[asc] = np.arange(N)
    if not split:
        rank = N - 1 - rank          # the join tree's order
    z, y, x = np.unravel_index(ids, (D, H, W))
    side = np.zeros(N, np.int64)      # bit d: neighbour d is above in the tree
    nbr = np.full((N, 14), -1, np.int64)
    for d, (dx, dy, dz) in enumerate(DIRS):
        xx, yy, zz = x + dx, y + dy, z + dz
        ok = (xx >= 0) & (xx < W) & (yy >= 0) & (yy < H) & (zz >= 0) & (zz < D)
        u = np.where(ok, xx + yy * W + zz * W * H, 0)
        nbr[:, d] = np.where(ok, u, -1)
        side |= (ok & (rank[u] > rank)).astype(np.int64) << d
    ext = np.flatnonzero(side == 0)
    ext = ext[np.argsort(rank[ext])]                 # ascending in the tree's order
    ne = len(ext)
    erank = np.full(N, -1, np.int64)
    erank[ext] = np.arange(ne)
    sad = np.flatnonzero(_TABLE[side] >= 2)
    sad = sad[np.argsort(-rank[sad])]                # descending
    ns = len(sad)
    ds, as_ = ffi.roots(f)
    lab = (ds if split else as_).ravel().astype(np.int64)
    e = np.full((ns, 14), -1, np.int64)
    for d in range(14):
        u = nbr[sad, d]
        on = (u >= 0) & ((side[sad] >> d) & 1).astype(bool)
        e[:, d] = np.where(on, erank[lab[np.where(on, u, 0)]], -1)
    rows, cnt = _rows_sorted_unique(e)
    opposite = int(np.argmax(rank == 0))            # first in the tree's order
    return {"rank": rank, "ext": ext, "sad": sad, "rows": rows, "cnt": cnt,
            "opposite": opposite}


def persistence_tree(f: np.ndarray, split: bool = True):
    """(pairs (n, 2), merge targets (n,)) of one tree, extrema by rank.

    pairs[k] = (partner vertex, extremum vertex); targets[k] = the vertex of
    the extremum it merges into (the global extremum: itself; unpaired: -1).
    """
    gr = extremum_graph(f, split)
    ext, sad, rows, cnt = gr["ext"], gr["sad"], gr["rows"], gr["cnt"]
    ne, ns = len(ext), len(sad)
    glob = ne - 1
    ptr = np.arange(ne)
    pair = np.full(ne, -1, np.int64)
    target = np.full(ne, -1, np.int64)
    while True:
        largest = np.full(ne, ns, np.int64)
        ri, ci = np.nonzero(rows >= 0)
        ent = rows[ri, ci]
        keep = ent != glob
        np.minimum.at(largest, ent[keep], ri[keep])
        cand = np.flatnonzero((largest < ns) & (pair < 0))
        li = largest[cand]
        win = rows[li, 0] == cand
        cand, li = cand[win], li[win]
        if len(cand) == 0:
            break
        pair[cand] = li
        last = rows[li, cnt[li] - 1]
        ptr[cand] = last
        target[cand] = last
        while True:
            nxt = ptr[ptr]
            if np.array_equal(nxt, ptr):
                break
            ptr = nxt
        e = np.where(rows >= 0, ptr[np.where(rows >= 0, rows, 0)], -1)
        rows, cnt = _rows_sorted_unique(e)
    opposite = gr["opposite"]
    out = np.empty((ne, 2), np.int64)
    out[:, 1] = ext
    out[:, 0] = np.where(pair >= 0, sad[np.maximum(pair, 0)], -1)
    out[glob, 0] = opposite
    tv = np.where(target >= 0, ext[np.maximum(target, 0)], -1)
    tv[glob] = ext[glob]
    return out, tv
