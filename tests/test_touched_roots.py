"""The rule behind the later manifold rounds' skipping, checked on the CPU.

A later round recomputes the steepest pointers of the tiles whose tile or halo
holds a changed value, marks the current labels of those tiles' vertices as
touched roots, and follows the chains only of vertices whose old label is
touched (k_direction_list, k_jump2).  That is exact when every vertex whose
label changes has a touched old label: its old path must meet a changed
pointer, which lies in a recomputed tile, and every vertex of a path carries
the path's label.  Here random fields are lowered at random voxels (as the
correction does) and the rule is checked against a full recomputation, with a
plain steepest-ascent stencil (the argument does not depend on the stencil).
"""

import numpy as np
import pytest

SHAPE = (12, 16, 24)  # z, y, x
TILE = (2, 4, 8)


def steepest(vals):
    """Steepest-ascent pointer of every voxel over its 6 neighbours, ties by
    the larger id; a voxel above all its neighbours points to itself."""
    d, h, w = vals.shape
    ids = np.arange(vals.size).reshape(vals.shape)
    best_v = vals.copy()
    best_i = ids.copy()
    for ax in range(3):
        for s in (-1, 1):
            nv = np.full(vals.shape, -np.inf)
            ni = np.full(vals.shape, -1)
            src = [slice(None)] * 3
            dst = [slice(None)] * 3
            if s == 1:
                src[ax], dst[ax] = slice(1, None), slice(None, -1)
            else:
                src[ax], dst[ax] = slice(None, -1), slice(1, None)
            nv[tuple(dst)] = vals[tuple(src)]
            ni[tuple(dst)] = ids[tuple(src)]
            better = (nv > best_v) | ((nv == best_v) & (ni > best_i))
            best_v = np.where(better, nv, best_v)
            best_i = np.where(better, ni, best_i)
    return best_i.reshape(-1)


def roots(ptr):
    lab = ptr.copy()
    while True:
        nxt = lab[lab]
        if np.array_equal(nxt, lab):
            return lab
        lab = nxt


def tile_of(idx):
    z, y, x = np.unravel_index(idx, SHAPE)
    return (z // TILE[0], y // TILE[1], x // TILE[2])


@pytest.mark.parametrize("seed", range(12))
def test_changed_labels_have_touched_old_labels(seed):
    rng = np.random.default_rng(seed)
    vals = rng.normal(size=SHAPE).cumsum(axis=2)  # smooth-ish along x: long paths
    ptr0 = steepest(vals)
    lab0 = roots(ptr0)
    # Lower a few voxels, as the correction's edits do.
    changed = rng.choice(vals.size, size=int(rng.integers(1, 12)), replace=False)
    new = vals.copy().reshape(-1)
    new[changed] -= rng.uniform(0.1, 3.0, size=changed.size)
    new = new.reshape(SHAPE)
    # Tiles whose tile or halo (one voxel) holds a changed value.
    marked = set()
    for c in changed:
        z, y, x = np.unravel_index(c, SHAPE)
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    zz, yy, xx = z + dz, y + dy, x + dx
                    if 0 <= zz < SHAPE[0] and 0 <= yy < SHAPE[1] and 0 <= xx < SHAPE[2]:
                        marked.add((zz // TILE[0], yy // TILE[1], xx // TILE[2]))
    ptr1 = steepest(new)
    all_ids = np.arange(vals.size)
    in_marked = np.array([tile_of(i) in marked for i in all_ids])
    # Pointers outside the recomputed tiles depend on nothing that changed.
    assert np.array_equal(ptr0[~in_marked], ptr1[~in_marked])
    lab1 = roots(ptr1)
    touched = set(lab0[in_marked].tolist())
    moved = np.flatnonzero(lab1 != lab0)
    assert all(int(lab0[v]) in touched for v in moved)
    # Following only the touched vertices' chains reproduces the labels.
    follow = np.isin(lab0, list(touched))
    fast = lab0.copy()
    fast[follow] = lab1[follow]
    assert np.array_equal(fast, lab1)
