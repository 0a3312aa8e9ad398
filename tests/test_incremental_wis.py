"""The rule behind the incremental wrong-saddle scan, checked on the CPU.

get_wrong_index_saddles gives each maximum the first entry (row order, then
entry order) of a row that names it and whose saddle outranks the maximum's
true largest saddle.  That result reads only the values of the saddles whose
rows name the maximum (the true largest saddle is one of them), so after a
change of some saddles' values only the maxima named in those saddles' rows
need recomputing (k_wis_mark, k_wis_update).  Here random row sets and value
changes are checked against a full recomputation.
"""

import numpy as np
import pytest


def first_wrong(rows, best, g, sad):
    """Per maximum: min key i*15+p over entries (i, p) naming it whose saddle
    outranks the maximum's true largest saddle (value, then id), else inf."""
    out = {}
    for i, row in enumerate(rows):
        s = sad[i]
        for p, m in enumerate(row):
            t = best[m]
            wrong = g[s] > g[t] or (g[s] == g[t] and s > t)
            if wrong:
                out[m] = min(out.get(m, np.inf), i * 15 + p)
    return out


@pytest.mark.parametrize("seed", range(20))
def test_recomputing_named_maxima_equals_full_scan(seed):
    rng = np.random.default_rng(seed)
    n_sad, n_max = 60, 15
    sad = np.sort(rng.choice(1000, size=n_sad, replace=False))
    rows = [sorted(set(rng.integers(0, n_max, size=int(rng.integers(1, 5))).tolist()))
            for _ in range(n_sad)]
    g = rng.integers(0, 8, size=1000).astype(float)  # ties happen
    # Each maximum's true largest saddle is a saddle whose row names it.
    best = {}
    for i, row in enumerate(rows):
        for m in row:
            if m not in best or rng.random() < 0.3:
                best[m] = sad[i]
    named = sorted(best)
    before = first_wrong(rows, best, g, sad)
    # Change the values of some saddles.
    idx = rng.choice(n_sad, size=int(rng.integers(1, 8)), replace=False)
    g2 = g.copy()
    g2[sad[idx]] += rng.integers(-3, 4, size=idx.size)
    full = first_wrong(rows, best, g2, sad)
    affected = {m for i in idx for m in rows[i]}
    inc = {m: v for m, v in before.items() if m not in affected}
    sub = first_wrong(rows, best, g2, sad)
    for m in affected:
        if m in sub:
            inc[m] = sub[m]
    assert {m: full.get(m) for m in named} == {m: inc.get(m) for m in named}
