"""The 14-entry sorting network of k_rows sorts every input.

k_rows orders each saddle row with the comparator list kSort14
(extrem_z_b200/csrc/extremz_kernels.cuh).  By the 0-1 principle a comparator
network sorts every input if it sorts every input of zeros and ones, so all
2^14 such inputs are run through the table as the header holds it.
"""

import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(os.path.dirname(HERE), "extrem_z_b200", "csrc", "extremz_kernels.cuh")


def network():
    text = open(SRC).read()
    size = int(re.search(r"constexpr int kSort14Size = (\d+);", text).group(1))
    body = re.search(r"kSort14\[kSort14Size\]\[2\] = \{(.*?)\};", text, re.S).group(1)
    pairs = [(int(a), int(b)) for a, b in re.findall(r"\{(\d+),\s*(\d+)\}", body)]
    assert len(pairs) == size
    return pairs


def test_network_sorts_every_zero_one_input():
    pairs = network()
    assert all(0 <= a < b < 14 for a, b in pairs)
    bits = (np.arange(1 << 14)[:, None] >> np.arange(14)[None, :]) & 1
    a = bits.copy()
    for x, y in pairs:
        lo = np.minimum(a[:, x], a[:, y])
        hi = np.maximum(a[:, x], a[:, y])
        a[:, x], a[:, y] = lo, hi
    assert np.array_equal(a, np.sort(bits, axis=1))


def test_network_sorts_rows_with_repeated_labels():
    """Random rows as k_rows builds them: (value, label) pairs, repeated labels
    carrying the same value, left-out entries as the largest key."""
    pairs = network()
    rng = np.random.default_rng(5)
    for _ in range(2000):
        n = int(rng.integers(0, 15))
        labels = rng.integers(0, 6, size=n)
        vals = rng.integers(0, 3, size=6).astype(np.float64)[labels]
        keys = [(v, int(lab)) for v, lab in zip(vals, labels)] + [(np.inf, 1 << 40)] * (14 - n)
        perm = rng.permutation(14)
        e = [keys[p] for p in perm]
        for x, y in pairs:
            if e[x] > e[y]:
                e[x], e[y] = e[y], e[x]
        assert e[:n] == sorted(keys[:n])
