"""The committed benchmark digests still follow from the oracle (CPU).

tests/golden/config_hashes.json is made once by
tests/golden/make_config_hashes.py; the GPU tests compare the library against
it.  Here the smallest configuration (64^3 float32, both final-join
settings) and a few fields of the mixed batch are recomputed by the oracle on
the CPU and must give the committed corrected-field digests, reports, traces
and censuses, so a change of the oracle cannot leave the fixtures behind
unnoticed.
"""

import hashlib
import importlib.util
import json
import os

import numpy as np
import pytest

from extrem_z_b200 import synth

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "config_hashes.json")) as _fh:
    DIGESTS = json.load(_fh)
_spec = importlib.util.spec_from_file_location(
    "make_config_hashes", os.path.join(HERE, "golden", "make_config_hashes.py"))
GEN = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(GEN)


def _check(entry, got, trace=True):
    for k in ("fixed_sha256", "status", "outer_iters", "cloop_rounds", "manifold_rounds",
              "edited", "counters", "census"):
        assert got[k] == entry[k], k
    if trace:
        assert got["trace_sha256"] == entry["trace_sha256"]


@pytest.mark.parametrize("final_join", [1, 0])
def test_plain64_f32_digest_from_oracle(final_join):
    fld = synth.plain_64(np.float32)
    got = GEN.digest(fld, bool(final_join))
    _check(DIGESTS["plain64_f32"][f"final_join_{final_join}"], got)


@pytest.mark.parametrize("k", [0, 21, 42, 63])
def test_mixed_batch_field_digest_from_oracle(k):
    s = synth.mixed_batch_specs(64)[k]
    entry = DIGESTS["mixed64"]["fields"][k]
    assert entry["seed"] == s["seed"]
    fld = synth.make_field(s["w"], s["h"], s["d"], n_gauss=s["n_gauss"], seed=s["seed"],
                           rel=s["rel"], dtype=s["dtype"])
    _check(entry["final_join_1"], GEN.digest(fld, True, trace=False), trace=False)
