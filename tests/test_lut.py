"""Critical-point lookup table pinned to the reference's src/LUT.bin."""

import hashlib
import json
import os

import numpy as np
import pytest

from oracle import ffi

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference checkout, when one is named (e.g. EXTREMZ_REFERENCE_DIR=<checkout>).
_REF_DIR = os.environ.get("EXTREMZ_REFERENCE_DIR", "")
REFERENCE_LUT = os.path.join(_REF_DIR, "src", "LUT.bin") if _REF_DIR else ""


def _digest():
    with open(os.path.join(HERE, "golden", "lut_digest.json")) as fh:
        return json.load(fh)


def test_oracle_lut_matches_reference_digest():
    lut = ffi.lut().astype("<i4")
    d = _digest()
    assert lut.size == d["entries"]
    assert hashlib.sha256(lut.tobytes()).hexdigest() == d["sha256"]
    vals, counts = np.unique(lut, return_counts=True)
    assert {str(int(v)): int(c) for v, c in zip(vals, counts)} == d["histogram"]


def test_library_lut_matches_oracle():
    from extrem_z_b200 import api
    assert np.array_equal(api.lut(), ffi.lut())


@pytest.mark.skipif(not os.path.exists(REFERENCE_LUT), reason="EXTREMZ_REFERENCE_DIR names no reference checkout")
def test_oracle_lut_matches_reference_file_entrywise():
    ref = np.fromfile(REFERENCE_LUT, dtype="<i4")
    assert np.array_equal(ffi.lut(), ref)
