"""The C-ABI library loads and exports every entry point include/extremz.h declares."""

import ctypes
import os
import re

import pytest

from extrem_z_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(inc, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(extremz_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(api.library_path())
    names = declared_functions()
    assert len(names) >= 9
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    assert set(declared_functions()) == set(api.EXPORTS)


def test_default_params_are_the_reference_defaults():
    p = api.make_params(0.5)
    assert (p.q, p.edit_type, p.thr, p.final_join, p.preserve_join) == (4, 1, 0.0, 1, 0)


def test_version():
    assert api.load().extremz_version() == api.ABI_VERSION == 2


def test_status_strings():
    for s in range(7):
        assert api.status_string(s)


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present")
    with pytest.raises(api.ExtremzError) as ei:
        api.Context(0)
    assert ei.value.status == api.NO_DEVICE
