"""libExtreMz.so, the reference's host API (include/api/ExtreM.h) over the C
ABI, on CPU: it exports every global and function the API restatement in
extrem_z_b200/compat/extrem_api.h declares, with C linkage as the reference
header gives them, and the reference's own driver main.cpp compiles and links
against it unchanged when a reference checkout is named."""

import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "extrem_z_b200")
HEADER = os.path.join(PKG, "compat", "extrem_api.h")


def _lib():
    from extrem_z_b200 import build
    return build.build_compat()


def _declared():
    text = open(HEADER).read()
    text = re.sub(r"//[^\n]*", "", text)
    body = text[text.index('extern "C" {'):]
    funcs = set(re.findall(r"\b(?:void|int)\s+([A-Za-z_][A-Za-z0-9_]*)\s*\(", body))
    vars_ = set()
    for decl in re.findall(r"extern\s+([^;(]+);", body):
        while "<" in decl:  # template arguments hold commas: drop them
            decl = re.sub(r"<[^<>]*>", "", decl)
        for part in decl.split(","):
            name = re.findall(r"([A-Za-z_][A-Za-z0-9_]*)\s*(?:\[[^\]]*\])*\s*$", part.strip())
            if name:
                vars_.add(name[0])
    return funcs, vars_


def _exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True,
                         check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if ln.strip()}


def test_layer_exports_the_whole_declared_api_with_c_linkage():
    funcs, vars_ = _declared()
    assert {"c_loops", "r_loops", "s_loops", "saddle_loops", "getdata", "compute_MergeT",
            "classifyAllVertices", "ComputeDescendingManifold"} <= funcs
    assert {"input_data", "decp_data", "bound", "directions", "count_f_max",
            "saddleTriplets"} <= vars_
    syms = _exported(_lib())
    missing = sorted((funcs | vars_) - syms)
    assert not missing, missing
    assert "_ZNK6Branch5printEv" in syms  # Branch::print() const


def test_directions_hold_the_reference_stencil():
    import ctypes
    lib = ctypes.CDLL(_lib())
    arr = (ctypes.c_int * 78).in_dll(lib, "directions")
    dirs = [tuple(arr[3 * d:3 * d + 3]) for d in range(14)]
    assert dirs == [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
                    (-1, 1, 0), (1, -1, 0), (0, 1, 1), (0, -1, -1), (-1, 0, 1), (1, 0, -1),
                    (-1, 1, 1), (1, -1, -1)]
    assert all(arr[i] == 0 for i in range(42, 78))


_REF = os.environ.get("EXTREMZ_REFERENCE_DIR", "")


@pytest.mark.skipif(not (_REF and os.path.exists(os.path.join(_REF, "main.cpp"))),
                    reason="EXTREMZ_REFERENCE_DIR names no reference checkout")
def test_reference_main_links_unchanged(tmp_path):
    _lib()
    out = tmp_path / "extrem_main"
    subprocess.run(["g++", "-std=c++17", "-O2", "-fopenmp", "-w", "-I",
                    os.path.join(_REF, "include", "api"), os.path.join(_REF, "main.cpp"),
                    "-L", PKG, "-lExtreMz", f"-Wl,-rpath,{PKG}", "-o", str(out)], check=True)
    assert out.exists()
