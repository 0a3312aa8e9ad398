"""The reference's own driver main.cpp, linked unchanged against libExtreMz.so
(the reference host API over this library), corrects a 3-D field on the GPU.

extrem_z_b200/compat/build_reference_main.sh builds the program from the
reference checkout when one is present (build() runs it); the built program
travels with the repository.  main.cpp lowers the global extrema and the
original saddles to f - bound before its first c_loops call
(main.cpp:74-75, :122-131) and preserves the join tree (main.cpp:21); its
fixed.bin must equal, byte for byte, the library's correction
(extremz_correct_host) of that field with the join tree preserved and no
final join-saddle pass, and the oracle's.
"""

import os
import subprocess

import numpy as np
import pytest

from extrem_z_b200 import synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROGRAM = os.path.join(ROOT, "extrem_z_b200", "compat", "_build", "extrem_main")
KW = dict(q=4, edit_type=1, max_outer=1000, max_cloop_rounds=100000, final_join=False,
          preserve_join=True)


def _main_cpp_edits(f, decp, bound):
    """The edits main.cpp makes before its first c_loops call."""
    from oracle import ffi
    g = decp.copy().reshape(-1)
    ff = f.reshape(-1)
    order = np.lexsort((np.arange(ff.size), ff))     # (value, id) ascending
    for v in (order[0], order[-1]):                  # main.cpp:74-75
        g[v] = ff[v] - bound
    t, _ = ffi.classify(f)
    sad = (t == 1) | (t == 2) | (t == 3)             # saddles2 and saddles1, main.cpp:122-131
    g[sad] = ff[sad] - bound
    return g.reshape(f.shape)


@pytest.mark.skipif(not os.path.exists(PROGRAM), reason="reference main.cpp not built here")
@pytest.mark.parametrize("shape,seed,rel", [((36, 30, 22), 51, 1e-3), ((48, 40, 1), 52, 2e-3)])
def test_reference_main_on_the_layer_matches_the_library(tmp_path, shape, seed, rel):
    from extrem_z_b200 import api
    from oracle import ffi
    w, h, d = shape
    fld = synth.make_field(w, h, d, n_gauss=12, seed=seed, rel=rel)
    fld.f.tofile(tmp_path / "orig.f64")
    fld.decp.tofile(tmp_path / "decp.f64")
    env = dict(os.environ, EXTREMZ_DECP_FILE=str(tmp_path / "decp.f64"))
    p = subprocess.run([PROGRAM, f"orig.f64,{w},{h},{d}", repr(rel), "sz3"], cwd=tmp_path,
                       env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    assert "ended" in p.stdout
    fixed = np.fromfile(tmp_path / "fixed.bin", dtype=np.float64).reshape(fld.f.shape)
    g = _main_cpp_edits(fld.f, fld.decp, fld.eb)
    lib_out, rep = api.correct(fld.f, g, fld.eb, **KW)
    assert rep.status == 0
    assert np.array_equal(fixed.view(np.uint8), lib_out.view(np.uint8))
    ref, rrep, _ = ffi.correct(fld.f, g, fld.eb, **KW)
    assert rrep["status"] == 0
    assert np.array_equal(fixed.view(np.uint8), ref.view(np.uint8))
    # main.cpp's loop ended on the corrected field's own counters, all zero.
    assert ffi.census(fld.f, fixed) == [0] * 11
