"""Edit streams on the GPU against the oracle's encoder.

The corrected field, the index stream (3-bit counters for edit_type 0,
delta-coded ids for edit_type 1) and the lossless edits must equal the
oracle's byte for byte; the edited and entry counts exactly; PSNR (a sum in
another order) to 1e-9 relative.
"""

import numpy as np
import pytest

from extrem_z_b200 import synth

pytestmark = pytest.mark.gpu

KW = dict(q=4, max_outer=500, max_cloop_rounds=100000, final_join=True)


def _both(fld, edit_type):
    import torch
    from extrem_z_b200 import api
    from oracle import ffi
    cnt = np.zeros(fld.f.size, np.int32)
    ref, rrep, _ = ffi.correct(fld.f, fld.decp, fld.eb, edit_type=edit_type, counter_out=cnt, **KW)
    ridx, redits, rs = ffi.encode(fld.f, fld.decp, ref, cnt, fld.eb, q=KW["q"],
                                  edit_type=edit_type)
    tf = torch.from_numpy(np.ascontiguousarray(fld.f)).cuda()
    tg = torch.from_numpy(np.ascontiguousarray(fld.decp)).cuda()
    rep, es = api.context(0).correct_encode(tf, tg, fld.eb, edit_type=edit_type, **KW)
    return (ref, rrep, ridx, redits, rs), (tg.cpu().numpy(), rep, es)


def _check(oracle, gpu):
    ref, rrep, ridx, redits, rs = oracle
    out, rep, es = gpu
    assert np.array_equal(out.view(np.uint8), ref.view(np.uint8))
    assert rep.status == rrep["status"]
    assert es["edited"] == rs["edited"] and es["n_edits"] == rs["n_edits"]
    assert np.array_equal(es["index"], ridx)
    assert np.array_equal(es["edits"].view(np.uint8), redits.view(np.uint8))
    for k in ("psnr_before", "psnr_after"):
        assert abs(es[k] - rs[k]) <= 1e-9 * abs(rs[k]), (k, es[k], rs[k])


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("edit_type", [0, 1])
def test_edit_stream_plain64(dtype, edit_type):
    fld = synth.plain_64(dtype)
    oracle, gpu = _both(fld, edit_type)
    _check(oracle, gpu)
    assert gpu[2]["edited"] > 0


@pytest.mark.parametrize("shape", [(37, 29, 1), (23, 17, 11)])
def test_edit_stream_uneven(shape):
    w, h, d = shape
    fld = synth.make_field(w, h, d, n_gauss=10, seed=w * h + d, rel=3e-3, dtype=np.float64)
    for et in (0, 1):
        oracle, gpu = _both(fld, et)
        _check(oracle, gpu)


def test_edit_stream_zstd_and_sizes():
    fld = synth.plain_64(np.float32)
    _, (out, rep, es) = _both(fld, 0)
    n = fld.f.size
    assert es["index_bytes"] == (3 * n + 7) // 8 == es["index"].size
    assert es["edit_bytes"] == 4 * es["n_edits"]
    assert es["index_zstd"] == -1 or 0 < es["index_zstd"] < es["index_bytes"]


def test_edit_stream_buffer_too_small():
    import ctypes
    import torch
    from extrem_z_b200 import api
    fld = synth.plain_64(np.float64)
    tf = torch.from_numpy(fld.f).cuda()
    tg = torch.from_numpy(fld.decp.copy()).cuda()
    small = torch.empty(16, dtype=torch.uint8, device="cuda")
    es = api.EditStream()
    es.index, es.index_cap = small.data_ptr(), 16
    es.edits, es.edits_cap = small.data_ptr(), 16
    p = api.make_params(fld.eb, edit_type=1, **KW)
    r = api.Report()
    ctx = api.context(0)
    st = api.load().extremz_correct_encode(ctx._h, tf.data_ptr(), tg.data_ptr(), api.F64, 64, 64,
                                           64, ctypes.byref(p), ctypes.byref(r), None,
                                           ctypes.byref(es))
    torch.cuda.synchronize()
    assert st == api.BAD_ARG
    assert es.index_bytes == 4 * es.edited > 16   # the sizes needed are reported
