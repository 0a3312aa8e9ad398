"""The allocation-free entry point gives the same field as the regular one.

extremz_correct_device_noalloc serves callers that cannot allocate device
memory while they correct a field (an application whose allocator owns the
device memory, real-time code that allows no allocation after start-up).  Its workspace is a static device array shared by
all calls, so two calls in a row must both match the regular entry point: the
second call must not see anything the first one left in the array.  This file
is collected last so that a failure here stops a -x run only after everything
else has run.
"""

import numpy as np
import pytest

from extrem_z_b200 import synth

pytestmark = pytest.mark.gpu

KW = dict(q=4, edit_type=1, max_outer=500, max_cloop_rounds=100000, final_join=True)


def _regular(f, decp, eb):
    import torch
    from extrem_z_b200 import api
    tf = torch.from_numpy(f).cuda()
    tg = torch.from_numpy(decp.copy()).cuda()
    rep, _ = api.Context(0).correct_device(tf, tg, eb, **KW)
    torch.cuda.synchronize()
    return tg.cpu().numpy(), rep


def _noalloc(f, decp, eb):
    import torch
    from extrem_z_b200 import api
    tf = torch.from_numpy(f).cuda()
    tg = torch.from_numpy(decp.copy()).cuda()
    rep = api.correct_device_noalloc(tf, tg, eb, **KW)
    torch.cuda.synchronize()
    return tg.cpu().numpy(), rep


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_noalloc_matches_regular_entry_point_twice(dtype):
    from extrem_z_b200 import api
    fld = synth.make_field(40, 32, 24, n_gauss=16, seed=31, rel=1e-3, dtype=dtype)
    assert fld.f.size <= api.noalloc_max_voxels()
    ref, rrep = _regular(fld.f, fld.decp, fld.eb)
    # Bit-exact (the tolerance of every parity test here): same bytes.
    for _ in range(2):
        out, rep = _noalloc(fld.f, fld.decp, fld.eb)
        assert rep.status == rrep.status == 0
        assert rep.outer_iters == rrep.outer_iters
        assert np.array_equal(out.view(np.uint8), ref.view(np.uint8))


def test_noalloc_second_call_unaffected_by_a_different_first_call():
    """A first call on another field (other shape, seed and dtype, near the
    maximum size, with many more critical points) leaves its state in the
    shared workspace; the next call must still match the regular entry point
    byte for byte, so nothing it reads may be left over."""
    from extrem_z_b200 import api
    n_max = api.noalloc_max_voxels()
    big = synth.make_field(48, 40, 32, n_gauss=40, seed=77, rel=3e-4, dtype=np.float64)
    small = synth.make_field(36, 28, 20, n_gauss=12, seed=78, rel=2e-3, dtype=np.float32)
    assert big.f.size <= n_max and big.f.size > 0.9 * n_max
    ref_big, _ = _regular(big.f, big.decp, big.eb)
    ref_small, rrep = _regular(small.f, small.decp, small.eb)
    for fld, ref in ((big, ref_big), (small, ref_small), (big, ref_big), (small, ref_small)):
        out, rep = _noalloc(fld.f, fld.decp, fld.eb)
        assert rep.status == 0
        assert np.array_equal(out.view(np.uint8), ref.view(np.uint8))
    assert rep.outer_iters == rrep.outer_iters


def test_noalloc_rejects_fields_beyond_its_maximum():
    import torch
    from extrem_z_b200 import api
    n = api.noalloc_max_voxels()
    d = n // (64 * 64) + 1
    f = torch.zeros((d, 64, 64), dtype=torch.float32, device="cuda")
    with pytest.raises(api.ExtremzError) as ei:
        api.correct_device_noalloc(f, f.clone(), 0.1, **KW)
    assert ei.value.status == api.TOO_LARGE
