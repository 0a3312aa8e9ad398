"""extremz_correct_host writes back only the voxels whose value changed.

The caller's buffer still holds the decompressed field when the correction
ends, so the library copies back the changed voxels' ids and values (or the
whole field when more than 1/16 of the voxels changed).  Either way the host
buffer must end bit-identical to the device-resident correction, including
fields whose decompressed values hold signed zeros.
"""

import dataclasses

import numpy as np
import pytest

from extrem_z_b200 import synth

pytestmark = pytest.mark.gpu

KW = dict(q=4, max_outer=500, max_cloop_rounds=100000, final_join=True)


def _device(fld, **kw):
    import torch
    from extrem_z_b200 import api
    tf = torch.from_numpy(np.ascontiguousarray(fld.f)).cuda()
    tg = torch.from_numpy(np.ascontiguousarray(fld.decp)).cuda()
    rep, _ = api.context(0).correct_device(tf, tg, fld.eb, **kw)
    return tg.cpu().numpy(), rep


def _changed(a, b):
    s = a.dtype.itemsize
    return int(np.count_nonzero((a.view(np.uint8) != b.view(np.uint8)).reshape(-1, s).any(axis=1)))


def _host(fld, **kw):
    from extrem_z_b200 import api
    host = np.ascontiguousarray(fld.decp).copy()
    rep = api.context(0).correct_host(np.ascontiguousarray(fld.f), host, fld.eb, **kw)
    return host, rep


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("edit_type", [0, 1])
def test_sparse_edits_come_back_as_a_list(dtype, edit_type):
    # 64^3, 64 Gaussians, eb 1e-4 rel: well under 1/16 of the voxels change.
    fld = synth.make_field(64, 64, 64, n_gauss=64, seed=1, rel=1e-4, dtype=dtype)
    dev, rdev = _device(fld, edit_type=edit_type, **KW)
    host, rhost = _host(fld, edit_type=edit_type, **KW)
    assert np.array_equal(dev.view(np.uint8), host.view(np.uint8))
    assert rhost.status == rdev.status
    n = fld.f.size
    s = np.dtype(dtype).itemsize
    changed = _changed(dev, fld.decp)
    assert 0 < changed and changed * 16 <= n
    # The list path: ids and values of the changed voxels (values only go
    # down, so a voxel that changed once differs at the end), plus the count.
    assert rhost.host_bytes_back == changed * (4 + s) + 4


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_plain64_host_equals_device(dtype):
    fld = synth.plain_64(dtype)
    dev, _ = _device(fld, **KW)
    host, rhost = _host(fld, **KW)
    assert np.array_equal(dev.view(np.uint8), host.view(np.uint8))
    n, s = fld.f.size, np.dtype(dtype).itemsize
    changed = _changed(dev, fld.decp)
    want = changed * (4 + s) + 4 if changed * 16 <= n else n * s + 4
    assert rhost.host_bytes_back == want


def test_signed_zeros_survive_the_write_back():
    # Decompressed values of -0.0 that the correction leaves alone must stay
    # -0.0 in the host buffer, and changed ones take the device's bits.
    fld = synth.make_field(40, 36, 12, n_gauss=12, seed=5, rel=2e-2, dtype=np.float64)
    decp = fld.decp.copy()
    zero = decp == 0                  # quantised to zero: same value, sign bit set
    decp[zero] = -0.0
    fld = dataclasses.replace(fld, decp=decp)
    assert np.signbit(decp[zero]).all() and zero.any()
    dev, _ = _device(fld, **KW)
    host, _ = _host(fld, **KW)
    assert np.array_equal(dev.view(np.uint8), host.view(np.uint8))


def test_dense_edits_copy_the_whole_field():
    # A coarse bound on a noisy field: more than 1/16 of the voxels change.
    fld = synth.make_field(48, 40, 24, n_gauss=4, seed=9, rel=5e-2, dtype=np.float32)
    dev, _ = _device(fld, **KW)
    host, rhost = _host(fld, **KW)
    assert np.array_equal(dev.view(np.uint8), host.view(np.uint8))
    changed = _changed(dev, fld.decp)
    assert changed * 16 > fld.f.size
    assert rhost.host_bytes_back == fld.f.size * 4 + 4
