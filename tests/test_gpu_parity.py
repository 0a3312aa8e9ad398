"""CUDA path against the oracle: bit-exact corrected fields and equal traces.

Every comparison is exact (byte equality of the corrected field); the trace
records the per-phase counters (mismatch counts, wrong neighbours, wrong
extremum / saddle pairs) and a checksum of the field after each outer
iteration, so a divergence is located to the phase where it starts.
"""

import os

import numpy as np
import pytest

from extrem_z_b200 import synth

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = np.load(os.path.join(HERE, "golden", "oracle_cases.npz"))
CASES = sorted({k.split("/")[0] for k in GOLDEN.files})
KW = dict(q=4, edit_type=1, max_outer=500, max_cloop_rounds=100000, final_join=True)


def gpu_correct(f, decp, eb, trace_cap=200000, **kw):
    import torch
    from extrem_z_b200 import api
    tf = torch.from_numpy(np.ascontiguousarray(f)).cuda()
    tg = torch.from_numpy(np.ascontiguousarray(decp)).cuda()
    rep, trace = api.context(0).correct_device(tf, tg, eb, trace_cap=trace_cap, **kw)
    torch.cuda.synchronize()
    return tg.cpu().numpy(), rep, trace


def first_divergence(a, b):
    n = min(len(a), len(b))
    for i in range(n):
        if not np.array_equal(a[i], b[i]):
            return i, a[i].tolist(), b[i].tolist()
    return n, None, None


@pytest.mark.parametrize("name", CASES)
def test_golden_cases_bit_exact(name):
    f, decp = GOLDEN[f"{name}/f"], GOLDEN[f"{name}/decp"]
    eb, et = GOLDEN[f"{name}/meta"][:2]
    kw = dict(KW, edit_type=int(et))
    out, rep, trace = gpu_correct(f, decp, eb, **kw)
    ref_trace = GOLDEN[f"{name}/trace"]
    assert np.array_equal(trace, ref_trace), first_divergence(trace, ref_trace)
    assert np.array_equal(out.view(np.uint8), GOLDEN[f"{name}/fixed"].view(np.uint8))
    assert rep.status == 0 and rep.error_bits == 0


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("edit_type", [1, 0])
def test_plain_64_bit_exact(dtype, edit_type):
    from oracle import ffi
    fld = synth.plain_64(dtype)
    kw = dict(KW, edit_type=edit_type)
    ref, rrep, rtrace = ffi.correct(fld.f, fld.decp, fld.eb, trace_cap=400000, **kw)
    out, rep, trace = gpu_correct(fld.f, fld.decp, fld.eb, trace_cap=400000, **kw)
    assert np.array_equal(trace, rtrace), first_divergence(trace, rtrace)
    assert np.array_equal(out.view(np.uint8), ref.view(np.uint8))
    assert rep.status == rrep["status"] == 0
    assert rep.counters == rrep["counters"] == [0] * 11


@pytest.mark.parametrize("seed", [3, 17])
def test_uneven_shapes_bit_exact(seed):
    from oracle import ffi
    rng = np.random.default_rng(seed)
    w, h, d = (int(x) for x in rng.integers(5, 40, size=3))
    dt = np.float32 if seed % 2 else np.float64
    fld = synth.make_field(w, h, d, n_gauss=12, seed=seed, rel=3e-3, dtype=dt)
    ref, rrep, rtrace = ffi.correct(fld.f, fld.decp, fld.eb, trace_cap=200000, **KW)
    out, rep, trace = gpu_correct(fld.f, fld.decp, fld.eb, **KW)
    assert np.array_equal(trace, rtrace), first_divergence(trace, rtrace)
    assert np.array_equal(out.view(np.uint8), ref.view(np.uint8))


def test_host_entry_point_equals_device_entry_point():
    from extrem_z_b200 import api
    fld = synth.make_field(33, 17, 9, n_gauss=8, seed=8, rel=2e-3)
    dev, _, _ = gpu_correct(fld.f, fld.decp, fld.eb, trace_cap=0, **KW)
    host, rep = api.correct(fld.f, fld.decp, fld.eb, **KW)
    assert np.array_equal(dev.view(np.uint8), host.view(np.uint8))
    assert rep.status == 0


def test_repeated_calls_on_one_context_are_identical():
    fld = synth.make_field(20, 20, 20, n_gauss=10, seed=4, rel=1e-3)
    a, _, _ = gpu_correct(fld.f, fld.decp, fld.eb, **KW)
    b, _, _ = gpu_correct(fld.f, fld.decp, fld.eb, **KW)
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8))


def test_fields_in_turn_on_one_context_bit_exact():
    """A field corrected after another of the same shape, whose labels,
    mismatch bits and changed-input bytes are still in the workspace: the
    jump skips the stores of label groups equal to the stored ones, so each
    job's first manifold round must still write every group's mismatch bits
    (N a multiple of 4: the four-vertices-per-thread path)."""
    from oracle import ffi
    a = synth.make_field(24, 20, 16, n_gauss=10, seed=21, rel=2e-3)
    b = synth.make_field(24, 20, 16, n_gauss=14, seed=22, rel=2e-3)
    assert a.f.size % 4 == 0
    for fld in (a, b, a, a):
        ref, rrep, _ = ffi.correct(fld.f, fld.decp, fld.eb, **KW)
        out, rep, _ = gpu_correct(fld.f, fld.decp, fld.eb, trace_cap=0, **KW)
        assert np.array_equal(out.view(np.uint8), ref.view(np.uint8))
        assert rep.status == rrep["status"] == 0


@pytest.mark.parametrize("tma", [True, False])
def test_tile_load_paths_agree(tma):
    """TMA halo tiles and plain-load tiles give the same bytes (64^3 f32)."""
    from oracle import ffi
    fld = synth.plain_64(np.float32)
    ref, _, _ = ffi.correct(fld.f, fld.decp, fld.eb, **KW)
    out, rep, _ = gpu_correct(fld.f, fld.decp, fld.eb, trace_cap=0, tma=tma, **KW)
    assert np.array_equal(out.view(np.uint8), ref.view(np.uint8))
    assert rep.error_bits == 0


@pytest.mark.parametrize("seed,dtype", [(5, np.float64), (12, np.float32)])
def test_preserve_join_tree_bit_exact(seed, dtype):
    """preserve_join_tree = true (the join-tree passes s_loops_join /
    saddle_loops_join inside the loop, src/ExtreM_cuda.cu:5724-5747)."""
    from oracle import ffi
    fld = synth.make_field(28, 22, 14, n_gauss=12, seed=seed, rel=2e-3, dtype=dtype)
    kw = dict(KW, preserve_join=True)
    ref, rrep, rtrace = ffi.correct(fld.f, fld.decp, fld.eb, trace_cap=200000, **kw)
    out, rep, trace = gpu_correct(fld.f, fld.decp, fld.eb, **kw)
    assert np.array_equal(trace, rtrace), first_divergence(trace, rtrace)
    assert np.array_equal(out.view(np.uint8), ref.view(np.uint8))
    assert rep.status == rrep["status"]


def test_device_iteration_limit_returns_status_and_context_survives():
    """A device-side limit that runs out ends the call with a status, not a
    hang or a fault, and the context stays usable."""
    import torch
    from extrem_z_b200 import api
    fld = synth.make_field(32, 32, 16, n_gauss=10, seed=6, rel=1e-3)
    ctx = api.Context(0)
    tf = torch.from_numpy(fld.f).cuda()
    tg = torch.from_numpy(fld.decp.copy()).cuda()
    with pytest.raises(api.ExtremzError) as ei:
        ctx.correct_device(tf, tg, fld.eb, device_iter_cap=1, **KW)
    assert ei.value.status == api.DEVICE_TIMEOUT
    tg.copy_(torch.from_numpy(fld.decp))
    rep, _ = ctx.correct_device(tf, tg, fld.eb, **KW)
    assert rep.status == 0 and rep.error_bits == 0


@pytest.mark.parametrize("max_outer", [0, 1])
def test_round_cap_returns_status(max_outer):
    """A cap on the outer iterations ends the call where the oracle's cap ends
    it: same status (the field below still has mismatches after the setup
    block, so a cap of 0 or 1 is reached) and the same bytes."""
    from extrem_z_b200 import api
    from oracle import ffi
    fld = synth.make_field(32, 32, 16, n_gauss=10, seed=6, rel=1e-3)
    kw = dict(KW, max_outer=max_outer)
    ref, rrep, _ = ffi.correct(fld.f, fld.decp, fld.eb, **kw)
    assert rrep["status"] == 1  # the oracle's round-cap status
    out, rep = api.correct(fld.f, fld.decp, fld.eb, **kw)
    assert rep.status == api.ROUND_CAP
    assert rep.outer_iters == rrep["outer_iters"] == max_outer
    assert np.array_equal(out.view(np.uint8), ref.view(np.uint8))


@pytest.mark.parametrize("case", [("cube64_s0", 64, 64, 64, 64, 0, 1e-3),
                                  ("box48x40x24_s12", 48, 40, 24, 24, 12, 3e-3)])
def test_ascending_resolution_bit_exact(case):
    """EXTREMZ_FLAG_WN_ASCENDING against the oracle's ascending resolution of
    the wrong-neighbour race: same trace, same bytes (float64 fields on which
    it differs from the default lockstep resolution)."""
    from oracle import ffi
    _, w, h, d, g, seed, rel = case
    fld = synth.make_field(w, h, d, n_gauss=g, seed=seed, rel=rel)
    ref, rrep, rtrace = ffi.correct(fld.f, fld.decp, fld.eb, trace_cap=200000,
                                    wn_order="ascending", **KW)
    lock, _, _ = ffi.correct(fld.f, fld.decp, fld.eb, **KW)
    assert not np.array_equal(ref.view(np.uint8), lock.view(np.uint8))
    out, rep, trace = gpu_correct(fld.f, fld.decp, fld.eb, wn_order="ascending", **KW)
    assert np.array_equal(trace, rtrace), first_divergence(trace, rtrace)
    assert np.array_equal(out.view(np.uint8), ref.view(np.uint8))
    assert rep.status == rrep["status"] == 0
