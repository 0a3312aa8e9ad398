"""Batched correction: every field of a mixed batch is bit-identical to the
same field corrected alone, with the same round counts and final counters.

The batch shares one launch per kernel among all fields at the same phase;
the branches of each field read only that field's counters, so the mix must
not change any field's result.  Fields differ in dtype, shape (3-D volumes,
2-D slices, non-cubic), bound and parameters.
"""

import numpy as np
import pytest

from extrem_z_b200 import synth

pytestmark = pytest.mark.gpu

KW = dict(q=4, edit_type=1, max_outer=500, max_cloop_rounds=100000, final_join=True)


def _plain(fld, **kw):
    import torch
    from extrem_z_b200 import api
    tf = torch.from_numpy(np.ascontiguousarray(fld.f)).cuda()
    tg = torch.from_numpy(np.ascontiguousarray(fld.decp)).cuda()
    rep, _ = api.context(0).correct_device(tf, tg, fld.eb, **kw)
    torch.cuda.synchronize()
    return tg.cpu().numpy(), rep


def _batch(fields, kws):
    import torch
    from extrem_z_b200 import api
    items, outs = [], []
    for fld, kw in zip(fields, kws):
        tf = torch.from_numpy(np.ascontiguousarray(fld.f)).cuda()
        tg = torch.from_numpy(np.ascontiguousarray(fld.decp)).cuda()
        items.append((tf, tg, fld.eb, kw))
        outs.append(tg)
    reps, launches = api.context(0).correct_batch(items)
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in outs], reps, launches


def _same_report(a, b):
    return (a.status, a.outer_iters, a.cloop_rounds, a.manifold_rounds, a.counters,
            a.error_bits) == (b.status, b.outer_iters, b.cloop_rounds, b.manifold_rounds,
                              b.counters, b.error_bits)


def _small(spec, scale):
    s = dict(spec)
    s["w"] = max(6, s["w"] // scale)
    s["h"] = max(6, s["h"] // scale)
    if s["d"] > 1:
        s["d"] = max(4, s["d"] // scale)
    s["n_gauss"] = max(8, s["n_gauss"] // 4)
    return s


def _make(spec):
    return synth.make_field(spec["w"], spec["h"], spec["d"], n_gauss=spec["n_gauss"],
                            seed=spec["seed"], rel=spec["rel"], dtype=spec["dtype"])


def test_mixed_batch_equals_plain():
    specs = [_small(s, 2) for s in synth.mixed_batch_specs(12)]
    fields = [_make(s) for s in specs]
    kws = [dict(KW) for _ in fields]
    kws[1]["preserve_join"] = True
    kws[2]["edit_type"] = 0
    # With a persistence filter this field never reaches zero (the oracle
    # agrees: a wrong_max_2 count of 4 stays); a small cap ends it.
    kws[3].update(thr=float(fields[3].eb) * 0.25, max_outer=20)
    outs, reps, launches = _batch(fields, kws)
    plain_launches = 0
    for i, (fld, kw) in enumerate(zip(fields, kws)):
        ref, rrep = _plain(fld, **kw)
        plain_launches += rrep.kernel_launches
        assert np.array_equal(outs[i].view(np.uint8), ref.view(np.uint8)), (i, specs[i])
        assert _same_report(reps[i], rrep), (i, reps[i], rrep)
        assert reps[i].status == (1 if i == 3 else 0)
    # Shared launches: the batch launches far fewer kernels than the loop.
    assert 0 < launches < plain_launches


def test_batch_beyond_slot_limit():
    # More fields of one dtype than the engine has slots: the rest are
    # admitted as earlier ones finish.
    fields, kws = [], []
    for i in range(70):
        dt = np.float32 if i % 9 else np.float64
        w, h, d = 10 + i % 7, 9 + i % 5, 1 + i % 6
        fields.append(synth.make_field(w, h, d, n_gauss=8, seed=500 + i, rel=1e-2, dtype=dt))
        kws.append(dict(KW))
    outs, reps, _ = _batch(fields, kws)
    for i, (fld, kw) in enumerate(zip(fields, kws)):
        ref, rrep = _plain(fld, **kw)
        assert np.array_equal(outs[i].view(np.uint8), ref.view(np.uint8)), i
        assert _same_report(reps[i], rrep), i


def test_batch_matches_oracle():
    from oracle import ffi
    specs = [_small(s, 4) for s in synth.mixed_batch_specs(6, first_seed=200)]
    fields = [_make(s) for s in specs]
    kws = [dict(KW) for _ in fields]
    outs, reps, _ = _batch(fields, kws)
    for i, fld in enumerate(fields):
        ref, rrep, _ = ffi.correct(fld.f, fld.decp, fld.eb, **KW)
        assert np.array_equal(outs[i].view(np.uint8), ref.view(np.uint8)), (i, specs[i])
        assert reps[i].status == rrep["status"] == 0
        assert reps[i].counters == rrep["counters"]


def test_batch_round_cap_per_field():
    # A cap on one field ends that field only; the others run to zero.
    fields = [synth.plain_64(np.float32)] + [
        synth.make_field(20, 18, 12, n_gauss=8, seed=700 + i, rel=3e-3, dtype=np.float64)
        for i in range(3)]
    kws = [dict(KW, max_outer=0)] + [dict(KW) for _ in range(3)]
    outs, reps, _ = _batch(fields, kws)
    for i, (fld, kw) in enumerate(zip(fields, kws)):
        ref, rrep = _plain(fld, **kw)
        assert np.array_equal(outs[i].view(np.uint8), ref.view(np.uint8)), i
        assert _same_report(reps[i], rrep), i
    assert reps[0].status == 1
    assert all(r.status == 0 for r in reps[1:])


def test_empty_batch():
    from extrem_z_b200 import api
    reps, launches = api.context(0).correct_batch([])
    assert reps == [] and launches == 0
