"""Serving loop: each request's result is the same alone and in the mix.

Requests arrive while others are on the device (continuous batching); the
loop admits them by HBM footprint.  A field's result, round counts and final
counters must be bit-identical whether it is served alone, in a mix, or
corrected by the plain entry point.
"""

import time

import numpy as np
import pytest

from extrem_z_b200 import synth

pytestmark = pytest.mark.gpu

KW = dict(q=4, edit_type=1, max_outer=500, max_cloop_rounds=100000, final_join=True)


def _dev(fld):
    import torch
    return (torch.from_numpy(np.ascontiguousarray(fld.f)).cuda(),
            torch.from_numpy(np.ascontiguousarray(fld.decp)).cuda())


def _plain(fld):
    import torch
    from extrem_z_b200 import api
    tf, tg = _dev(fld)
    rep, _ = api.context(0).correct_device(tf, tg, fld.eb, **KW)
    torch.cuda.synchronize()
    return tg.cpu().numpy(), rep


def _key(r):
    return (r.status, r.outer_iters, r.cloop_rounds, r.manifold_rounds, r.counters, r.error_bits)


def _request(i, scale=4):
    s = synth.serving_request_spec(i)
    w, h, d = (max(6, x // scale) for x in (s["w"], s["h"], s["d"]))
    return synth.make_field(w, h, d, n_gauss=max(8, s["n_gauss"] // 8), seed=s["seed"],
                            rel=s["rel"], dtype=s["dtype"])


def test_result_alone_equals_in_mix():
    import torch
    from extrem_z_b200 import api
    probe = synth.make_field(40, 36, 24, n_gauss=24, seed=77, rel=1e-3, dtype=np.float64)
    ref, rrep = _plain(probe)
    with api.Server(0) as srv:
        # Alone.
        tf, tg = _dev(probe)
        t = srv.submit(tf, tg, probe.eb, **KW)
        rep_alone, lat = srv.wait(t)
        alone = tg.cpu().numpy()
        assert lat > 0
        # In a mix: requests arrive staggered, the probe among them.
        mix = [_request(i) for i in range(16)]
        tickets, bufs = [], []
        for i, fld in enumerate(mix):
            if i == 7:
                pf, pg = _dev(probe)
                tickets.append(srv.submit(pf, pg, probe.eb, **KW))
                bufs.append((probe, pg))
            a, b = _dev(fld)
            tickets.append(srv.submit(a, b, fld.eb, **KW))
            bufs.append((fld, b))
            time.sleep(0.002)
        results = [srv.wait(t) for t in tickets]
        stats = srv.stats()
    torch.cuda.synchronize()
    assert np.array_equal(alone.view(np.uint8), ref.view(np.uint8))
    assert _key(rep_alone) == _key(rrep)
    for (fld, buf), (rep, lat) in zip(bufs, results):
        out = buf.cpu().numpy()
        pref, prep = _plain(fld)
        assert np.array_equal(out.view(np.uint8), pref.view(np.uint8))
        assert _key(rep) == _key(prep)
        assert lat > 0
    assert stats["completed"] == stats["submitted"] == len(tickets) + 1
    assert stats["bytes_in_use"] == 0 and stats["running"] == 0 and stats["queued"] == 0
    # Requests overlapped on the device.
    assert stats["peak_running"] >= 2


def test_admission_respects_budget():
    from extrem_z_b200 import api
    fields = [synth.make_field(24, 20, 16, n_gauss=8, seed=900 + i, rel=3e-3,
                               dtype=np.float32 if i % 2 else np.float64) for i in range(10)]
    # Footprint of the largest request x 2.5: at most two in flight at once.
    n = 24 * 20 * 16
    budget = int(2.5 * (api.job_footprint(n, np.float64)))
    with api.Server(0, hbm_budget_bytes=budget) as srv:
        bufs, tickets = [], []
        for fld in fields:
            a, b = _dev(fld)
            tickets.append(srv.submit(a, b, fld.eb, **KW))
            bufs.append((fld, b))
        results = [srv.wait(t) for t in tickets]
        stats = srv.stats()
    assert stats["peak_bytes_in_use"] <= budget
    assert 1 <= stats["peak_running"] <= 2
    for (fld, buf), (rep, _) in zip(bufs, results):
        pref, prep = _plain(fld)
        assert np.array_equal(buf.cpu().numpy().view(np.uint8), pref.view(np.uint8))
        assert _key(rep) == _key(prep)


def test_request_beyond_budget_rejected():
    from extrem_z_b200 import api
    fld = synth.make_field(16, 16, 16, n_gauss=8, seed=5, rel=1e-2, dtype=np.float32)
    with api.Server(0, hbm_budget_bytes=1 << 20) as srv:
        a, b = _dev(fld)
        with pytest.raises(api.ExtremzError) as e:
            srv.submit(a, b, fld.eb, **KW)
        assert e.value.status == api.TOO_LARGE


def test_server_round_cap_reported():
    from extrem_z_b200 import api
    fld = synth.plain_64(np.float32)
    with api.Server(0) as srv:
        a, b = _dev(fld)
        rep, _ = srv.wait(srv.submit(a, b, fld.eb, **dict(KW, max_outer=0)))
    assert rep.status == api.ROUND_CAP
