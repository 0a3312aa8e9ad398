"""The benchmark configurations, byte for byte against the oracle.

tests/golden/config_hashes.json holds, per benchmark field (64^3 float32,
256^3 float64 and float32, 512^3 float64, the 64 fields of the mixed batch)
and with the final join-saddle pass on and off, the SHA-256 of the oracle's
corrected field and of its per-phase trace, its report and the mismatch
census of its corrected field (made by tests/golden/make_config_hashes.py on
the CPU).  Here the same seeded fields are corrected through the library --
the plain device entry point and the batched one -- and every digest must
match: bit-exact, the tolerance of all parity tests here.
"""

import hashlib
import json
import os

import numpy as np
import pytest

from extrem_z_b200 import synth

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "config_hashes.json")) as _fh:
    DIGESTS = json.load(_fh)

PLAIN = {
    "plain64_f32": lambda: synth.plain_64(np.float32),
    "plain256_f64": lambda: synth.plain_256(np.float64),
    "plain256_f32": lambda: synth.plain_256(np.float32),
    "plain512_f64": lambda: synth.plain_512(),
}
PLAIN_CASES = [(n, fj) for n in PLAIN if n in DIGESTS for fj in (1, 0)]


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def check(entry, fixed_sha, rep, census, trace_sha=None):
    assert fixed_sha == entry["fixed_sha256"]
    if trace_sha is not None:
        assert trace_sha == entry["trace_sha256"]
    assert rep.status == entry["status"]
    assert rep.outer_iters == entry["outer_iters"]
    assert rep.counters == entry["counters"]
    assert census == entry["census"]


_fields = {}


def field(name):
    if name not in _fields:
        _fields.clear()  # one large field in memory at a time
        _fields[name] = PLAIN[name]()
    return _fields[name]


@pytest.mark.parametrize("name,final_join", PLAIN_CASES)
def test_plain_config_matches_oracle_digest(name, final_join):
    import torch
    from extrem_z_b200 import api
    fld = field(name)
    entry = DIGESTS[name][f"final_join_{final_join}"]
    params = dict(DIGESTS[name]["params"])
    f = torch.from_numpy(fld.f).cuda()
    g = torch.from_numpy(fld.decp).cuda()
    ctx = api.context(0)
    rep, trace = ctx.correct_device(f, g, fld.eb, trace_cap=1 << 16, final_join=bool(final_join),
                                    **params)
    census = ctx.mismatch_census(f, g)["counters"]
    out_sha = sha(g.cpu().numpy())
    check(entry, out_sha, rep, census, sha(trace.astype(np.int32)))
    del f, g
    torch.cuda.empty_cache()


@pytest.mark.skipif("mixed64" not in DIGESTS, reason="no mixed-batch digests")
@pytest.mark.parametrize("final_join", [1, 0])
def test_mixed_batch_matches_oracle_digests(final_join):
    """All 64 fields of the mixed batch in one extremz_correct_batch call."""
    import torch
    from extrem_z_b200 import api
    entries = DIGESTS["mixed64"]["fields"]
    params = dict(DIGESTS["mixed64"]["params"], final_join=bool(final_join))
    specs = synth.mixed_batch_specs(64)
    assert [s["seed"] for s in specs] == [e["seed"] for e in entries]
    fields = [synth.make_field(s["w"], s["h"], s["d"], n_gauss=s["n_gauss"], seed=s["seed"],
                               rel=s["rel"], dtype=s["dtype"]) for s in specs]
    F = [torch.from_numpy(x.f).cuda() for x in fields]
    G = [torch.from_numpy(x.decp).cuda() for x in fields]
    ctx = api.context(0)
    reps, _ = ctx.correct_batch([(f, g, x.eb, params) for f, g, x in zip(F, G, fields)])
    torch.cuda.synchronize()
    for f, g, rep, e in zip(F, G, reps, entries):
        d = e[f"final_join_{final_join}"]
        census = ctx.mismatch_census(f, g)["counters"]
        check(d, sha(g.cpu().numpy()), rep, census)


with open(os.path.join(HERE, "golden", "ref_gpu_cases.json")) as _fh:
    REF_RUNS = json.load(_fh)


@pytest.mark.parametrize("name,order", [("plain256_f64", "lockstep"), ("plain512_f64", "lockstep"),
                                        ("plain512_f64", "ascending")])
def test_benchmark_fields_equal_the_reference_gpu_output(name, order):
    """The reference's own GPU correction of the 256^3 and 512^3 float64
    benchmark fields (its runs agree with one another): the library's output
    is byte-identical to it with the default (lockstep) resolution of the
    wrong-neighbour race, and at 512^3 with the ascending one as well."""
    import torch
    from extrem_z_b200 import api
    fld = field(name)
    runs = REF_RUNS[name]["run_sha256"]
    assert REF_RUNS[name]["runs_agree"]
    f = torch.from_numpy(fld.f).cuda()
    g = torch.from_numpy(fld.decp).cuda()
    rep, _ = api.context(0).correct_device(f, g, fld.eb, q=4, edit_type=1, max_outer=1000,
                                           final_join=True, wn_order=order)
    assert rep.status == 0
    assert sha(g.cpu().numpy()) == runs[0]
    del f, g
    torch.cuda.empty_cache()
