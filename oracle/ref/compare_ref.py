"""Compare the reference GPU correction with the oracle and the CUDA path.

Test infrastructure: runs oracle/_ref/ref_gpu (built from the reference's own
src/ExtreM_cuda.cu by build_ref.sh) several times per case, the oracle once,
and the library once, on seeded float64 fields, and prints a markdown table:
whether the reference's runs agree with one another, how many voxels the
reference's result differs from the oracle's in, and whether the library's
result equals the oracle's byte for byte.

    python oracle/ref/compare_ref.py [--runs 3] [--timing]
"""

from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from extrem_z_b200 import synth  # noqa: E402
from oracle import ffi  # noqa: E402
sys.path.insert(0, HERE)
import run_ref  # noqa: E402

CASES = [
    ("plain64 (64^3, G=64, seed 0, rel 1e-3)", lambda: synth.plain_64(np.float64)),
    ("32^3, G=16, seed 11, rel 1e-3", lambda: synth.make_field(32, 32, 32, n_gauss=16, seed=11,
                                                                rel=1e-3)),
    ("48x40x24, G=24, seed 12, rel 3e-3", lambda: synth.make_field(48, 40, 24, n_gauss=24,
                                                                    seed=12, rel=3e-3)),
    ("96^3, G=128, seed 13, rel 1e-4", lambda: synth.make_field(96, 96, 96, n_gauss=128,
                                                                 seed=13, rel=1e-4)),
    ("128x128 slice, G=32, seed 14, rel 1e-3", lambda: synth.make_field(128, 128, 1,
                                                                         n_gauss=32, seed=14,
                                                                         rel=1e-3)),
    ("64^3, G=64, seed 15, rel 1e-2", lambda: synth.make_field(64, 64, 64, n_gauss=64,
                                                                seed=15, rel=1e-2)),
]


def timing():
    """The reference's own timer ("whole time", src/ExtreM_cuda.cu:5020-6000: from
    after getdata to after the final saddle_loops_join, its allocations
    included) beside the library's device time on the 256^3 float64 field."""
    import re
    import torch
    from extrem_z_b200 import api
    fld = synth.plain_256(np.float64)
    _, stdout, wall = run_ref.run(fld.f, fld.decp, fld.rel, ffi.lut(), q=4, edit_type=1,
                                  timeout=900)
    m = re.search(r"whole time:([0-9.eE+-]+)", stdout)
    ref_s = float(m.group(1)) if m else float("nan")
    ctx = api.Context(0)
    f = torch.from_numpy(fld.f).cuda()
    g0 = torch.from_numpy(fld.decp).cuda()
    best = None
    for _ in range(4):
        g = g0.clone()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ctx.correct_device(f, g, fld.eb, q=4, edit_type=1)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    print(f"| 256^3 float64 | reference GPU {ref_s * 1e3:.1f} ms (own timer; process wall "
          f"{wall:.2f} s) | library {best:.2f} ms | {ref_s * 1e3 / best:.0f}x |")
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--runs", type=int, default=3)
    ap.add_argument("--timing", action="store_true",
                    help="time the reference binary and the library on the 256^3 field")
    args = ap.parse_args()
    if not run_ref.available():
        print("reference binary absent (oracle/_ref/ref_gpu)")
        return 1
    if args.timing:
        return timing()
    import torch
    from extrem_z_b200 import api
    lut = ffi.lut()
    print("| case | reference runs agree | voxels ref != oracle | max abs diff | "
          "library == oracle | oracle outer iters |")
    print("|---|---|---:|---:|---|---:|")
    for name, mk in CASES:
        fld = mk()
        rel = fld.rel
        outs = [run_ref.run(fld.f, fld.decp, rel, lut, q=4, edit_type=1)[0]
                for _ in range(args.runs)]
        agree = all(np.array_equal(outs[0].view(np.uint8), o.view(np.uint8)) for o in outs[1:])
        ref, rep, _ = ffi.correct(fld.f, fld.decp, fld.eb, q=4, edit_type=1)
        ndiff = [int(np.count_nonzero(o != ref)) for o in outs]
        mdiff = max(float(np.max(np.abs(o - ref))) for o in outs)
        tf = torch.from_numpy(fld.f).cuda()
        tg = torch.from_numpy(fld.decp.copy()).cuda()
        api.context(0).correct_device(tf, tg, fld.eb, q=4, edit_type=1)
        torch.cuda.synchronize()
        same = np.array_equal(tg.cpu().numpy().view(np.uint8), ref.view(np.uint8))
        print(f"| {name} | {'yes' if agree else 'no'} | {', '.join(map(str, ndiff))} | "
              f"{mdiff:.3g} | {'yes' if same else 'no'} | {rep['outer_iters']} |", flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
