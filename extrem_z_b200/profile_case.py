"""One correction of a named workload, for running under a profiler.

    python -m extrem_z_b200.profile_case [plain256_f64|plain256_f32|plain64_f32|plain512_f64]

Generates the workload's seeded field, copies both fields to cuda:0 and
corrects once through ``api.Context.correct_device``; prints the report.
"""

from __future__ import annotations

import sys

import numpy as np

from . import api, synth

CASES = {
    "plain256_f64": lambda: synth.plain_256(np.float64),
    "plain256_f32": lambda: synth.plain_256(np.float32),
    "plain64_f32": lambda: synth.plain_64(np.float32),
    "plain512_f64": synth.plain_512,
}


def main(argv=None) -> int:
    import torch
    argv = sys.argv[1:] if argv is None else argv
    name = argv[0] if argv else "plain256_f64"
    fld = CASES[name]()
    f = torch.from_numpy(fld.f).cuda()
    g = torch.from_numpy(fld.decp).cuda()
    ctx = api.Context(0)
    rep, _ = ctx.correct_device(f, g, fld.eb)
    torch.cuda.synchronize()
    print(f"{name}: status {rep.status} outer {rep.outer_iters} manifold rounds "
          f"{rep.manifold_rounds} (reused {rep.manifold_reused}) critical points {rep.cp_counts}")
    ctx.close()
    return 0 if rep.status == 0 else 1


if __name__ == "__main__":
    raise SystemExit(main())
