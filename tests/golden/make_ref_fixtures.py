"""Outputs of the reference's own GPU correction, for pinning the oracle.

Runs oracle/_ref/ref_gpu -- the reference's src/ExtreM_cuda.cu compiled
unmodified by oracle/ref/build_ref.sh -- several times per seeded float64
field (q 4, sim 0) and records:
  * ref_gpu_cases.json: per case the generator parameters, the SHA-256 of each
    run's corrected field and whether the runs agree with one another;
  * ref_gpu_edits.npz: for the small cases, the first run's corrected field as
    (ids, values) of the voxels that differ from the decompressed field.
Needs a GPU and the reference binary; writes into --out (a scratch folder
whose files are then copied next to this script).

    python tests/golden/make_ref_fixtures.py --out <dir> [--only NAME ...]
"""

from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle", "ref"))

from extrem_z_b200 import synth  # noqa: E402
from oracle import ffi  # noqa: E402
import run_ref  # noqa: E402

# name -> (w, h, d, gaussians, seed, rel, edit_type, runs, keep edits); float64
# (the reference's GPU path is float64-only).
CASES = {
    "cube64_s0_e1": (64, 64, 64, 64, 0, 1e-3, 1, 3, True),
    "cube32_s11_e1": (32, 32, 32, 16, 11, 1e-3, 1, 3, True),
    "box48x40x24_s12_e1": (48, 40, 24, 24, 12, 3e-3, 1, 3, True),
    "cube96_s13_e1": (96, 96, 96, 128, 13, 1e-4, 1, 3, True),
    "slice128_s14_e1": (128, 128, 1, 32, 14, 1e-3, 1, 3, True),
    "cube64_s15_e1": (64, 64, 64, 64, 15, 1e-2, 1, 3, True),
    "cube32_s11_e0": (32, 32, 32, 16, 11, 1e-3, 0, 3, True),
    "box40x36x28_s16_e0": (40, 36, 28, 20, 16, 2e-3, 0, 3, True),
    "cube48_s17_e1": (48, 48, 48, 32, 17, 5e-4, 1, 3, True),
    "slice200x150_s18_e1": (200, 150, 1, 40, 18, 5e-4, 1, 3, True),
    # The benchmark fields: only digests are kept (tests compare them with the
    # oracle's digests of the same fields).
    "plain256_f64": "plain256_f64",
    "plain512_f64": "plain512_f64",
}
RUNS_LARGE = {"plain256_f64": 2, "plain512_f64": 1}


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def make(name):
    spec = CASES[name]
    if spec == "plain256_f64":
        return synth.plain_256(np.float64), 1, RUNS_LARGE[name], False
    if spec == "plain512_f64":
        return synth.plain_512(), 1, RUNS_LARGE[name], False
    w, h, d, g, seed, rel, et, runs, keep = spec
    return synth.make_field(w, h, d, n_gauss=g, seed=seed, rel=rel), et, runs, keep


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--only", nargs="*", default=None)
    args = ap.parse_args()
    if not run_ref.available():
        print("reference binary absent (oracle/_ref/ref_gpu)")
        return 1
    os.makedirs(args.out, exist_ok=True)
    lut = ffi.lut()
    meta, edits = {}, {}
    for name in CASES:
        if args.only and name not in args.only:
            continue
        fld, et, runs, keep = make(name)
        entry = {"edit_type": et, "q": 4, "sim": 0.0, "shape_whd": list(fld.shape_whd),
                 "rel": fld.rel, "seed": fld.seed, "run_sha256": [], "run_seconds": []}
        if isinstance(CASES[name], tuple):
            entry["gaussians"] = CASES[name][3]
        first = None
        for _ in range(runs):
            t0 = time.perf_counter()
            out, _, _ = run_ref.run(fld.f, fld.decp, fld.rel, lut, q=4, edit_type=et,
                                    timeout=1800 if fld.f.size > 1e7 else 300)
            entry["run_seconds"].append(round(time.perf_counter() - t0, 2))
            entry["run_sha256"].append(sha(out))
            if first is None:
                first = out
        entry["runs_agree"] = len(set(entry["run_sha256"])) == 1
        if keep:
            ids = np.flatnonzero(first.view(np.uint64) != fld.decp.view(np.uint64)).astype(np.int32)
            edits[f"{name}/ids"] = ids
            edits[f"{name}/values"] = first.reshape(-1)[ids]
        meta[name] = entry
        print(name, entry, flush=True)
        with open(os.path.join(args.out, "ref_gpu_cases.json"), "w") as fh:
            json.dump(meta, fh, indent=1, sort_keys=True)
            fh.write("\n")
        np.savez_compressed(os.path.join(args.out, "ref_gpu_edits.npz"), **edits)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
