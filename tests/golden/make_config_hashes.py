"""Oracle digests of the benchmark configurations (tests/golden/config_hashes.json).

The benchmark fields are too large to commit and too slow for the oracle to
correct inside a GPU test run (a 512^3 float64 field takes the OpenMP oracle
minutes), so this script corrects them once on the CPU and commits, per
case, the SHA-256 of the corrected field's bytes, the SHA-256 of the
oracle's per-phase trace, the report, and the mismatch census of the
corrected field.  The GPU tests regenerate the same seeded fields, correct
them through the library and compare digests.

    python tests/golden/make_config_hashes.py [--only NAME ...] [--threads N]

Cases (both with and without the final join-saddle pass, q 4, edit_type 1):
  plain64_f32   64^3 float32, 64 Gaussians, seed 0, eb 1e-3 rel
  plain256_f64  256^3 float64, 512 Gaussians, seed 1, eb 1e-4 rel
  plain256_f32  the same field in float32
  plain512_f64  512^3 float64, 4096 Gaussians + k^-5/3 noise, seed 2, eb 1e-5 rel
  mixed64       the 64 fields of the mixed batch (seeds 100-163), one digest each
The wrong-neighbour race of the reference is resolved in the default
(lockstep) order.  Existing entries of the JSON file are kept unless
recomputed.  --ascending adds, for the named fields, the digest of the
correction with the race resolved in ascending saddle order (entry
ascending_final_join_1).
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

from extrem_z_b200 import synth  # noqa: E402
from oracle import ffi  # noqa: E402

OUT = os.path.join(HERE, "config_hashes.json")
PARAMS = dict(q=4, edit_type=1, thr=0.0, max_outer=1000, max_cloop_rounds=100000)
TRACE_CAP = 1 << 16

PLAIN = {
    "plain64_f32": lambda: synth.plain_64(np.float32),
    "plain256_f64": lambda: synth.plain_256(np.float64),
    "plain256_f32": lambda: synth.plain_256(np.float32),
    "plain512_f64": lambda: synth.plain_512(),
}


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def digest(fld, final_join: bool, trace: bool = True, wn_order: str = "lockstep"):
    t0 = time.perf_counter()
    fixed, rep, tr = ffi.correct(fld.f, fld.decp, fld.eb, final_join=final_join,
                                 trace_cap=TRACE_CAP if trace else 0, wn_order=wn_order,
                                 **PARAMS)
    secs = time.perf_counter() - t0
    out = {"fixed_sha256": sha(fixed), "status": rep["status"],
           "outer_iters": rep["outer_iters"], "cloop_rounds": rep["cloop_rounds"],
           "manifold_rounds": rep["manifold_rounds"], "edited": rep["edited"],
           "counters": rep["counters"], "census": ffi.census(fld.f, fixed, wn_order=wn_order),
           "oracle_seconds": round(secs, 2)}
    if trace:
        out["trace_sha256"] = sha(tr.astype(np.int32))
        out["trace_records"] = int(len(tr))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*", default=None)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--ascending", nargs="*", default=None)
    args = ap.parse_args()
    ffi.set_threads(args.threads)
    data = {}
    if os.path.exists(OUT):
        with open(OUT) as fh:
            data = json.load(fh)
    if args.ascending:
        for name in args.ascending:
            fld = PLAIN[name]()
            data[name]["ascending_final_join_1"] = digest(fld, True, wn_order="ascending")
            print(name, "ascending", data[name]["ascending_final_join_1"], flush=True)
            with open(OUT, "w") as fh:
                json.dump(data, fh, indent=1, sort_keys=True)
                fh.write("\n")
        return
    names = list(PLAIN) + ["mixed64"]
    for name in names:
        if args.only and name not in args.only:
            continue
        entry = dict(data.get(name, {}), params=PARAMS)  # other entries stay
        if name in PLAIN:
            fld = PLAIN[name]()
            entry["eb"] = fld.eb
            entry["shape_whd"] = list(fld.shape_whd)
            for fj in (True, False):
                entry[f"final_join_{int(fj)}"] = digest(fld, fj)
                print(name, fj, entry[f"final_join_{int(fj)}"], flush=True)
            del fld
        else:
            specs = synth.mixed_batch_specs(64)
            fields = []
            for s in specs:
                fld = synth.make_field(s["w"], s["h"], s["d"], n_gauss=s["n_gauss"],
                                       seed=s["seed"], rel=s["rel"], dtype=s["dtype"])
                fields.append({"seed": s["seed"], "shape_whd": [s["w"], s["h"], s["d"]],
                               "final_join_1": digest(fld, True, trace=False),
                               "final_join_0": digest(fld, False, trace=False)})
            entry["fields"] = fields
            print(name, "done", flush=True)
        data[name] = entry
        with open(OUT, "w") as fh:
            json.dump(data, fh, indent=1, sort_keys=True)
            fh.write("\n")


if __name__ == "__main__":
    main()
