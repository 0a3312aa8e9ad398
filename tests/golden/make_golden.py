"""Regenerate the golden fixtures of tests/golden/.

* lut_digest.json -- SHA-256, size and value histogram of the reference's
  src/LUT.bin (the critical-point lookup table it ships).  Read from the
  reference checkout; run where it is mounted:
      python tests/golden/make_golden.py --reference /path/to/ExtreM_z
* oracle_cases.npz -- small seeded inputs and the oracle's corrected outputs,
  reports and traces, pinning the oracle's behaviour across changes.
* encode_cases.npz -- int32 inputs and the outputs of the reference's own
  encodeTo3BitBitmap and get_diff_index (src/ExtreM_cuda.cu:4282-4323), run
  through the reference harness binary oracle/_ref/ref_gpu (built from the
  reference's source by oracle/ref/build_ref.sh; these modes use no GPU):
      python tests/golden/make_golden.py --encode
"""

import argparse
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from extrem_z_b200 import synth  # noqa: E402
from oracle import ffi  # noqa: E402

# (name, w, h, d, gaussians, seed, rel, dtype, edit_type)
CASES = [
    ("cube16_f64_e1", 16, 16, 16, 8, 0, 1e-3, np.float64, 1),
    ("cube16_f64_e0", 16, 16, 16, 8, 0, 1e-3, np.float64, 0),
    ("box_f32_e1", 24, 18, 12, 12, 5, 2e-3, np.float32, 1),
    ("box_f32_e0", 24, 18, 12, 12, 5, 2e-3, np.float32, 0),
    ("thin_f64_e1", 40, 3, 9, 6, 11, 1e-3, np.float64, 1),
    ("slice_f64_e1", 48, 40, 1, 8, 3, 1e-3, np.float64, 1),
    ("tiny_f32_e1", 3, 3, 3, 2, 7, 5e-2, np.float32, 1),
    ("line_f64_e1", 1, 30, 2, 3, 9, 1e-2, np.float64, 1),
]
ORACLE_KW = dict(q=4, max_outer=500, max_cloop_rounds=100000, final_join=True)


def lut_digest(reference: str):
    ref = np.fromfile(os.path.join(reference, "src", "LUT.bin"), dtype="<i4")
    vals, counts = np.unique(ref, return_counts=True)
    return {"sha256": hashlib.sha256(ref.tobytes()).hexdigest(), "entries": int(ref.size),
            "histogram": {str(int(v)): int(c) for v, c in zip(vals, counts)},
            "source": "src/LUT.bin of the reference"}


def oracle_cases():
    out = {}
    for name, w, h, d, g, seed, rel, dt, et in CASES:
        fld = synth.make_field(w, h, d, n_gauss=g, seed=seed, rel=rel, dtype=dt)
        fixed, rep, trace = ffi.correct(fld.f, fld.decp, fld.eb, edit_type=et, trace_cap=200000,
                                        **ORACLE_KW)
        out[f"{name}/f"] = fld.f
        out[f"{name}/decp"] = fld.decp
        out[f"{name}/fixed"] = fixed
        out[f"{name}/meta"] = np.array([fld.eb, et, rep["status"], rep["outer_iters"],
                                        rep["cloop_rounds"], rep["manifold_rounds"]],
                                       dtype=np.float64)
        out[f"{name}/trace"] = trace
    return out


def encode_cases():
    import subprocess
    import tempfile
    binary = os.path.join(ROOT, "oracle", "_ref", "ref_gpu")
    rng = np.random.default_rng(2024)
    out = {}
    lengths = [1, 2, 3, 7, 8, 9, 16, 24, 100, 1001]
    with tempfile.TemporaryDirectory() as tmp:
        src, dst = os.path.join(tmp, "in.i32"), os.path.join(tmp, "out.bin")
        for n in lengths:
            v = rng.integers(0, 8, size=n).astype("<i4")
            v.tofile(src)
            subprocess.run([binary, "--encode3", src, dst], check=True)
            out[f"pack3/{n}/in"] = v
            out[f"pack3/{n}/out"] = np.fromfile(dst, dtype=np.uint8)
            ids = np.sort(rng.choice(10 * n + 5, size=n, replace=False)).astype("<i4")
            ids.tofile(src)
            subprocess.run([binary, "--diff", src, dst], check=True)
            out[f"diff/{n}/in"] = ids
            out[f"diff/{n}/out"] = np.fromfile(dst, dtype="<i4")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None, help="reference checkout (for LUT.bin)")
    ap.add_argument("--encode", action="store_true",
                    help="only regenerate encode_cases.npz from the reference harness binary")
    args = ap.parse_args()
    if args.encode:
        np.savez_compressed(os.path.join(HERE, "encode_cases.npz"), **encode_cases())
        return
    if args.reference:
        with open(os.path.join(HERE, "lut_digest.json"), "w") as fh:
            json.dump(lut_digest(args.reference), fh, indent=1)
            fh.write("\n")
    np.savez_compressed(os.path.join(HERE, "oracle_cases.npz"), **oracle_cases())


if __name__ == "__main__":
    main()
