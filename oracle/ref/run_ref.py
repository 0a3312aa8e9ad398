"""Run the reference GPU correction (oracle/_ref/ref_gpu) on one field.

Test infrastructure only.  The binary is built from the reference's own
src/ExtreM_cuda.cu by oracle/ref/build_ref.sh; it is float64-only, as the
reference is.  Returns the corrected field, the reference's stdout and the
wall time, or raises if the binary is absent.
"""

from __future__ import annotations

import os
import subprocess
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BINARY = os.path.join(os.path.dirname(HERE), "_ref", "ref_gpu")


def available() -> bool:
    return os.path.exists(BINARY)


def run(f: np.ndarray, decp: np.ndarray, rel: float, lut: np.ndarray, *, sim: float = 0.0,
        q: int = 4, edit_type: int = 1, timeout: float = 300.0):
    assert f.dtype == np.float64 and decp.dtype == np.float64 and f.shape == decp.shape
    d, h, w = f.shape if f.ndim == 3 else (1,) + f.shape
    with tempfile.TemporaryDirectory() as tmp:
        work = os.path.join(tmp, "run")
        os.makedirs(work)
        os.makedirs(os.path.join(tmp, "stat_result"))
        np.ascontiguousarray(f).tofile(os.path.join(work, "orig.f64"))
        np.ascontiguousarray(decp).tofile(os.path.join(work, "decp.f64"))
        lut.astype("<i4").tofile(os.path.join(work, "LUT.bin"))
        env = dict(os.environ, EXTREMZ_REF_DECP=os.path.join(work, "decp.f64"))
        args = [BINARY, "orig.f64", str(w), str(h), str(d), repr(float(rel)), repr(float(sim)),
                str(q), str(edit_type), "out.f64"]
        t0 = time.perf_counter()
        p = subprocess.run(args, cwd=work, env=env, timeout=timeout, capture_output=True,
                           text=True)
        wall = time.perf_counter() - t0
        if p.returncode != 0:
            raise RuntimeError(f"reference exited {p.returncode}: {p.stderr[-2000:]}")
        out = np.fromfile(os.path.join(work, "out.f64"), dtype=np.float64).reshape(f.shape)
    return out, p.stdout, wall
