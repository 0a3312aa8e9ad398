"""ctypes binding of the CPU oracle (test infrastructure only).

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this module; the product path never imports it.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

PHASES = {1: "cloop_detect", 2: "wrong_nbr", 3: "s_loops", 4: "saddle_loops",
          5: "detect3", 6: "s_loops_join", 7: "saddle_loops_join", 8: "outer",
          9: "checksum"}


class Params(ctypes.Structure):
    _fields_ = [("bound", ctypes.c_double), ("thr", ctypes.c_double),
                ("q", ctypes.c_int), ("edit_type", ctypes.c_int),
                ("max_outer", ctypes.c_int), ("max_cloop_rounds", ctypes.c_int),
                ("final_join", ctypes.c_int), ("preserve_join", ctypes.c_int),
                ("wn_lag", ctypes.c_int)]


class Report(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("outer_iters", ctypes.c_int),
                ("cloop_rounds", ctypes.c_int), ("manifold_rounds", ctypes.c_int),
                ("edited", ctypes.c_longlong), ("counters", ctypes.c_int * 11)]


class EditReport(ctypes.Structure):
    _fields_ = [("index_bytes", ctypes.c_longlong), ("edit_bytes", ctypes.c_longlong),
                ("edited", ctypes.c_longlong), ("n_edits", ctypes.c_longlong),
                ("psnr_before", ctypes.c_double), ("psnr_after", ctypes.c_double)]


def build(force: bool = False) -> str:
    """Compile liboracle.so with the Makefile next to this file."""
    src = os.path.join(_HERE, "extremz_oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or \
            os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-C", _HERE, "liboracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        vp, i32 = ctypes.c_void_p, ctypes.c_int
        L.oracle_set_threads.argtypes = [i32]
        L.oracle_set_threads.restype = i32
        L.oracle_lut.argtypes = [vp, i32]
        L.oracle_classify.argtypes = [vp, i32, i32, i32, i32, vp, vp]
        L.oracle_roots.argtypes = [vp, i32, i32, i32, i32, vp, vp]
        L.oracle_correct.argtypes = [vp, vp, i32, i32, i32, i32,
                                     ctypes.POINTER(Params), ctypes.POINTER(Report), vp, i32, vp]
        L.oracle_persistence_pairs.argtypes = [vp, i32, i32, i32, i32, vp, ctypes.c_longlong,
                                               vp, ctypes.c_longlong,
                                               ctypes.POINTER(ctypes.c_longlong),
                                               ctypes.POINTER(ctypes.c_longlong)]
        L.oracle_persistence_tree.argtypes = [vp, i32, i32, i32, i32, vp, ctypes.c_longlong,
                                              vp, ctypes.c_longlong, vp, vp,
                                              ctypes.POINTER(ctypes.c_longlong),
                                              ctypes.POINTER(ctypes.c_longlong)]
        L.oracle_census.argtypes = [vp, vp, i32, i32, i32, i32, ctypes.c_double, i32, vp]
        L.oracle_encode.argtypes = [vp, vp, vp, vp, i32, ctypes.c_longlong, ctypes.c_double,
                                    i32, i32, vp, ctypes.c_longlong, vp, ctypes.c_longlong,
                                    ctypes.POINTER(EditReport)]
        _lib = L
    return _lib


def set_threads(n: int) -> int:
    """Threads of the oracle's dense passes (results do not depend on it)."""
    return lib().oracle_set_threads(int(n))


def _dtype_code(a: np.ndarray) -> int:
    if a.dtype == np.float32:
        return 0
    if a.dtype == np.float64:
        return 1
    raise TypeError(f"unsupported dtype {a.dtype}")


def _dims(a: np.ndarray):
    if a.ndim == 2:
        return a.shape[1], a.shape[0], 1
    d, h, w = a.shape
    return w, h, d


def lut() -> np.ndarray:
    out = np.zeros(24800, dtype=np.int32)
    n = lib().oracle_lut(out.ctypes.data, out.size)
    assert n == 24800
    return out


def classify(f: np.ndarray):
    f = np.ascontiguousarray(f)
    w, h, d = _dims(f)
    t = np.zeros(f.size, dtype=np.int8)
    m = np.zeros(f.size, dtype=np.uint16)
    rc = lib().oracle_classify(f.ctypes.data, _dtype_code(f), w, h, d, t.ctypes.data, m.ctypes.data)
    assert rc == 0
    return t, m


def roots(f: np.ndarray):
    f = np.ascontiguousarray(f)
    w, h, d = _dims(f)
    ds = np.zeros(f.size, dtype=np.int32)
    a_s = np.zeros(f.size, dtype=np.int32)
    rc = lib().oracle_roots(f.ctypes.data, _dtype_code(f), w, h, d, ds.ctypes.data, a_s.ctypes.data)
    assert rc == 0
    return ds, a_s


def correct(f: np.ndarray, decp: np.ndarray, bound: float, *, thr: float = 0.0, q: int = 4,
            edit_type: int = 1, max_outer: int = 500, max_cloop_rounds: int = 100000,
            final_join: bool = True, preserve_join: bool = False, trace_cap: int = 0,
            counter_out: np.ndarray = None, wn_order: str = "lockstep", wn_lag: int = None):
    """Run the oracle correction; returns (corrected copy, report dict, trace).

    counter_out (optional, int32 of the field's size) receives the final edit
    counters (the reference's delta_counter).  wn_order: the resolution of the
    reference's wrong-neighbour race, "lockstep" (default) or "ascending";
    wn_lag (>= 0) selects the lockstep model with that visibility lag."""
    f = np.ascontiguousarray(f)
    out = np.ascontiguousarray(decp).copy()
    assert f.dtype == out.dtype and f.shape == out.shape
    w, h, d = _dims(f)
    p = Params(bound, thr, q, edit_type, max_outer, max_cloop_rounds,
               int(final_join), int(preserve_join),
               int(WN_ORDERS[wn_order] if wn_lag is None else wn_lag))
    r = Report()
    tr = np.zeros(max(trace_cap, 1) * 4, dtype=np.int32)
    rc = lib().oracle_correct(f.ctypes.data, out.ctypes.data, _dtype_code(f), w, h, d,
                              ctypes.byref(p), ctypes.byref(r), tr.ctypes.data, trace_cap * 4,
                              counter_out.ctypes.data if counter_out is not None else None)
    if rc < 0:
        raise ValueError("oracle rejected the arguments")
    rep = dict(status=r.status, outer_iters=r.outer_iters, cloop_rounds=r.cloop_rounds,
               manifold_rounds=r.manifold_rounds, edited=int(r.edited),
               counters=list(r.counters))
    trace = tr.reshape(-1, 4)
    if trace_cap:
        trace = trace[trace[:, 0] != 0]
    return out, rep, trace


COUNTER_NAMES = ("wrong_split_nbrs", "wrong_join_nbrs", "false_max", "false_min", "false_saddle",
                 "wrong_max", "wrong_max_2", "wrong_saddle", "wrong_min", "wrong_min_2",
                 "wrong_saddle_join")


WN_ORDERS = {"lockstep": 0, "ascending": -1}


def census(f: np.ndarray, decp: np.ndarray, *, thr: float = 0.0, wn_order: str = "lockstep"):
    """Mismatch census of decp against f: the eleven loop-test counters
    (order of ``Report.counters``) evaluated once, no edit."""
    f = np.ascontiguousarray(f)
    g = np.ascontiguousarray(decp)
    assert f.dtype == g.dtype and f.shape == g.shape
    w, h, d = _dims(f)
    out = np.zeros(11, dtype=np.int32)
    rc = lib().oracle_census(f.ctypes.data, g.ctypes.data, _dtype_code(f), w, h, d, float(thr),
                             WN_ORDERS[wn_order], out.ctypes.data)
    if rc != 0:
        raise ValueError(f"oracle_census returned {rc}")
    return [int(x) for x in out]


def encode(f: np.ndarray, decp0: np.ndarray, fixed: np.ndarray, counter, bound: float, *,
           q: int = 4, edit_type: int = 1):
    """Edit stream of a correction: (index stream bytes, edits array, report dict)."""
    f = np.ascontiguousarray(f)
    d0 = np.ascontiguousarray(decp0)
    d1 = np.ascontiguousarray(fixed)
    assert f.dtype == d0.dtype == d1.dtype and f.shape == d0.shape == d1.shape
    n = f.size
    cnt = None if counter is None else np.ascontiguousarray(counter, dtype=np.int32)
    index = np.zeros(max(4 * n, (3 * n + 7) // 8), dtype=np.uint8)
    edits = np.zeros(n, dtype=f.dtype)
    r = EditReport()
    rc = lib().oracle_encode(f.ctypes.data, d0.ctypes.data, d1.ctypes.data,
                             cnt.ctypes.data if cnt is not None else None, _dtype_code(f), n,
                             float(bound), int(q), int(edit_type), index.ctypes.data, index.size,
                             edits.ctypes.data, edits.nbytes, ctypes.byref(r))
    if rc != 0:
        raise ValueError(f"oracle_encode returned {rc}")
    rep = dict(index_bytes=r.index_bytes, edit_bytes=r.edit_bytes, edited=r.edited,
               n_edits=r.n_edits, psnr_before=r.psnr_before, psnr_after=r.psnr_after)
    return index[:r.index_bytes].copy(), edits[:r.n_edits].copy(), rep


def persistence_pairs(f: np.ndarray):
    """Elder-rule persistence pairs: (max pairs (n, 2), min pairs (m, 2)) of
    (partner vertex, extremum vertex), extrema by rank."""
    f = np.ascontiguousarray(f)
    w, h, d = _dims(f)
    cap = 2 * f.size
    mx = np.zeros(cap, np.int32)
    mn = np.zeros(cap, np.int32)
    nx, nn = ctypes.c_longlong(), ctypes.c_longlong()
    rc = lib().oracle_persistence_pairs(f.ctypes.data, _dtype_code(f), w, h, d, mx.ctypes.data,
                                        cap, mn.ctypes.data, cap, ctypes.byref(nx),
                                        ctypes.byref(nn))
    if rc != 0:
        raise ValueError(f"oracle_persistence_pairs returned {rc}")
    return mx[:2 * nx.value].reshape(-1, 2), mn[:2 * nn.value].reshape(-1, 2)


def persistence_tree(f: np.ndarray):
    """Elder-rule pairs and branch parents: (max pairs (n, 2), min pairs (m, 2),
    max parents (n,), min parents (m,)); a parent is the extremum whose branch
    the extremum joins at its partner vertex (the global extremum its own)."""
    f = np.ascontiguousarray(f)
    w, h, d = _dims(f)
    cap = 2 * f.size
    mx, mn = np.zeros(cap, np.int32), np.zeros(cap, np.int32)
    px, pn = np.zeros(f.size, np.int32), np.zeros(f.size, np.int32)
    nx, nn = ctypes.c_longlong(), ctypes.c_longlong()
    rc = lib().oracle_persistence_tree(f.ctypes.data, _dtype_code(f), w, h, d, mx.ctypes.data,
                                       cap, mn.ctypes.data, cap, px.ctypes.data, pn.ctypes.data,
                                       ctypes.byref(nx), ctypes.byref(nn))
    if rc != 0:
        raise ValueError(f"oracle_persistence_tree returned {rc}")
    return (mx[:2 * nx.value].reshape(-1, 2), mn[:2 * nn.value].reshape(-1, 2),
            px[:nx.value].copy(), pn[:nn.value].copy())
