"""Python host side of the ExtreM correction, over the C ABI of libextremz.so.

Mirrors the reference's correction call (src/ExtreM_cuda.cu main(), and the
host API include/api/ExtreM.h used by main.cpp): an original field, its
decompressed copy and the absolute bound go in; the decompressed copy comes
back corrected in place.  Status codes of the C ABI become exceptions, except
``EXTREMZ_ROUND_CAP``, which is reported in the returned report.

There is no CPU fallback: if the CUDA library is missing or no device is
present, these functions raise.
"""

from __future__ import annotations

import ctypes
import dataclasses
import os
import threading

import numpy as np

from . import build as _build

_lib = None
_lock = threading.Lock()

OK, ROUND_CAP, BAD_ARG, OOM, CUDA_ERR, DEVICE_TIMEOUT, NO_DEVICE, TOO_LARGE, PENDING = range(9)
# EXTREMZ_ABI_VERSION of include/extremz.h that the structures below follow.
ABI_VERSION = 2
F32, F64 = 0, 1

# Every entry point declared in include/extremz.h.
EXPORTS = ("extremz_version", "extremz_default_params", "extremz_ctx_create",
           "extremz_ctx_destroy", "extremz_correct_device", "extremz_mismatch_census",
           "extremz_correct_host",
           "extremz_correct_batch", "extremz_correct_encode", "extremz_edit_stream_caps",
           "extremz_zstd_size", "extremz_classify", "extremz_persistence_pairs",
           "extremz_persistence_tree",
           "extremz_server_create", "extremz_server_destroy",
           "extremz_server_submit", "extremz_server_poll", "extremz_server_wait",
           "extremz_server_get_stats", "extremz_job_footprint",
           "extremz_correct_device_noalloc", "extremz_noalloc_max_voxels",
           "extremz_lut", "extremz_status_string", "extremz_last_cuda_error")


class ExtremzError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"extremz status {status}: {msg}")
        self.status = status


class Params(ctypes.Structure):
    _fields_ = [("bound", ctypes.c_double), ("thr", ctypes.c_double),
                ("q", ctypes.c_int), ("edit_type", ctypes.c_int),
                ("max_outer", ctypes.c_int), ("max_cloop_rounds", ctypes.c_int),
                ("final_join", ctypes.c_int), ("preserve_join", ctypes.c_int),
                ("flags", ctypes.c_int), ("device_iter_cap", ctypes.c_int),
                ("tune_blocks_per_sm", ctypes.c_int), ("tune_pass_chunk", ctypes.c_int),
                ("reserved", ctypes.c_int * 2)]


class Report(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("outer_iters", ctypes.c_int),
                ("cloop_rounds", ctypes.c_int), ("manifold_rounds", ctypes.c_int),
                ("counters", ctypes.c_int * 11), ("error_bits", ctypes.c_int),
                ("kernel_launches", ctypes.c_longlong),
                ("prof_ms", ctypes.c_float * 12), ("prof_launches", ctypes.c_int * 12),
                ("manifold_reused", ctypes.c_int), ("cp_counts", ctypes.c_int * 4),
                ("graph_launches", ctypes.c_int), ("host_bytes_back", ctypes.c_longlong)]

class EditStream(ctypes.Structure):
    _fields_ = [("index", ctypes.c_void_p), ("index_cap", ctypes.c_longlong),
                ("edits", ctypes.c_void_p), ("edits_cap", ctypes.c_longlong),
                ("index_bytes", ctypes.c_longlong), ("edit_bytes", ctypes.c_longlong),
                ("edited", ctypes.c_longlong), ("n_edits", ctypes.c_longlong),
                ("psnr_before", ctypes.c_double), ("psnr_after", ctypes.c_double),
                ("reserved", ctypes.c_int * 4)]


class Field(ctypes.Structure):
    _fields_ = [("orig", ctypes.c_void_p), ("decp", ctypes.c_void_p), ("dtype", ctypes.c_int),
                ("width", ctypes.c_int), ("height", ctypes.c_int), ("depth", ctypes.c_int),
                ("params", Params)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_longlong), ("reserve_bytes", ctypes.c_longlong),
                ("split_voxels", ctypes.c_longlong), ("max_jobs", ctypes.c_int),
                ("reserved", ctypes.c_int * 7)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_longlong), ("completed", ctypes.c_longlong),
                ("queued", ctypes.c_longlong), ("running", ctypes.c_longlong),
                ("bytes_in_use", ctypes.c_longlong), ("peak_bytes_in_use", ctypes.c_longlong),
                ("ticks", ctypes.c_longlong), ("kernel_launches", ctypes.c_longlong),
                ("peak_running", ctypes.c_int), ("reserved", ctypes.c_int * 7)]


FLAG_PROFILE = 1
FLAG_NO_TMA = 2
FLAG_WN_ASCENDING = 4
PROFILE_CLASS_SHIFT = 8
KCLASS_NAMES = ("setup_classify", "classify_detect", "direction", "jump", "propose", "apply",
                "rows", "wrong_nbr", "fixpath", "other", "direction_first", "jump_first")


@dataclasses.dataclass
class CorrectionReport:
    status: int
    outer_iters: int
    cloop_rounds: int
    manifold_rounds: int
    counters: list
    error_bits: int
    kernel_launches: int = 0
    prof_ms: dict = None
    prof_launches: dict = None
    manifold_reused: int = 0
    cp_counts: list = None      # original 2-saddles, 1-saddles, maxima, minima
    graph_launches: int = 0     # ticks launched as one CUDA graph
    host_bytes_back: int = 0    # correct_host: bytes copied device -> host

    @staticmethod
    def of(r: Report) -> "CorrectionReport":
        return CorrectionReport(r.status, r.outer_iters, r.cloop_rounds, r.manifold_rounds,
                                list(r.counters), r.error_bits, int(r.kernel_launches),
                                dict(zip(KCLASS_NAMES, [float(x) for x in r.prof_ms])),
                                dict(zip(KCLASS_NAMES, [int(x) for x in r.prof_launches])),
                                int(r.manifold_reused), list(r.cp_counts),
                                int(r.graph_launches), int(r.host_bytes_back))


def library_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load libextremz.so (building it first if it is absent or stale)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = _build.LIB
        if build_if_missing and (not os.path.exists(path) or _build._stale()):
            try:
                _build.build()
            except Exception:
                if not os.path.exists(path):
                    raise
        if not os.path.exists(path):
            raise ExtremzError(NO_DEVICE, f"CUDA library missing: {path}")
        L = ctypes.CDLL(path)
        vp, i32 = ctypes.c_void_p, ctypes.c_int
        L.extremz_version.restype = i32
        if L.extremz_version() != ABI_VERSION:  # the report layout would not match
            raise ExtremzError(BAD_ARG, f"{path} has ABI version {L.extremz_version()}, "
                                        f"this binding {ABI_VERSION}: rebuild it")
        L.extremz_default_params.argtypes = [ctypes.POINTER(Params)]
        L.extremz_ctx_create.argtypes = [i32, ctypes.POINTER(vp)]
        L.extremz_ctx_create.restype = i32
        L.extremz_ctx_destroy.argtypes = [vp]
        L.extremz_correct_device.argtypes = [vp, vp, vp, i32, i32, i32, i32,
                                             ctypes.POINTER(Params), ctypes.POINTER(Report),
                                             vp, vp, i32]
        L.extremz_correct_device.restype = i32
        L.extremz_mismatch_census.argtypes = [vp, vp, vp, i32, i32, i32, i32, ctypes.c_double,
                                              vp, vp]
        L.extremz_mismatch_census.restype = i32
        L.extremz_classify.argtypes = [vp, vp, i32, i32, i32, i32, vp, vp, vp, vp]
        L.extremz_classify.restype = i32
        L.extremz_correct_host.argtypes = [vp, vp, vp, i32, i32, i32, i32,
                                           ctypes.POINTER(Params), ctypes.POINTER(Report), vp]
        L.extremz_correct_host.restype = i32
        L.extremz_correct_encode.argtypes = [vp, vp, vp, i32, i32, i32, i32,
                                             ctypes.POINTER(Params), ctypes.POINTER(Report), vp,
                                             ctypes.POINTER(EditStream)]
        L.extremz_correct_encode.restype = i32
        L.extremz_edit_stream_caps.argtypes = [i32, i32, i32, i32, i32,
                                               ctypes.POINTER(ctypes.c_longlong),
                                               ctypes.POINTER(ctypes.c_longlong)]
        L.extremz_edit_stream_caps.restype = i32
        L.extremz_persistence_pairs.argtypes = [vp, vp, i32, i32, i32, i32, vp,
                                                ctypes.c_longlong, vp, ctypes.c_longlong,
                                                ctypes.POINTER(ctypes.c_longlong),
                                                ctypes.POINTER(ctypes.c_longlong), vp]
        L.extremz_persistence_pairs.restype = i32
        L.extremz_persistence_tree.argtypes = [vp, vp, i32, i32, i32, i32, vp,
                                               ctypes.c_longlong, vp, ctypes.c_longlong, vp, vp,
                                               ctypes.POINTER(ctypes.c_longlong),
                                               ctypes.POINTER(ctypes.c_longlong), vp]
        L.extremz_persistence_tree.restype = i32
        L.extremz_zstd_size.argtypes = [vp, ctypes.c_longlong, i32]
        L.extremz_zstd_size.restype = ctypes.c_longlong
        L.extremz_correct_batch.argtypes = [vp, ctypes.POINTER(Field), i32,
                                            ctypes.POINTER(Report), vp]
        L.extremz_correct_batch.restype = i32
        L.extremz_server_create.argtypes = [i32, ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]
        L.extremz_server_create.restype = i32
        L.extremz_server_destroy.argtypes = [vp]
        L.extremz_server_submit.argtypes = [vp, ctypes.POINTER(Field), vp,
                                            ctypes.POINTER(ctypes.c_longlong)]
        L.extremz_server_submit.restype = i32
        L.extremz_server_poll.argtypes = [vp, ctypes.c_longlong, ctypes.POINTER(Report),
                                          ctypes.POINTER(ctypes.c_double)]
        L.extremz_server_poll.restype = i32
        L.extremz_server_wait.argtypes = [vp, ctypes.c_longlong, i32, ctypes.POINTER(Report),
                                          ctypes.POINTER(ctypes.c_double)]
        L.extremz_server_wait.restype = i32
        L.extremz_server_get_stats.argtypes = [vp, ctypes.POINTER(ServerStats)]
        L.extremz_job_footprint.argtypes = [i32, i32, i32, i32]
        L.extremz_job_footprint.restype = ctypes.c_longlong
        L.extremz_correct_device_noalloc.argtypes = [vp, vp, i32, i32, i32, i32,
                                                     ctypes.POINTER(Params),
                                                     ctypes.POINTER(Report), vp]
        L.extremz_correct_device_noalloc.restype = i32
        L.extremz_noalloc_max_voxels.restype = ctypes.c_longlong
        L.extremz_lut.argtypes = [vp, i32]
        L.extremz_lut.restype = i32
        L.extremz_status_string.argtypes = [i32]
        L.extremz_status_string.restype = ctypes.c_char_p
        L.extremz_last_cuda_error.restype = ctypes.c_char_p
        _lib = L
        return L


def status_string(st: int) -> str:
    return load().extremz_status_string(st).decode()


def _check(st: int, allow_cap: bool = True):
    if st == OK or (allow_cap and st == ROUND_CAP):
        return
    msg = status_string(st)
    if st == CUDA_ERR:
        msg += ": " + load().extremz_last_cuda_error().decode()
    raise ExtremzError(st, msg)


def make_params(bound: float, *, thr: float = 0.0, q: int = 4, edit_type: int = 1,
                max_outer: int = 1000, max_cloop_rounds: int = 100000,
                final_join: bool = True, preserve_join: bool = False,
                profile=False, tma=None, device_iter_cap: int = 0,
                blocks_per_sm: int = 0, pass_chunk: int = 0, tuned: bool = True,
                tuning_key=None, wn_order: str = "lockstep") -> Params:
    """profile: False, True (time every kernel class) or an iterable of class
    names from KCLASS_NAMES to time only those.

    wn_order: how the reference's wrong-neighbour race is resolved:
    "lockstep" (default, the reference's own outcome) or "ascending" (saddles
    in ascending id, EXTREMZ_FLAG_WN_ASCENDING).

    tma, blocks_per_sm, pass_chunk: launch-shape knobs (results do not depend
    on them).  Those left unset come from the autotuner's table for the
    field's dtype and size (tuning_key = (dtype name, voxels)) when ``tuned``
    and a table exists, else the library defaults."""
    p = Params()
    load().extremz_default_params(ctypes.byref(p))
    p.bound, p.thr, p.q, p.edit_type = float(bound), float(thr), int(q), int(edit_type)
    p.max_outer, p.max_cloop_rounds = int(max_outer), int(max_cloop_rounds)
    p.final_join, p.preserve_join = int(bool(final_join)), int(bool(preserve_join))
    p.device_iter_cap = int(device_iter_cap)
    if tuned and tuning_key is not None:
        from . import autotune
        t = autotune.lookup(*tuning_key)
        if t:
            if tma is None:
                tma = t["halo"] == "tma"
            blocks_per_sm = blocks_per_sm or t["blocks_per_sm"]
            pass_chunk = pass_chunk or t["pass_chunk"]
    p.tune_blocks_per_sm, p.tune_pass_chunk = int(blocks_per_sm), int(pass_chunk)
    p.flags = 0 if (tma is None or tma) else FLAG_NO_TMA
    if wn_order not in ("lockstep", "ascending"):
        raise ValueError(f"wn_order must be 'lockstep' or 'ascending', not {wn_order!r}")
    if wn_order == "ascending":
        p.flags |= FLAG_WN_ASCENDING
    if profile:
        p.flags |= FLAG_PROFILE
        if profile is not True:
            for name in profile:
                p.flags |= 1 << (PROFILE_CLASS_SHIFT + KCLASS_NAMES.index(name))
    return p


class Context:
    """One device workspace.  Not thread-safe: one correction at a time."""

    def __init__(self, device: int = 0):
        L = load()
        h = ctypes.c_void_p()
        _check(L.extremz_ctx_create(int(device), ctypes.byref(h)), allow_cap=False)
        self._h = h
        self.device = device

    def close(self):
        if self._h:
            load().extremz_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- device tensors -----------------------------------------------------
    def correct_device(self, f, decp, bound: float, *, stream=None, trace_cap: int = 0,
                       **kw):
        """Correct the CUDA tensor ``decp`` in place; ``f`` is the original.

        Both are contiguous float32/float64 CUDA tensors of shape (D, H, W) or
        (H, W).  Returns (CorrectionReport, trace array or None).
        """
        import torch
        assert f.is_cuda and decp.is_cuda and f.dtype == decp.dtype and f.shape == decp.shape
        assert f.is_contiguous() and decp.is_contiguous()
        dt = {torch.float32: F32, torch.float64: F64}[f.dtype]
        w, h, d = _whd(tuple(f.shape))
        if stream is None:
            stream = torch.cuda.current_stream(f.device).cuda_stream
        p = make_params(bound, tuning_key=(_dtname(dt), w * h * d), **kw)
        r = Report()
        tr = np.zeros(max(trace_cap, 1) * 4, dtype=np.int32)
        st = load().extremz_correct_device(self._h, f.data_ptr(), decp.data_ptr(), dt, w, h, d,
                                           ctypes.byref(p), ctypes.byref(r), stream,
                                           tr.ctypes.data if trace_cap else None, trace_cap * 4)
        _check(st)
        trace = None
        if trace_cap:
            trace = tr.reshape(-1, 4)
            trace = trace[trace[:, 0] != 0]
        return CorrectionReport.of(r), trace

    def mismatch_census(self, f, g, *, thr: float = 0.0, stream=None):
        """The eleven loop-test counters of field ``g`` against the original
        ``f`` (CUDA tensors), evaluated once with no edit; a dict by name
        (``COUNTER_NAMES``) plus the list under ``"counters"``."""
        import torch
        assert f.is_cuda and g.is_cuda and f.dtype == g.dtype and f.shape == g.shape
        assert f.is_contiguous() and g.is_contiguous()
        dt = {torch.float32: F32, torch.float64: F64}[f.dtype]
        w, h, d = _whd(tuple(f.shape))
        if stream is None:
            stream = torch.cuda.current_stream(f.device).cuda_stream
        out = np.zeros(11, dtype=np.int32)
        st = load().extremz_mismatch_census(self._h, f.data_ptr(), g.data_ptr(), dt, w, h, d,
                                            float(thr), out.ctypes.data, stream)
        _check(st, allow_cap=False)
        c = [int(x) for x in out]
        res = dict(zip(COUNTER_NAMES, c))
        res["counters"] = c
        return res

    def classify(self, field, *, stream=None):
        """Vertex types (int8) and steepest-ascent / steepest-descent roots
        (int32) of the CUDA tensor ``field``: three CUDA tensors of its shape."""
        import torch
        assert field.is_cuda and field.is_contiguous()
        dt = {torch.float32: F32, torch.float64: F64}[field.dtype]
        w, h, d = _whd(tuple(field.shape))
        if stream is None:
            stream = torch.cuda.current_stream(field.device).cuda_stream
        t = torch.empty(field.shape, dtype=torch.int8, device=field.device)
        ds = torch.empty(field.shape, dtype=torch.int32, device=field.device)
        as_ = torch.empty(field.shape, dtype=torch.int32, device=field.device)
        st = load().extremz_classify(self._h, field.data_ptr(), dt, w, h, d, t.data_ptr(),
                                     ds.data_ptr(), as_.data_ptr(), stream)
        _check(st, allow_cap=False)
        return t, ds, as_

    # -- edit streams -------------------------------------------------------
    def correct_encode(self, f, decp, bound: float, *, stream=None, zstd_level: int = 3, **kw):
        """Correct the CUDA tensor ``decp`` in place and return its edit stream.

        Returns (CorrectionReport, dict) with the index stream (numpy uint8),
        the edits (numpy, the field's dtype), the edited-voxel and entry
        counts, PSNR before and after, and the zstd sizes of both streams
        (-1 without libzstd).  See extremz_correct_encode.
        """
        import torch
        assert f.is_cuda and decp.is_cuda and f.dtype == decp.dtype and f.shape == decp.shape
        assert f.is_contiguous() and decp.is_contiguous()
        dt = {torch.float32: F32, torch.float64: F64}[f.dtype]
        w, h, d = _whd(tuple(f.shape))
        p = make_params(bound, tuning_key=(_dtname(dt), w * h * d), **kw)
        L = load()
        icap, ecap = ctypes.c_longlong(), ctypes.c_longlong()
        _check(L.extremz_edit_stream_caps(dt, w, h, d, p.edit_type, ctypes.byref(icap),
                                          ctypes.byref(ecap)), allow_cap=False)
        ibuf = torch.empty(max(1, icap.value), dtype=torch.uint8, device=f.device)
        ebuf = torch.empty(max(1, ecap.value), dtype=torch.uint8, device=f.device)
        es = EditStream()
        es.index, es.index_cap = ibuf.data_ptr(), icap.value
        es.edits, es.edits_cap = ebuf.data_ptr(), ecap.value
        if stream is None:
            stream = torch.cuda.current_stream(f.device).cuda_stream
        r = Report()
        st = L.extremz_correct_encode(self._h, f.data_ptr(), decp.data_ptr(), dt, w, h, d,
                                      ctypes.byref(p), ctypes.byref(r), stream, ctypes.byref(es))
        _check(st)
        torch.cuda.synchronize(f.device)
        index = ibuf[:es.index_bytes].cpu().numpy()
        npdt = np.float32 if dt == F32 else np.float64
        edits = ebuf[:es.edit_bytes].cpu().numpy().view(npdt)
        out = dict(index=index, edits=edits, edited=int(es.edited), n_edits=int(es.n_edits),
                   index_bytes=int(es.index_bytes), edit_bytes=int(es.edit_bytes),
                   psnr_before=float(es.psnr_before), psnr_after=float(es.psnr_after),
                   index_zstd=zstd_size(index, zstd_level), edits_zstd=zstd_size(edits, zstd_level))
        return CorrectionReport.of(r), out

    # -- topology -----------------------------------------------------------
    def persistence_pairs(self, field, *, stream=None):
        """Merge-tree persistence pairs of a CUDA tensor field.

        Returns (max_pairs, min_pairs): int32 arrays of shape (n, 2) holding
        (partner vertex, extremum vertex), extrema by rank (maxima ascending,
        minima descending in value then id).  See extremz_persistence_pairs.
        """
        import torch
        assert field.is_cuda and field.is_contiguous()
        dt = {torch.float32: F32, torch.float64: F64}[field.dtype]
        w, h, d = _whd(tuple(field.shape))
        n = w * h * d
        mx = torch.empty(2 * n, dtype=torch.int32, device=field.device)
        mn = torch.empty(2 * n, dtype=torch.int32, device=field.device)
        nx, nn = ctypes.c_longlong(), ctypes.c_longlong()
        if stream is None:
            stream = torch.cuda.current_stream(field.device).cuda_stream
        _check(load().extremz_persistence_pairs(self._h, field.data_ptr(), dt, w, h, d,
                                                mx.data_ptr(), 2 * n, mn.data_ptr(), 2 * n,
                                                ctypes.byref(nx), ctypes.byref(nn), stream),
               allow_cap=False)
        torch.cuda.synchronize(field.device)
        return (mx[:2 * nx.value].view(-1, 2).cpu().numpy(),
                mn[:2 * nn.value].view(-1, 2).cpu().numpy())

    def persistence_tree(self, field, *, stream=None):
        """Persistence pairs plus each extremum's merge target.

        Returns (max_pairs, min_pairs, max_parent, min_parent): the pairs of
        persistence_pairs() and, per extremum in the same order, the vertex of
        the extremum it merges into at its partner (the largest maximum /
        smallest minimum of its saddle's row, before constructMergeTree's
        compression; the global extremum holds itself).  See
        extremz_persistence_tree and merge_tree_branches().
        """
        import torch
        assert field.is_cuda and field.is_contiguous()
        dt = {torch.float32: F32, torch.float64: F64}[field.dtype]
        w, h, d = _whd(tuple(field.shape))
        n = w * h * d
        mx = torch.empty(2 * n, dtype=torch.int32, device=field.device)
        mn = torch.empty(2 * n, dtype=torch.int32, device=field.device)
        px = torch.empty(n, dtype=torch.int32, device=field.device)
        pn = torch.empty(n, dtype=torch.int32, device=field.device)
        nx, nn = ctypes.c_longlong(), ctypes.c_longlong()
        if stream is None:
            stream = torch.cuda.current_stream(field.device).cuda_stream
        _check(load().extremz_persistence_tree(self._h, field.data_ptr(), dt, w, h, d,
                                               mx.data_ptr(), 2 * n, mn.data_ptr(), 2 * n,
                                               px.data_ptr(), pn.data_ptr(), ctypes.byref(nx),
                                               ctypes.byref(nn), stream),
               allow_cap=False)
        torch.cuda.synchronize(field.device)
        return (mx[:2 * nx.value].view(-1, 2).cpu().numpy(),
                mn[:2 * nn.value].view(-1, 2).cpu().numpy(),
                px[:nx.value].cpu().numpy(), pn[:nn.value].cpu().numpy())

    def compare_topology(self, f, g):
        """Topology report of a corrected field g against its original f: the
        merge-tree persistence pairs of both (split and join trees), how many
        pairs are identical (same saddle, same extremum), and the largest
        change of a pair's persistence (value difference)."""
        out = {}
        fv = f.double().flatten().cpu().numpy()
        gv = g.double().flatten().cpu().numpy()
        for name, pa, pb in zip(("split", "join"), self.persistence_pairs(f),
                                self.persistence_pairs(g)):
            sa = {(int(p), int(e)) for p, e in pa}
            sb = {(int(p), int(e)) for p, e in pb}
            common = sa & sb
            dper = max((abs(abs(fv[e] - fv[p]) - abs(gv[e] - gv[p])) for p, e in common
                        if p >= 0), default=0.0)
            out[name] = {"pairs_original": len(sa), "pairs_corrected": len(sb),
                         "identical": len(common), "same": sa == sb,
                         "max_persistence_change": float(dper)}
        # Branch decompositions of the split tree, compared branch by branch
        # as the CPU driver does (main.cpp:478-504).
        tf, tg = self.persistence_tree(f), self.persistence_tree(g)
        bf = merge_tree_branches(fv, tf[0], tf[2], split=True)
        bg = merge_tree_branches(gv, tg[0], tg[2], split=True)
        out["split"]["branches"] = compare_branches(bf, bg)
        return out

    # -- batches ------------------------------------------------------------
    def correct_batch(self, items, *, stream=None):
        """Correct many CUDA tensors in place with shared launches.

        items: sequence of (f, decp, bound) or (f, decp, bound, kwargs) where
        kwargs are make_params() options for that field.  Fields may differ
        in dtype, shape and parameters.  Returns (list of CorrectionReport,
        total kernel launches of the batch).
        """
        import torch
        n = len(items)
        arr = (Field * max(n, 1))()
        keep = []
        for i, it in enumerate(items):
            f, decp, bound = it[0], it[1], it[2]
            kw = it[3] if len(it) > 3 else {}
            assert f.is_cuda and decp.is_cuda and f.dtype == decp.dtype and f.shape == decp.shape
            assert f.is_contiguous() and decp.is_contiguous()
            w, h, d = _whd(tuple(f.shape))
            arr[i].orig, arr[i].decp = f.data_ptr(), decp.data_ptr()
            arr[i].dtype = {torch.float32: F32, torch.float64: F64}[f.dtype]
            arr[i].width, arr[i].height, arr[i].depth = w, h, d
            arr[i].params = make_params(bound, tuning_key=(_dtname(arr[i].dtype), w * h * d),
                                        **kw)
            keep.append((f, decp))
        if stream is None:
            dev = items[0][0].device if n else torch.device("cuda", self.device)
            stream = torch.cuda.current_stream(dev).cuda_stream
        reps = (Report * max(n, 1))()
        st = load().extremz_correct_batch(self._h, arr, n, reps, stream)
        _check(st, allow_cap=False)
        out = [CorrectionReport.of(reps[i]) for i in range(n)]
        return out, (int(reps[0].kernel_launches) if n else 0)

    # -- host arrays ----------------------------------------------------------
    def correct_host(self, f: np.ndarray, decp: np.ndarray, bound: float, *, stream=None, **kw):
        """Correct the numpy array ``decp`` in place through host buffers."""
        assert f.dtype == decp.dtype and f.shape == decp.shape
        assert f.flags.c_contiguous and decp.flags.c_contiguous
        dt = {np.dtype(np.float32): F32, np.dtype(np.float64): F64}[f.dtype]
        w, h, d = _whd(f.shape)
        p = make_params(bound, tuning_key=(_dtname(dt), w * h * d), **kw)
        r = Report()
        st = load().extremz_correct_host(self._h, f.ctypes.data, decp.ctypes.data, dt, w, h, d,
                                         ctypes.byref(p), ctypes.byref(r), stream)
        _check(st)
        return CorrectionReport.of(r)


def _tree_rank(values: np.ndarray, verts: np.ndarray, split: bool) -> np.ndarray:
    """Rank of vertices in a tree's order: by (value, id) ascending for the
    split tree, descending for the join tree; a vertex listed twice gets the
    same rank."""
    verts = np.asarray(verts, np.int64)
    u = np.unique(verts)
    r = np.lexsort((u, np.asarray(values, np.float64)[u]))   # ascending (value, id)
    rank_u = np.empty(len(u), np.int64)
    rank_u[r] = np.arange(len(u))
    if not split:
        rank_u = len(u) - 1 - rank_u
    return rank_u[np.searchsorted(u, verts)]


def _compress_parents(values, pairs, par, split: bool) -> np.ndarray:
    """constructMergeTree's loop (:1869-1885) on parent ranks: a parent whose
    own partner comes before the extremum's partner in the descending order
    (it died first) is replaced by its parent, until nothing moves."""
    pairs = np.asarray(pairs, np.int64)
    n = len(pairs)
    par = np.array(par, np.int64)
    root = n - 1
    par[root] = root
    # Partner position in the descending order (smaller = earlier).
    srank = np.full(n, np.iinfo(np.int64).max)
    srank[:root] = -_tree_rank(values, pairs[:root, 0], split)
    while True:
        nxt = par[par]
        move = (nxt != par) & (srank[par] < srank)
        if not move.any():
            return par
        par = np.where(move, nxt, par)


def merge_tree_branches(values, pairs, parent, *, split: bool = True):
    """Branch decomposition of a merge tree (constructMergeTree,
    src/ExtreM.cpp:1863-1918) from persistence_tree() output.

    values: the field, flat.  pairs: (n, 2) (partner, extremum) by extremum
    rank, the global extremum last.  parent: per extremum, the extremum it
    merges into at its partner.  Each parent is first compressed to the
    first extremum along the parent chain that is still alive at the
    extremum's partner (whose own partner comes later in the tree order),
    as constructMergeTree's loop does.  Returns one int64 array of vertex
    ids per extremum: the extremum, the partners of the branches that join
    it, and its own partner (the opposite global extremum for the global
    one), in descending tree order -- the vertices of a reference Branch.
    The reference orders vertices by getSortedPositions, a sort by value
    alone whose order among equal values is unspecified; here ties go by id.
    """
    pairs = np.asarray(pairs, np.int64)
    n = len(pairs)
    if n == 0:
        return []
    ext, sad = pairs[:, 1], pairs[:, 0]
    idx = np.argsort(ext)
    par = _compress_parents(values, pairs, idx[np.searchsorted(ext[idx], np.asarray(parent, np.int64))],
                            split)
    # Vertices of every branch with their tree-order keys.
    allv = np.concatenate([ext, sad])
    key = _tree_rank(values, allv, split)
    kext, ksad = key[:n], key[n:]
    members = [[(int(kext[b]), int(ext[b]))] for b in range(n)]
    for b in range(n):
        p = int(par[b])
        if p != b:
            members[b].append((int(ksad[b]), int(sad[b])))
            members[p].append((int(ksad[b]), int(sad[b])))
        else:
            members[b].append((-1, int(sad[b])))
    return [np.array([v for _, v in sorted(m, reverse=True)], np.int64) for m in members]


def compare_branches(a, b):
    """Comparison of two branch decompositions.

    by rank: branch i against branch i, as the CPU driver prints it
    (main.cpp:478-504) -- a correction that reorders two maxima by value
    shifts every branch between them; by extremum: each branch against the
    branch of the same extremum vertex, the count that shows whether the
    merge tree kept its shape.  first_differences lists a few branches (by
    rank) that differ, with the first position where they do.
    """
    same_rank, diffs = 0, []
    for i, (x, y) in enumerate(zip(a, b)):
        if len(x) == len(y) and np.array_equal(x, y):
            same_rank += 1
        elif len(diffs) < 8:
            k = next((p for p in range(min(len(x), len(y))) if x[p] != y[p]), min(len(x), len(y)))
            diffs.append({"branch": i, "position": int(k)})
    by_ext = {int(y[0]): y for y in b if len(y)}
    same_ext = sum(1 for x in a if len(x) and int(x[0]) in by_ext
                   and np.array_equal(x, by_ext[int(x[0])]))
    return {"branches_original": len(a), "branches_corrected": len(b),
            "identical_by_rank": same_rank, "identical_by_extremum": same_ext,
            "same": same_rank == len(a) == len(b), "first_differences": diffs}


class Server:
    """Request loop with continuous batching (extremz_server_*).

    submit() queues a CUDA field pair and returns a ticket at once; the loop
    admits requests in arrival order while their device footprint fits the
    HBM budget, and serves all admitted requests with shared launches.
    """

    def __init__(self, device: int = 0, *, hbm_budget_bytes: int = 0, max_jobs: int = 0,
                 reserve_bytes: int = 0, split_voxels: int = 0):
        L = load()
        cfg = ServerConfig()
        cfg.hbm_budget_bytes, cfg.max_jobs = int(hbm_budget_bytes), int(max_jobs)
        cfg.reserve_bytes, cfg.split_voxels = int(reserve_bytes), int(split_voxels)
        h = ctypes.c_void_p()
        _check(L.extremz_server_create(int(device), ctypes.byref(cfg), ctypes.byref(h)),
               allow_cap=False)
        self._h = h
        self.device = device
        self._keep = {}

    def close(self):
        if self._h:
            load().extremz_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, f, decp, bound: float, *, stream=None, **kw) -> int:
        """Queue ``decp`` (corrected in place) against the original ``f``.

        The server's work starts after what is queued on ``stream`` (default:
        the current torch stream) at the time of the call."""
        import torch
        assert f.is_cuda and decp.is_cuda and f.dtype == decp.dtype and f.shape == decp.shape
        assert f.is_contiguous() and decp.is_contiguous()
        fd = Field()
        fd.orig, fd.decp = f.data_ptr(), decp.data_ptr()
        fd.dtype = {torch.float32: F32, torch.float64: F64}[f.dtype]
        fd.width, fd.height, fd.depth = _whd(tuple(f.shape))
        fd.params = make_params(bound, tuning_key=(_dtname(fd.dtype),
                                                   fd.width * fd.height * fd.depth), **kw)
        if stream is None:
            stream = torch.cuda.current_stream(f.device).cuda_stream
        t = ctypes.c_longlong()
        _check(load().extremz_server_submit(self._h, ctypes.byref(fd), stream, ctypes.byref(t)),
               allow_cap=False)
        self._keep[t.value] = (f, decp)
        return t.value

    def _take(self, st, t, r, lat):
        if st == PENDING:
            return None
        self._keep.pop(t, None)
        if st not in (OK, ROUND_CAP):
            _check(st)
        return CorrectionReport.of(r), lat.value

    def poll(self, ticket: int):
        """None while pending, else (CorrectionReport, latency in ms)."""
        r, lat = Report(), ctypes.c_double()
        st = load().extremz_server_poll(self._h, ticket, ctypes.byref(r), ctypes.byref(lat))
        return self._take(st, ticket, r, lat)

    def wait(self, ticket: int, timeout_ms: int = -1):
        r, lat = Report(), ctypes.c_double()
        st = load().extremz_server_wait(self._h, ticket, int(timeout_ms), ctypes.byref(r),
                                        ctypes.byref(lat))
        return self._take(st, ticket, r, lat)

    def stats(self) -> dict:
        s = ServerStats()
        load().extremz_server_get_stats(self._h, ctypes.byref(s))
        return {k: int(getattr(s, k)) for k, _ in ServerStats._fields_ if k != "reserved"}


def zstd_size(buf: np.ndarray, level: int = 3) -> int:
    """zstd-compressed size of a host array (-1 when libzstd is absent)."""
    b = np.ascontiguousarray(buf)
    return int(load().extremz_zstd_size(b.ctypes.data, b.nbytes, int(level)))


def job_footprint(voxels_or_shape, dtype) -> int:
    """Device bytes a Server charges a request against its HBM budget.

    voxels_or_shape: a voxel count or a (W, H, D) triple; dtype: numpy or
    torch float32/float64."""
    if isinstance(voxels_or_shape, (tuple, list)):
        w, h, d = (int(x) for x in voxels_or_shape)
    else:
        w, h, d = int(voxels_or_shape), 1, 1
    dt = F32 if str(dtype).endswith("float32") else F64
    return int(load().extremz_job_footprint(dt, w, h, d))


# Names of the eleven loop-test counters (extremz_report.counters order).
COUNTER_NAMES = ("wrong_split_nbrs", "wrong_join_nbrs", "false_max", "false_min", "false_saddle",
                 "wrong_max", "wrong_max_2", "wrong_saddle", "wrong_min", "wrong_min_2",
                 "wrong_saddle_join")


def _dtname(code: int) -> str:
    return "f32" if code == F32 else "f64"


def _whd(shape):
    if len(shape) == 2:
        return shape[1], shape[0], 1
    if len(shape) == 3:
        return shape[2], shape[1], shape[0]
    raise ValueError(f"field must be 2-D or 3-D, got shape {shape}")


_default_ctx = {}


def context(device: int = 0) -> Context:
    if device not in _default_ctx:
        _default_ctx[device] = Context(device)
    return _default_ctx[device]


def correct(f: np.ndarray, decp: np.ndarray, bound: float, *, device: int = 0, **kw):
    """Host-array correction call: returns (corrected copy, report)."""
    out = np.ascontiguousarray(decp).copy()
    rep = context(device).correct_host(np.ascontiguousarray(f), out, bound, **kw)
    return out, rep


def noalloc_max_voxels() -> int:
    return int(load().extremz_noalloc_max_voxels())


def correct_device_noalloc(f, decp, bound: float, *, stream=None, **kw) -> CorrectionReport:
    """Allocation-free correction of the CUDA tensor ``decp`` in place.

    For callers that cannot allocate device memory while correcting
    (applications whose allocator owns the device memory, real-time code that
    forbids allocation after start-up):
    the workspace is a static device array of the library, for fields of at
    most noalloc_max_voxels() voxels.  Calls share that array, so they must not
    overlap on the GPU.  The first call on a device does a synchronous set-up;
    make it before any stream capture.
    """
    import torch
    assert f.is_cuda and decp.is_cuda and f.dtype == decp.dtype and f.shape == decp.shape
    assert f.is_contiguous() and decp.is_contiguous()
    dt = {torch.float32: F32, torch.float64: F64}[f.dtype]
    w, h, d = _whd(tuple(f.shape))
    if stream is None:
        stream = torch.cuda.current_stream(f.device).cuda_stream
    p = make_params(bound, **kw)
    r = Report()
    with torch.cuda.device(f.device):
        st = load().extremz_correct_device_noalloc(f.data_ptr(), decp.data_ptr(), dt, w, h, d,
                                                   ctypes.byref(p), ctypes.byref(r), stream)
    _check(st)
    return CorrectionReport.of(r)


def lut() -> np.ndarray:
    out = np.zeros(24800, dtype=np.int32)
    n = load().extremz_lut(out.ctypes.data, out.size)
    assert n == 24800
    return out
