"""Benchmark: ExtreM topology correction, Mvox/s to zero topological mismatch.

One step = one full correction (setup, c_loops, the outer loop to zero
mismatch counters, final join-saddle pass) of a fresh copy of the synthetic
decompressed field, inputs resident in HBM.  The default workload is the
512^3 float64 field (4096 Gaussians, k^-5/3 noise, seed 2, eb 1e-5 relative);
the 256^3 fields in float64 and float32 are measured beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
                    [--impl ours|reference]

With N > 1 (launched by torch.distributed.run) every rank corrects its own
field of the same workload: the path has no data exchange, so ranks are
replicas and the value is all ranks' voxels over the max-over-ranks time.

--impl reference times the reference algorithm's CPU implementation on the
host cores (the CPU restatement of the reference's GPU correction, built
with OpenMP) on a bounded crop of the same workload, rank 0 only; its
config names the crop's shape.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from extrem_z_b200 import synth  # noqa: E402

METRIC = "Mvox/s to zero topological mismatch"
UNIT = "Mvox/s"

# name -> (constructor, description); the headline is the 512^3 float64 field.
WORKLOADS = {
    "plain256_f64": (lambda: synth.plain_256(np.float64),
                     "256^3 float64, 512 Gaussians + k^-2 noise, seed 1, eb 1e-4 rel"),
    "plain256_f32": (lambda: synth.plain_256(np.float32),
                     "256^3 float32, 512 Gaussians + k^-2 noise, seed 1, eb 1e-4 rel"),
    "plain64_f32": (lambda: synth.plain_64(np.float32),
                    "64^3 float32, 64 Gaussians + k^-2 noise, seed 0, eb 1e-3 rel"),
    "plain512_f64": (lambda: synth.plain_512(),
                     "512^3 float64, 4096 Gaussians + k^-5/3 noise, seed 2, eb 1e-5 rel"),
}
# Batched and served forms (not plain fields): their own lines.
FORM_WORKLOADS = {
    "mixed64": "64 fields, edges log-uniform 32-192 (25% 2-D slices), f32/f64 50/50, "
               "eb log-uniform 1e-5..1e-2 rel, seeds 100-163",
    "serve": "Poisson request stream, voxels log-uniform 32^3-384^3, f32/f64 50/50, eb "
             "log-uniform 1e-5..1e-2 rel, seed 10000+id, HBM admission budget 120 GB",
}
DEFAULT_WORKLOAD = "plain512_f64"
# Measured beside the headline (fewer steps): the 256^3 field in both dtypes.
SECONDARY = ("plain256_f64", "plain256_f32")
# Edge of the cubic crop the CPU legs correct (a full 512^3 correction takes
# the OpenMP oracle minutes per step).
CPU_EDGE = 128
SERVE_RATES = (10, 30, 100, 300, 1000, 2000)
# Workspace memory the server maps at start-up (within its 120 GB budget).
SERVE_RESERVE_BYTES = 48 << 30
PARAMS = dict(q=4, edit_type=1, thr=0.0, max_outer=1000, max_cloop_rounds=100000,
              final_join=True)

# Dominant work: the manifold rounds of the decompressed field, the steepest
# directions (k_direction) and the pointer jumping (k_jump2).  A correction's
# first round computes every tile and follows every vertex's chains (kernel
# classes "direction_first" and "jump_first"); its algorithmic bytes are
# N*(S + 8): read every decompressed value (S bytes) and write its two int32
# labels.  Everything else the kernels move (tile-compressed pointers, original
# roots, change marks, chain hops) is the design's own traffic, not counted.
# The later rounds (classes "direction" and "jump") recompute only the tiles
# whose values changed and follow only chains whose root was touched, so a
# full-field byte count does not describe them; they are reported beside it.
DOMINANT = ("direction_first", "jump_first")
LATER = ("direction", "jump")
DOMINANT_KERNEL = ("first manifold round of the decompressed field (k_direction + k_jump2, "
                   "every tile and vertex)")
# The next kernel by device time (the saddle pass after each manifold round),
# timed beside the dominant ones in a few extra steps.
RUNNER_UP = "rows"
RUNNER_UP_KERNEL = "k_saddle_pass"


def round_bytes(n: int, s: int) -> int:
    """Algorithmic bytes of one manifold round of an n-voxel field of s-byte
    values: the value read and the two label writes per voxel."""
    return n * (s + 8)


def jump_design_bytes(n: int, rounds: int) -> int:
    """Bytes k_jump2 itself must move in `rounds` first (full) manifold rounds:
    per voxel it reads the two tile-compressed pointers and the two original
    roots (16 B; a first round needs no old labels) and writes both labels,
    the mismatch byte and the changed-input byte (10 B); the change bits
    (N / 8 bytes) are not counted."""
    return 26 * n * rounds


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of the first
# decompressed manifold round (k_direction + k_jump2 over every tile and
# vertex), by workload: the ncu capture of the 256^3 float64 correction
# (226.3 MB for k_direction + 458.0 MB for k_jump2 per first round), and the same
# per voxel for the 512^3 field (eight times the voxels; both kernels stream
# whole arrays once).  Not captured for float32.
MEASURED_TRAFFIC = {"plain256_f64": 684_300_000, "plain512_f64": 8 * 684_300_000}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            pk = json.load(fh)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.dev)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi's start-up (driver library load and init) must not
            # overlap the timed region: wait for its first sample.
            t0 = time.time()
            while not self.lines and time.time() - t0 < 10.0:
                time.sleep(0.02)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = os.environ.get("EXTREMZ_DIST_BACKEND") or (
            "nccl" if torch.cuda.is_available() else "gloo")
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def crop(field, edge: int):
    """Leading edge^3 sub-volume of a workload (same values, same bound)."""
    f = np.ascontiguousarray(field.f[:edge, :edge, :edge])
    g = np.ascontiguousarray(field.decp[:edge, :edge, :edge])
    return f, g


def time_oracle(field, edge: int, threads: int):
    """Oracle correction of a crop; returns (seconds, voxels, report)."""
    from oracle import ffi
    ffi.set_threads(threads)
    f, g = crop(field, edge)
    t0 = time.perf_counter()
    _, rep, _ = ffi.correct(f, g, field.eb, q=PARAMS["q"], edit_type=PARAMS["edit_type"],
                            thr=PARAMS["thr"], max_outer=PARAMS["max_outer"],
                            max_cloop_rounds=PARAMS["max_cloop_rounds"],
                            final_join=PARAMS["final_join"])
    return time.perf_counter() - t0, f.size, rep


def run_reference_form(args):
    """Reference arm of the batched / served workloads: the CPU restatement on
    all host threads over a bounded sample of the same fields, fields/s."""
    from oracle import ffi
    threads = os.cpu_count() or 1
    ffi.set_threads(threads)
    if args.workload == "mixed64":
        specs = synth.mixed_batch_specs(64)
    else:
        specs = [synth.serving_request_spec(i) for i in range(64)]
    # Bounded sample: the smallest fields of the workload, up to 16.
    order = sorted(range(len(specs)), key=lambda i: specs[i]["w"] * specs[i]["h"] * specs[i]["d"])
    sample = [specs[i] for i in order[:16]]
    fields = [synth.make_field(s["w"], s["h"], s["d"], n_gauss=s["n_gauss"], seed=s["seed"],
                               rel=s["rel"], dtype=s["dtype"]) for s in sample]
    total = 0.0
    for step in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        for x in fields[:4] if step < args.warmup else fields:
            ffi.correct(x.f, x.decp, x.eb, q=PARAMS["q"], edit_type=PARAMS["edit_type"],
                        thr=PARAMS["thr"], max_outer=PARAMS["max_outer"],
                        max_cloop_rounds=PARAMS["max_cloop_rounds"],
                        final_join=PARAMS["final_join"])
        if step >= args.warmup:
            total += time.perf_counter() - t0
    value = len(fields) * args.steps / total
    desc = (f"the {len(fields)} smallest fields of the {args.workload} workload, each corrected "
            f"to zero mismatch by the CPU restatement of the reference correction")
    line = {"impl": "reference", "metric": "fields/s to zero topological mismatch", "value": value,
            "unit": "fields/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": args.workload, "description": FORM_WORKLOADS[args.workload]},
            "cpu_baseline": {"value": value, "unit": "fields/s", "cores": threads, "kind": "port",
                             "sample": desc},
            "e2e": {"value": value, "unit": "fields/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_reference(args, world, rank):
    if rank != 0:
        return
    if args.workload in FORM_WORKLOADS:
        return run_reference_form(args)
    field = WORKLOADS[args.workload][0]()
    threads = os.cpu_count() or 1
    edge = min(args.cpu_edge, *field.f.shape)
    for _ in range(args.warmup):
        time_oracle(field, edge, threads)
    total_s, vox = 0.0, 0
    for _ in range(args.steps):
        s, n, rep = time_oracle(field, edge, threads)
        total_s += s
        vox += n
    value = vox / total_s / 1e6
    sample = (f"leading {edge}^3 crop of the {args.workload} field (same bound), full "
              f"correction to zero mismatch, CPU restatement of the reference correction")
    # The config names what was timed: the crop, not the whole field (the
    # rate to zero mismatch depends on the field's size and round count).
    cfg = config_of(args, field, shape_whd=list(crop(field, edge)[0].shape[::-1]))
    cfg["sample_of"] = {"workload": args.workload, "shape_whd": list(field.shape_whd)}
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * total_s / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dtype_name(field),
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def dtype_name(field):
    return "f64" if field.f.dtype == np.float64 else "f32"


def config_of(args, field, shape_whd=None):
    d, h, w = field.f.shape
    return {"workload": args.workload, "description": WORKLOADS[args.workload][1],
            "shape_whd": shape_whd or [w, h, d], "eb_abs": field.eb, "params": PARAMS,
            "l2": "inputs larger than L2 (two fields of N*S bytes > 126 MB)" if
            2 * field.f.nbytes > 126e6 else "inputs smaller than L2",
            "parallelism": f"replicas x{args.gpus}" if args.gpus > 1 else "single"}


def correct_steps(ctx, f, g, g0, field, stream, steps, profile=False, **over):
    """`steps` corrections of fresh copies of the decompressed field; reports."""
    params = dict(PARAMS, **over)
    reps = []
    for _ in range(steps):
        g.copy_(g0)
        rep, _ = ctx.correct_device(f, g, field.eb, stream=stream.cuda_stream,
                                    profile=profile or False, **params)
        reps.append(rep)
    return reps


def timed_steps(ctx, f, g, g0, field, stream, steps, profile=False, **over):
    """Device time (ms, CUDA events on the launching stream) of `steps`
    corrections, and their reports."""
    import torch
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    reps = correct_steps(ctx, f, g, g0, field, stream, steps, profile, **over)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), reps


def manifold_roofline(reps, n, s, step_ms, peak, peak_kind, traffic=None):
    """Roofline of the first decompressed manifold round of each correction in
    `reps` (run with the first-round and later-round classes timed), and the
    later rounds beside it."""
    dir_ms = sum(r.prof_ms["direction_first"] for r in reps)
    jump_ms = sum(r.prof_ms["jump_first"] for r in reps)
    firsts = sum(r.prof_launches["jump_first"] for r in reps)
    ms = dir_ms + jump_ms
    alg = round_bytes(n, s) * firsts
    achieved = alg / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
    jb = jump_design_bytes(n, firsts)
    jump_gbs = jb / (jump_ms * 1e-3) / 1e9 if jump_ms > 0 else 0.0
    later = sum(r.manifold_rounds - r.manifold_reused for r in reps) - firsts
    ldir = sum(r.prof_ms["direction"] for r in reps)
    ljump = sum(r.prof_ms["jump"] for r in reps)
    return {"bound": "hbm", "kernel": DOMINANT_KERNEL, "achieved": achieved, "peak": peak,
            "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic,
            "traffic_note": "ncu DRAM bytes of the first manifold round (k_direction + "
                            "k_jump2) of the 256^3 float64 correction, scaled to this field "
                            "by its voxel count; the excess over the algorithmic bytes is "
                            "the design's own arrays (tile pointers, old labels, original "
                            "roots)" if traffic else None,
            "algorithmic_bytes_per_launch": round_bytes(n, s),
            "algorithmic_bytes_note": "N*(S+8) per round: the value read and two int32 label "
                                      "writes per voxel",
            "launches": firsts, "kernel_ms": ms, "direction_ms": dir_ms, "jump_ms": jump_ms,
            "share_of_step": ms / step_ms if step_ms else None,
            "jump_design_bytes": {"kernel": "k_jump2", "bytes": jb, "achieved_gbs": jump_gbs,
                                  "frac": jump_gbs / peak,
                                  "note": "the bytes k_jump2 itself moves in a first round "
                                          "(pointers and original roots read, labels, mismatch "
                                          "and changed-input bytes written: 26 B per voxel), "
                                          "a lower bound"},
            "later_rounds": {
                "rounds": later, "reused": sum(r.manifold_reused for r in reps),
                "direction_ms": ldir, "jump_ms": ljump,
                "ms_per_round": (ldir + ljump) / later if later else None,
                "share_of_step": (ldir + ljump) / step_ms if step_ms else None,
                "note": "changed tiles' directions and touched chains only"}}


def census_of(ctx, f, g):
    """Mismatch census of the corrected field g against f (GPU, untimed)."""
    import torch
    c = ctx.mismatch_census(f, g)
    torch.cuda.synchronize()
    c["critical_point_mismatches"] = c["false_max"] + c["false_min"] + c["false_saddle"]
    c["label_mismatches"] = c["wrong_split_nbrs"] + c["wrong_join_nbrs"]
    c["split_tree_zero"] = all(c[k] == 0 for k in ("wrong_split_nbrs", "false_max", "false_min",
                                                   "false_saddle", "wrong_max", "wrong_max_2",
                                                   "wrong_saddle"))
    return c


def measure_secondary(ctx, local, name, steps, peak, peak_kind):
    """One 256^3 line beside the headline: Mvox/s to zero mismatch, rounds,
    manifold-round roofline and the census of the corrected field."""
    import torch
    dev = torch.device("cuda", local)
    field = WORKLOADS[name][0]()
    n, s = field.f.size, field.f.itemsize
    f = torch.from_numpy(field.f).to(dev)
    g0 = torch.from_numpy(field.decp).to(dev)
    g = torch.empty_like(g0)
    stream = torch.cuda.current_stream(dev)
    # Three warm-up corrections: a tick's launches become a CUDA graph at the
    # third sighting, so the timed steps replay graphs as the headline's do.
    correct_steps(ctx, f, g, g0, field, stream, 3)
    ms, reps = timed_steps(ctx, f, g, g0, field, stream, steps,
                           profile=list(DOMINANT) + list(LATER))
    r0 = reps[-1]
    out = {"workload": name, "description": WORKLOADS[name][1], "steps": steps,
           "value": n * steps / (ms * 1e-3) / 1e6, "unit": UNIT, "ms_per_step": ms / steps,
           "rounds": {"outer_iters": r0.outer_iters, "cloop_rounds": r0.cloop_rounds,
                      "manifold_rounds": r0.manifold_rounds,
                      "manifold_reused": r0.manifold_reused, "status": r0.status},
           "roofline": manifold_roofline(reps, n, s, ms, peak, peak_kind,
                                         MEASURED_TRAFFIC.get(name)),
           "census": census_of(ctx, f, g)}
    del f, g, g0
    torch.cuda.empty_cache()
    return out


def run_ours(args, world, rank, local):
    import torch
    from extrem_z_b200 import api
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    field = WORKLOADS[args.workload][0]()
    n = field.f.size
    s = field.f.itemsize
    tdt = torch.float64 if s == 8 else torch.float32
    f = torch.from_numpy(field.f).to(dev)
    g0 = torch.from_numpy(field.decp).to(dev)
    g = torch.empty_like(g0)
    ctx = api.Context(local)
    stream = torch.cuda.current_stream(dev)

    reps = correct_steps(ctx, f, g, g0, field, stream, args.warmup)
    torch.cuda.synchronize()
    if reps and reps[-1].status != 0:
        raise RuntimeError(f"correction did not converge: {reps[-1]}")

    # Timed region: device time of exactly K steps, max over ranks.  The
    # manifold-round kernels record CUDA events around themselves (inside the
    # tick graphs) for the roofline.
    sampler = ClockSampler(local)  # every rank samples its own GPU; rank 0 reports
    sampler.start()
    barrier(world)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # An NVTX range names the timed steps for a profiler's kernel filter
    # (ncu --nvtx --nvtx-include "timed/").
    torch.cuda.nvtx.range_push("timed")
    ev0.record(stream)
    reps = correct_steps(ctx, f, g, g0, field, stream, args.steps,
                         profile=list(DOMINANT) + list(LATER))
    ev1.record(stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    barrier(world)
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms, world)
    value = world * n * args.steps / (ms_max * 1e-3) / 1e6
    launches = sum(r.kernel_launches for r in reps)
    # What the corrected field (final join pass on, as in the reference's
    # main()) still differs in: the loop test's counters evaluated once more.
    census = census_of(ctx, f, g)

    peak, peak_kind = measured_peaks()
    roofline = manifold_roofline(reps, n, s, ms, peak, peak_kind,
                                 MEASURED_TRAFFIC.get(args.workload))
    # The next kernel by device time, timed beside the dominant ones in a few
    # steps after the timed region.
    ru_reps = correct_steps(ctx, f, g, g0, field, stream, 2, profile=list(DOMINANT) + [RUNNER_UP])
    torch.cuda.synchronize()
    roofline["runner_up"] = {
        "kernel": RUNNER_UP_KERNEL, "steps": len(ru_reps),
        "kernel_ms": sum(r.prof_ms[RUNNER_UP] for r in ru_reps),
        "dominant_kernel_ms": sum(r.prof_ms[k] for r in ru_reps for k in DOMINANT),
        "launches": sum(r.prof_launches[RUNNER_UP] for r in ru_reps)}

    # The same correction without the final join-saddle pass: the loop ends
    # at zero counters, so the field keeps zero split-tree mismatch.
    fj_steps = max(1, min(args.steps, 5))
    fj_ms, fj_reps = timed_steps(ctx, f, g, g0, field, stream, fj_steps, final_join=False)
    final_join_off = {"steps": fj_steps, "value": n * fj_steps / (fj_ms * 1e-3) / 1e6,
                      "unit": UNIT, "ms_per_step": fj_ms / fj_steps,
                      "status": fj_reps[-1].status, "census": census_of(ctx, f, g)}

    # End to end through the host-buffer entry point: H2D of both fields from
    # pinned memory, correction, D2H of the corrected field, every step.
    hf = torch.from_numpy(field.f).pin_memory().numpy()
    hg0 = field.decp
    hg = torch.empty(field.decp.shape, dtype=tdt).pin_memory().numpy()
    np.copyto(hg, hg0)
    ctx.correct_host(hf, hg, field.eb, stream=stream.cuda_stream, **PARAMS)
    e2e_s = 0.0
    e2e_steps = max(1, min(args.steps, 5))
    back = 0
    barrier(world)
    for _ in range(e2e_steps):
        np.copyto(hg, hg0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        hrep = ctx.correct_host(hf, hg, field.eb, stream=stream.cuda_stream, **PARAMS)
        e2e_s += time.perf_counter() - t0
        back += hrep.host_bytes_back
    e2e_s = max_over_ranks(e2e_s, world)
    # Device -> host: the changed voxels' ids and values (the host buffer
    # already holds the rest), as the library reports them.
    g.copy_(g0)
    ctx.correct_device(f, g, field.eb, stream=stream.cuda_stream, **PARAMS)
    e2e = {"value": world * n * e2e_steps / e2e_s / 1e6, "unit": UNIT,
           "h2d_bytes_per_step": 2 * n * s, "d2h_bytes_per_step": back // e2e_steps,
           "entry_point": "extremz_correct_host",
           # the host buffer against the device-resident correction (outside the timing)
           "bit_identical_to_device": bool(np.array_equal(
               hg.view(np.uint8), g.cpu().numpy().view(np.uint8)))}
    del hf, hg

    # The CPU restatement of the reference correction on all host cores, on a
    # crop of the same field (a full 512^3 correction takes it minutes), and
    # this library on the same crop, so that the two rates compare like with
    # like.
    cpu = None
    same_crop = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        edge = min(args.cpu_edge, *field.f.shape)
        secs, vox, crep = time_oracle(field, edge, threads)
        cpu = {"value": vox / secs / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"leading {edge}^3 crop of the same field and bound, full "
                         f"correction to zero mismatch by the OpenMP CPU restatement of the "
                         f"reference correction ({secs:.2f} s, status {crep['status']})"}
        cf, cg = crop(field, edge)
        tf = torch.from_numpy(cf).to(dev)
        tg0 = torch.from_numpy(cg).to(dev)
        tg = torch.empty_like(tg0)
        crop_field = synth.Field(f=cf, decp=cg, eb=field.eb, seed=field.seed, rel=field.rel)
        correct_steps(ctx, tf, tg, tg0, crop_field, stream, 2)
        cms, _ = timed_steps(ctx, tf, tg, tg0, crop_field, stream, 5)
        same_crop = {"shape_whd": [edge] * 3, "value": vox * 5 / (cms * 1e-3) / 1e6, "unit": UNIT,
                     "cpu_value": cpu["value"], "ratio": vox * 5 / (cms * 1e-3) / 1e6 / cpu["value"],
                     "note": "this library, device-resident, on the crop the CPU leg corrects"}
        del tf, tg, tg0

    # Edit stream of the same correction (extremz_correct_encode): the extra
    # device time of the encoder over the plain correction, the stream sizes
    # and their zstd sizes, beside the oracle's CPU encoder on the whole field.
    edit_stream = None
    if rank == 0 and world == 1 and not args.no_forms:
        edit_stream = measure_edit_stream(ctx, f, g, g0, field, stream, args.no_cpu_baseline)

    # Topology check of the corrected field: merge-tree persistence pairs of
    # the original and the corrected field on the GPU, beside the oracle's
    # union-find on a crop.
    topology = None
    if rank == 0 and world == 1 and not args.no_forms:
        topology = measure_topology(ctx, f, g, g0, field, stream, args)

    r0 = reps[-1]
    rounds = {"outer_iters": r0.outer_iters, "cloop_rounds": r0.cloop_rounds,
              "manifold_rounds": r0.manifold_rounds, "manifold_reused": r0.manifold_reused,
              "status": r0.status, "counters": r0.counters, "cp_counts": r0.cp_counts}
    del f, g, g0
    torch.cuda.empty_cache()

    secondary = None
    if rank == 0 and world == 1 and not args.no_secondary:
        secondary = [measure_secondary(ctx, local, name, 5, peak, peak_kind)
                     for name in SECONDARY if name != args.workload]

    forms = None
    if not args.no_forms and world == 1:
        b = measure_batched(local, 2, 3)
        sv = measure_served(local, SERVE_RATES)
        forms = {"batched": {"workload": "mixed64", "fields_per_s": b["batched"]["fields_per_s"],
                             "plain_loop_fields_per_s": b["plain_loop"]["fields_per_s"],
                             "speedup": b["speedup"],
                             "bit_identical_to_plain": b["bit_identical_to_plain"],
                             "gpu_launches": b["batched"]["gpu_launches"],
                             "plain_loop_gpu_launches": b["plain_loop"]["gpu_launches"]},
                 "served": {"workload": f"serve ({sv['requests_max']} requests at most per rate)",
                            "plain_loop_fields_per_s": sv["plain_loop"]["fields_per_s"],
                            "alone_ms": sv["alone_ms"],
                            "peak_running": sv["peak_running"],
                            "sweep": [{k: x[k] for k in ("rate_req_s", "requests", "p50_ms",
                                                         "p99_ms", "slowdown_p50",
                                                         "slowdown_p99", "fields_per_s",
                                                         "mean_in_system")}
                                      for x in sv["sweep"]],
                            "bit_identical_to_plain": sv["bit_identical_to_plain"]}}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": dtype_name(field), "data": "synthetic (seeded generator, no dataset)",
                "config": config_of(args, field), "e2e": e2e, "gpu_launches": launches,
                "roofline": roofline, "cpu_baseline": cpu, "gpu_same_crop": same_crop,
                "clocks": clocks,
                "headline": "final join-saddle pass on, as the reference's main() runs it "
                            "unconditionally (src/ExtreM_cuda.cu:5997); the output is the "
                            "reference's control flow, bit-exact with the oracle",
                "census": census, "final_join_off": final_join_off,
                "secondary": secondary, "forms": forms,
                "edit_stream": edit_stream, "topology": topology, "rounds": rounds}
        print(json.dumps(line), flush=True)
    ctx.close()


def measure_edit_stream(ctx, f, g, g0, field, stream, skip_cpu):
    """Device time of extremz_correct_encode against extremz_correct_device
    on the same field (streams into preallocated device buffers), the stream
    sizes and zstd sizes, and the oracle's CPU encoder on the whole field."""
    import ctypes
    import torch
    from extrem_z_b200 import api
    L = api.load()
    dt = api.F64 if field.f.dtype == np.float64 else api.F32
    d, h, w = field.f.shape
    icap, ecap = ctypes.c_longlong(), ctypes.c_longlong()
    L.extremz_edit_stream_caps(dt, w, h, d, PARAMS["edit_type"], ctypes.byref(icap),
                               ctypes.byref(ecap))
    ibuf = torch.empty(icap.value, dtype=torch.uint8, device=f.device)
    ebuf = torch.empty(ecap.value, dtype=torch.uint8, device=f.device)
    es = api.EditStream()
    es.index, es.index_cap, es.edits, es.edits_cap = (ibuf.data_ptr(), icap.value,
                                                      ebuf.data_ptr(), ecap.value)
    p = api.make_params(field.eb, tuning_key=("f64" if dt == api.F64 else "f32", field.f.size),
                        **PARAMS)
    r = api.Report()

    def timed(encode):
        best = None
        for _ in range(3):
            g.copy_(g0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if encode:
                st = L.extremz_correct_encode(ctx._h, f.data_ptr(), g.data_ptr(), dt, w, h, d,
                                              ctypes.byref(p), ctypes.byref(r),
                                              stream.cuda_stream, ctypes.byref(es))
            else:
                st = L.extremz_correct_device(ctx._h, f.data_ptr(), g.data_ptr(), dt, w, h, d,
                                              ctypes.byref(p), ctypes.byref(r),
                                              stream.cuda_stream, None, 0)
            e1.record(stream)
            torch.cuda.synchronize()
            assert st == 0, st
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        return best

    plain_ms = timed(False)
    enc_ms = timed(True)
    index = ibuf[:es.index_bytes].cpu().numpy()
    edits = ebuf[:es.edit_bytes].cpu().numpy()
    n = field.f.size
    out = {"entry_point": "extremz_correct_encode", "edit_type": PARAMS["edit_type"],
           "edited": int(es.edited), "edit_ratio": es.edited / n, "n_edits": int(es.n_edits),
           "index_bytes": int(es.index_bytes), "edit_bytes": int(es.edit_bytes),
           "index_zstd_bytes": api.zstd_size(index), "edits_zstd_bytes": api.zstd_size(edits),
           "psnr_before": es.psnr_before, "psnr_after": es.psnr_after,
           "correct_ms": plain_ms, "encode_extra_ms": enc_ms - plain_ms}
    if not skip_cpu:
        from oracle import ffi
        fixed = g.cpu().numpy()
        t0 = time.perf_counter()
        ffi.encode(field.f, field.decp, fixed, None, field.eb, q=PARAMS["q"],
                   edit_type=PARAMS["edit_type"])
        out["cpu_encode_ms"] = 1e3 * (time.perf_counter() - t0)
        out["cpu_encode_cores"] = 1
    return out


def measure_topology(ctx, f, g, g0, field, stream, args):
    import torch
    g.copy_(g0)
    ctx.correct_device(f, g, field.eb, stream=stream.cuda_stream, **PARAMS)
    torch.cuda.synchronize()
    ctx.persistence_pairs(f)  # warm
    best = None
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.persistence_pairs(f)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    rep = ctx.compare_topology(f, g)
    out = {"entry_point": "extremz_persistence_pairs", "gpu_ms_per_field": 1e3 * best,
           "note": "wall time of one call (analysis pass, sorts, pairing rounds, copy to host)",
           "split": rep["split"], "join": rep["join"]}
    if not args.no_cpu_baseline:
        from oracle import ffi
        fc, _ = crop(field, args.cpu_edge)
        t0 = time.perf_counter()
        ffi.persistence_pairs(fc)
        out["cpu_union_find_ms"] = 1e3 * (time.perf_counter() - t0)
        out["cpu_sample"] = f"leading {args.cpu_edge}^3 crop of the original field, 1 thread"
        tc = torch.from_numpy(np.ascontiguousarray(fc)).to(f.device)
        t0 = time.perf_counter()
        ctx.persistence_pairs(tc)
        torch.cuda.synchronize()
        out["gpu_ms_same_crop"] = 1e3 * (time.perf_counter() - t0)
    return out


# ---------------------------------------------------------------------------
# Batched form: the 64-field mixed batch, batched vs the plain per-field loop.
# ---------------------------------------------------------------------------
def mixed_fields():
    specs = synth.mixed_batch_specs(64)
    return specs, [synth.make_field(s["w"], s["h"], s["d"], n_gauss=s["n_gauss"], seed=s["seed"],
                                    rel=s["rel"], dtype=s["dtype"]) for s in specs]


def measure_batched(local, steps, warmup, fields=None):
    """fields/s of extremz_correct_batch and of the plain loop on the same
    fields (device-resident inputs, a fresh decompressed copy per step)."""
    import torch
    from extrem_z_b200 import api
    dev = torch.device("cuda", local)
    if fields is None:
        _, fields = mixed_fields()
    F = [torch.from_numpy(x.f).to(dev) for x in fields]
    G0 = [torch.from_numpy(x.decp).to(dev) for x in fields]
    G = [torch.empty_like(g) for g in G0]
    ctx = api.Context(local)
    stream = torch.cuda.current_stream(dev)
    vox = sum(x.f.size for x in fields)

    def reset():
        for g, g0 in zip(G, G0):
            g.copy_(g0)

    def batched():
        reps, launches = ctx.correct_batch([(f, g, x.eb, PARAMS) for f, g, x in zip(F, G, fields)],
                                           stream=stream.cuda_stream)
        return reps, launches

    def loop():
        launches, reps = 0, []
        for f, g, x in zip(F, G, fields):
            r, _ = ctx.correct_device(f, g, x.eb, stream=stream.cuda_stream, **PARAMS)
            launches += r.kernel_launches
            reps.append(r)
        return reps, launches

    def timed(fn):
        total, launches, reps = 0.0, 0, None
        for i in range(warmup + steps):
            reset()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            reps, ln = fn()
            e1.record(stream)
            torch.cuda.synchronize()
            if i >= warmup:
                total += e0.elapsed_time(e1)
                launches += ln
        return total / steps, launches // steps, reps

    ms_b, l_b, reps_b = timed(batched)
    out_b = [g.clone() for g in G]
    ms_p, l_p, reps_p = timed(loop)
    same = all(torch.equal(a, b) for a, b in zip(out_b, G))
    ctx.close()
    return {"fields": len(fields), "voxels": vox,
            "batched": {"fields_per_s": len(fields) / (ms_b * 1e-3), "ms": ms_b,
                        "mvox_per_s": vox / (ms_b * 1e-3) / 1e6, "gpu_launches": l_b},
            "plain_loop": {"fields_per_s": len(fields) / (ms_p * 1e-3), "ms": ms_p,
                           "mvox_per_s": vox / (ms_p * 1e-3) / 1e6, "gpu_launches": l_p},
            "speedup": ms_p / ms_b, "bit_identical_to_plain": bool(same),
            "statuses": sorted({r.status for r in reps_b}),
            "max_outer_iters": max(r.outer_iters for r in reps_b)}


# ---------------------------------------------------------------------------
# Served form: Poisson arrivals into the request loop.
# ---------------------------------------------------------------------------
def serving_requests(n, dev):
    reqs = []
    for i in range(n):
        s = synth.serving_request_spec(i)
        f, g, eb = synth.make_field_device(s["w"], s["h"], s["d"], n_gauss=s["n_gauss"],
                                           seed=s["seed"], rel=s["rel"], dtype=s["dtype"],
                                           device=dev)
        reqs.append((f, g, eb))
    return reqs


def measure_served(local, rates, n_max=96, seconds=3.0, reqs=None):
    """Per rate: p50/p99 latency and served fields/s of a Poisson stream;
    beside them the plain loop's fields/s on the same requests."""
    import torch
    from extrem_z_b200 import api
    dev = torch.device("cuda", local)
    if reqs is None:
        reqs = serving_requests(n_max, dev)
    n_max = len(reqs)
    work = [torch.empty_like(g) for _, g, _ in reqs]
    vox = [f.numel() for f, _, _ in reqs]
    stream = torch.cuda.current_stream(dev)

    # Plain loop: every request alone, one after another (warmed with the
    # largest request, so that its workspace pool has grown).
    ctx = api.Context(local)
    big = max(range(n_max), key=lambda i: vox[i])
    for i in [big] + list(range(min(3, n_max))):
        work[i].copy_(reqs[i][1])
        ctx.correct_device(reqs[i][0], work[i], reqs[i][2], stream=stream.cuda_stream, **PARAMS)
    for (f, g0, eb), w in zip(reqs, work):
        w.copy_(g0)
    torch.cuda.synchronize()
    # Each request alone, timed on its own: the service time that a served
    # request's latency is compared with (its slowdown).
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in reqs]
    for (f, g0, eb), w, (a, b) in zip(reqs, work, evs):
        a.record(stream)
        ctx.correct_device(f, w, eb, stream=stream.cuda_stream, **PARAMS)
        b.record(stream)
    torch.cuda.synchronize()
    alone_ms = np.array([a.elapsed_time(b) for a, b in evs])
    plain_ms = evs[0][0].elapsed_time(evs[-1][1])
    plain_out = [w.clone() for w in work]
    ctx.close()

    sweep = []
    identical = True
    with api.Server(local, reserve_bytes=SERVE_RESERVE_BYTES) as srv:
        # Warm-up burst.
        warm = list(range(min(8, n_max)))
        for i in warm:
            work[i].copy_(reqs[i][1])
        torch.cuda.synchronize()
        for t in [srv.submit(reqs[i][0], work[i], reqs[i][2], stream=stream.cuda_stream,
                             **PARAMS) for i in warm]:
            srv.wait(t)
        for rate in rates:
            n = int(min(n_max, max(24, rate * seconds)))
            for (f, g0, eb), w in zip(reqs[:n], work[:n]):
                w.copy_(g0)
            torch.cuda.synchronize()
            gaps = np.random.default_rng(int(rate)).exponential(1.0 / rate, size=n)
            t_start = time.perf_counter()
            due = t_start
            tickets = []
            for i in range(n):
                due += gaps[i]
                pause = due - time.perf_counter()
                if pause > 0:
                    time.sleep(pause)
                f, _, eb = reqs[i]
                tickets.append(srv.submit(f, work[i], eb, stream=stream.cuda_stream, **PARAMS))
            results = [srv.wait(t) for t in tickets]
            t_end = time.perf_counter()
            lat = np.array([r[1] for r in results])
            identical &= all(torch.equal(work[i], plain_out[i]) for i in range(n))
            span = t_end - t_start
            # Slowdown: latency over the request's own service time alone.  At
            # light load the latency spread is the spread of request sizes
            # (32^3 to 384^3 voxels); the slowdown shows what waiting and
            # sharing the device add.
            slow = lat / np.maximum(alone_ms[:n], 1e-3)
            sweep.append({"rate_req_s": rate, "requests": n,
                          "p50_ms": float(np.percentile(lat, 50)),
                          "p99_ms": float(np.percentile(lat, 99)),
                          "slowdown_p50": float(np.percentile(slow, 50)),
                          "slowdown_p99": float(np.percentile(slow, 99)),
                          "fields_per_s": n / span,
                          "mvox_per_s": sum(vox[:n]) / span / 1e6,
                          # Little's law: time-averaged number of requests in the system.
                          "mean_in_system": float(lat.sum() * 1e-3 / span),
                          "statuses": sorted({r[0].status for r in results})})
        st = srv.stats()
    return {"requests_max": n_max, "voxels_total": int(sum(vox)),
            "alone_ms": {"p50": float(np.percentile(alone_ms, 50)),
                         "p99": float(np.percentile(alone_ms, 99)),
                         "max": float(alone_ms.max())},
            "plain_loop": {"fields_per_s": n_max / (plain_ms * 1e-3),
                           "mvox_per_s": sum(vox) / (plain_ms * 1e-3) / 1e6, "ms": plain_ms},
            "sweep": sweep, "bit_identical_to_plain": bool(identical),
            "peak_running": st["peak_running"], "peak_gb_in_use": st["peak_bytes_in_use"] / 1e9,
            "hbm_budget_gb": 120.0,
            "inputs": "generated on the device (torch CUDA generator seeded per request)"}


def run_form(args, world, rank, local):
    """Lines of the batched (mixed64) and served (serve) workloads.  The
    batch's fields are partitioned across the ranks by voxel count
    (extrem_z_b200.shard, longest first to the least-loaded rank): the value
    is the whole batch over the slowest rank's time.  The served form runs
    replicas and sums over ranks."""
    import torch
    from extrem_z_b200 import shard
    torch.cuda.set_device(local)
    barrier(world)
    if args.workload == "mixed64":
        _, fields = mixed_fields()
        parts = shard.plan([x.f.size for x in fields], world)
        mine = [fields[i] for i in parts[rank]]
        r = measure_batched(local, args.steps, args.warmup, fields=mine) if mine else None
        ms = max_over_ranks(r["batched"]["ms"] if r else 0.0, world)
        value = len(fields) / (ms * 1e-3)
        line = {"metric": "fields/s to zero topological mismatch, batched form", "value": value,
                "unit": "fields/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms, "higher_is_better": True,
                "scaling": "strong" if world > 1 else "weak",
                "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded generator)",
                "config": {"workload": "mixed64", "description": FORM_WORKLOADS["mixed64"],
                           "params": PARAMS,
                           "parallelism": (f"fields sharded x{world} (longest first)"
                                           if world > 1 else "single")},
                "gpu_launches": r["batched"]["gpu_launches"] if r else 0,
                "shard_voxels": shard.loads([x.f.size for x in fields], parts), "batched": r}
    else:
        rates = SERVE_RATES if args.rates is None else tuple(args.rates)
        r = measure_served(local, rates)
        top = max(r["sweep"], key=lambda x: x["fields_per_s"])
        value = max_over_ranks(-top["fields_per_s"], world) * -world
        line = {"metric": "fields/s served (Poisson stream), p50/p99 latency", "value": value,
                "unit": "fields/s", "n_gpus": world, "steps": len(rates), "warmup": 0,
                "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded generator)",
                "config": {"workload": "serve", "description": FORM_WORKLOADS["serve"],
                           "params": PARAMS, "parallelism": f"replicas x{world}"},
                "served": r}
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD,
                    choices=sorted(WORKLOADS) + sorted(FORM_WORKLOADS))
    ap.add_argument("--rates", type=float, nargs="*", default=None,
                    help="serving arrival rates in req/s (serve workload)")
    ap.add_argument("--no-forms", action="store_true",
                    help="omit the batched / served summaries from the plain line")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-edge", type=int, default=CPU_EDGE)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true",
                    help="omit the 256^3 lines measured beside the headline")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        elif args.workload in FORM_WORKLOADS:
            run_form(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
