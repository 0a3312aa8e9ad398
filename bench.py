"""Benchmark: ExtreM topology correction, Mvox/s to zero topological mismatch.

One step = one full correction (setup, c_loops, the outer loop to zero
mismatch counters, final join-saddle pass) of a fresh copy of the synthetic
decompressed field, inputs resident in HBM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
                    [--impl ours|reference]

With N > 1 (launched by torch.distributed.run) every rank corrects its own
field of the same workload: the path has no data exchange, so ranks are
replicas and the value is all ranks' voxels over the max-over-ranks time.

--impl reference times the reference algorithm's CPU implementation on the
host cores (the CPU restatement of the reference's GPU correction, built
with OpenMP) on a bounded crop of the same workload, rank 0 only.
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

# name -> (constructor, description); the headline is the 256^3 float64 field.
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
DEFAULT_WORKLOAD = "plain256_f64"
PARAMS = dict(q=4, edit_type=1, thr=0.0, max_outer=1000, max_cloop_rounds=100000,
              final_join=True)

# Dominant kernel and its algorithmic bytes per voxel per launch:
# k_direction reads the decompressed value (S bytes) and writes two int32
# labels (8 bytes) per voxel.
DOMINANT = "direction"


def dominant_bytes_per_launch(n: int, s: int) -> int:
    return n * (s + 8)


# DRAM bytes per voxel per k_direction launch from one ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum over voxels, 256^3 field), by
# value size (profiles/k_direction_256cube_f64.md); None where not captured.
MEASURED_TRAFFIC_PER_VOXEL = {8: (134.239488e6 + 96.382976e6) / 256 ** 3, 4: None}


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
            time.sleep(0.3)
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


def run_reference(args, world, rank):
    if rank != 0:
        return
    field = WORKLOADS[args.workload][0]()
    threads = os.cpu_count() or 1
    edge = args.cpu_edge
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
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * total_s / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dtype_name(field),
            "data": "synthetic", "config": config_of(args, field),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def dtype_name(field):
    return "f64" if field.f.dtype == np.float64 else "f32"


def config_of(args, field):
    d, h, w = field.f.shape
    return {"workload": args.workload, "description": WORKLOADS[args.workload][1],
            "shape_whd": [w, h, d], "eb_abs": field.eb, "params": PARAMS,
            "l2": "inputs larger than L2 (two fields of N*S bytes > 126 MB)" if
            2 * field.f.nbytes > 126e6 else "inputs smaller than L2",
            "parallelism": f"replicas x{args.gpus}" if args.gpus > 1 else "single"}


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

    def step(profile=False):
        g.copy_(g0)
        rep, _ = ctx.correct_device(f, g, field.eb, stream=stream.cuda_stream,
                                    profile=[DOMINANT] if profile else False, **PARAMS)
        return rep

    for _ in range(args.warmup):
        rep = step()
    torch.cuda.synchronize()
    if rep.status != 0:
        raise RuntimeError(f"correction did not converge: {rep}")

    # Timed region: device time of exactly K steps, max over ranks.
    sampler = ClockSampler(local) if rank == 0 or True else None
    sampler.start()
    barrier(world)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    reps = []
    for _ in range(args.steps):
        reps.append(step(profile=True))
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms, world)
    value = world * n * args.steps / (ms_max * 1e-3) / 1e6
    launches = sum(r.kernel_launches for r in reps)

    # Roofline of the dominant kernel from its CUDA-event time in the timed steps.
    dom_ms = sum(r.prof_ms[DOMINANT] for r in reps)
    dom_n = sum(r.prof_launches[DOMINANT] for r in reps)
    peak, peak_kind = measured_peaks()
    per_launch = dominant_bytes_per_launch(n, s)
    achieved = per_launch * dom_n / (dom_ms * 1e-3) / 1e9 if dom_ms > 0 else 0.0
    tpv = MEASURED_TRAFFIC_PER_VOXEL.get(s)
    roofline = {"bound": "hbm", "kernel": "k_direction", "achieved": achieved, "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                "traffic": (tpv * n) if tpv else None,
                "algorithmic_bytes_per_launch": per_launch, "launches": dom_n,
                "kernel_ms": dom_ms, "share_of_step": dom_ms / ms if ms else None}

    # End to end through the host-buffer entry point: H2D of both fields from
    # pinned memory, correction, D2H of the corrected field, every step.
    hf = torch.from_numpy(field.f).pin_memory().numpy()
    hg0 = field.decp
    hg = torch.empty(field.decp.shape, dtype=tdt).pin_memory().numpy()
    np.copyto(hg, hg0)
    ctx.correct_host(hf, hg, field.eb, stream=stream.cuda_stream, **PARAMS)
    e2e_s = 0.0
    e2e_steps = max(1, min(args.steps, 5))
    barrier(world)
    for _ in range(e2e_steps):
        np.copyto(hg, hg0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.correct_host(hf, hg, field.eb, stream=stream.cuda_stream, **PARAMS)
        e2e_s += time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, world)
    e2e = {"value": world * n * e2e_steps / e2e_s / 1e6, "unit": UNIT,
           "h2d_bytes_per_step": 2 * n * s, "d2h_bytes_per_step": n * s,
           "entry_point": "extremz_correct_host"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = 1
        secs, vox, crep = time_oracle(field, args.cpu_edge, threads)
        cpu = {"value": vox / secs / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"leading {args.cpu_edge}^3 crop of the same field and bound, full "
                         f"correction to zero mismatch ({secs:.1f} s, status {crep['status']})"}

    if rank == 0:
        r0 = reps[-1]
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": dtype_name(field), "data": "synthetic (seeded generator, no dataset)",
                "config": config_of(args, field), "e2e": e2e, "gpu_launches": launches,
                "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
                "rounds": {"outer_iters": r0.outer_iters, "cloop_rounds": r0.cloop_rounds,
                           "manifold_rounds": r0.manifold_rounds, "status": r0.status,
                           "counters": r0.counters}}
        print(json.dumps(line), flush=True)
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-edge", type=int, default=96)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
