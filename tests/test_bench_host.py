"""Host-side parts of bench.py, on CPU: the dominant kernel's algorithmic
bytes, the parsing of the clock samples that decide whether a run was
throttled, and the reference arm's JSON line."""

import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import bench  # noqa: E402


def test_manifold_round_bytes_are_value_read_plus_two_label_writes():
    n = 512 ** 3
    assert bench.round_bytes(n, 8) == 16 * n
    assert bench.round_bytes(n, 4) == 12 * n


class _Rep:
    """The fields of api.CorrectionReport that the roofline reads."""

    def __init__(self, rounds, reused, ms, launches):
        self.manifold_rounds, self.manifold_reused = rounds, reused
        self.prof_ms, self.prof_launches = ms, launches


def test_roofline_is_the_first_full_round_with_later_rounds_beside_it():
    n, s = 512 ** 3, 8
    ms = {"direction_first": 2.0, "jump_first": 1.2, "direction": 1.5, "jump": 3.5}
    reps = [_Rep(13, 5, ms, {"jump_first": 1}) for _ in range(2)]
    r = bench.manifold_roofline(reps, n, s, step_ms=2 * 34.0, peak=6539.2, peak_kind="measured",
                                traffic=5.47e9)
    # Two corrections, one first round each: 2 x N*(S+8) bytes over 2 x 3.2 ms.
    assert r["launches"] == 2
    assert abs(r["achieved"] - 2 * 16 * n / (6.4e-3) / 1e9) < 1e-6
    assert abs(r["frac"] - r["achieved"] / 6539.2) < 1e-12
    assert r["algorithmic_bytes_per_launch"] == 16 * n and r["traffic"] == 5.47e9
    later = r["later_rounds"]
    assert later["rounds"] == 2 * (13 - 5) - 2 and later["reused"] == 10
    assert abs(later["ms_per_round"] - 10.0 / 14) < 1e-12
    assert abs(r["jump_design_bytes"]["bytes"] - 2 * 26 * n) == 0


def test_jump_design_bytes_of_first_rounds():
    n = 256 ** 3
    # A first round reads pointers and original roots (16 B per voxel) and
    # writes labels, mismatch and changed-input bytes (10 B).
    assert bench.jump_design_bytes(n, 1) == 26 * n
    assert bench.jump_design_bytes(n, 30) == 30 * 26 * n


class _Proc:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0

    def kill(self):
        pass


def _stopped(lines, monkeypatch):
    s = bench.ClockSampler(0)
    s.proc = _Proc()
    s.lines = lines
    monkeypatch.setattr(bench.time, "sleep", lambda _: None)
    return s.stop()


def test_clock_sampler_reports_median_and_active_reasons(monkeypatch):
    c = _stopped(["0, 1965, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, Not Active",
                  "0, 1800, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
                  "0, 1700, 1965, 1000.0, 0x4, Not Active, Not Active, Not Active, Active",
                  "garbled line"], monkeypatch)
    assert c["sm_mhz"] == 1800.0 and c["sm_max_mhz"] == 1965.0
    assert c["reasons"] == ["sw_power_cap"] and c["samples"] == 3


def test_clock_sampler_flags_thermal_slowdown(monkeypatch):
    c = _stopped(["0, 1400, 1965, 900.0, 0x40, Not Active, Active, Not Active, Not Active"],
                 monkeypatch)
    assert c["reasons"] == ["hw_thermal_slowdown"]


def test_clock_sampler_without_nvidia_smi_says_unsampled():
    s = bench.ClockSampler(0)
    assert s.stop()["reasons"] == ["unsampled"]


def test_reference_arm_prints_one_contract_line():
    """`bench.py --impl reference` (the CPU restatement on the host cores, on a
    small crop here) prints one JSON line with the contract's keys."""
    import json
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference",
                          "--workload", "plain256_f64", "--steps", "1", "--warmup", "0",
                          "--cpu-edge", "16"],
                         cwd=root, capture_output=True, text=True, timeout=600, check=True)
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    for key in ("metric", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "scaling",
                "vs_baseline", "dtype", "data", "config"):
        assert key in d
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    # The config names the crop that was timed, and the field it was cut from.
    assert d["config"]["shape_whd"] == [16, 16, 16]
    assert d["config"]["sample_of"] == {"workload": "plain256_f64", "shape_whd": [256, 256, 256]}
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
