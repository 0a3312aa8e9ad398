"""Host-side arithmetic of bench.py, on CPU: the dominant kernel's algorithmic
bytes and the parsing of the clock samples that decide whether a run was
throttled."""

import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import bench  # noqa: E402


def test_dominant_bytes_first_round_full_later_rounds_lower_bound():
    n = 256 ** 3
    # One correction: the first computed round reads 24 B and writes 10 B per
    # voxel; later rounds read 24 B and write the changed-input byte.
    assert bench.dominant_bytes(n, 1, 1) == 34 * n
    assert bench.dominant_bytes(n, 13, 1) == 34 * n + 12 * 25 * n
    # Thirty corrections of twelve computed rounds each.
    assert bench.dominant_bytes(n, 360, 30) == 30 * 34 * n + 330 * 25 * n


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
