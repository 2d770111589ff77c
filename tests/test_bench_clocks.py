"""bench.py's clock record, from NVML samples taken on a thread (no GPU: the samples are planted).

The record must cover the timed region: only samples inside [mark_start, mark_end] count, a
timed region shorter than the poll period falls back to the samples within 50 ms of it (and
says so), and the throttle bits map to the reason names a run is judged by.
"""
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

import bench  # noqa: E402


class _FakeNvml:
    def nvmlShutdown(self):
        pass


class _Done:
    def join(self, timeout=None):
        pass


def _sampler(samples, t0, t1):
    s = object.__new__(bench.NvmlClockSampler)
    s.nv, s.th, s.run = _FakeNvml(), _Done(), False
    s.max_mhz = 1965
    s.samples = samples
    s.t0, s.t1 = t0, t1
    return s


def test_only_samples_inside_the_timed_region_count():
    S = bench.NvmlClockSampler
    samples = [(0.90, 900, 0), (1.00, 1965, 0), (1.05, 1950, S.SW_POWER), (1.10, 1965, 0), (1.30, 600, S.HW)]
    rec = _sampler(samples, 0.99, 1.11).stop()
    assert rec["samples"] == 3 and rec["sm_mhz"] == 1965.0 and rec["sm_max_mhz"] == 1965.0
    assert rec["reasons"] == ["sw_power_cap"] and rec["window"] == "timed region"


def test_a_short_region_between_two_polls_takes_the_nearest_samples():
    S = bench.NvmlClockSampler
    samples = [(0.50, 700, S.HW_THERMAL), (0.98, 1965, 0), (1.04, 1950, S.SW_THERMAL)]
    rec = _sampler(samples, 1.00, 1.02).stop()  # 20 ms, no sample inside
    assert rec["samples"] == 2 and rec["window"] == "timed region +- 50 ms"
    assert rec["reasons"] == ["sw_thermal_slowdown"]  # the sample 0.5 s away does not count
    assert _sampler([(0.50, 700, 0)], 1.00, 1.02).stop() is None  # nothing near: no record
