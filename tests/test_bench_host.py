"""Host-side parts of bench.py that decide whether a bench line is accepted,
checked without a GPU: the clock sampler's parsing of nvidia-smi samples and
its behaviour where neither nvidia-smi nor NVML answers."""
import shutil
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def test_clock_samples_and_throttle_reasons_are_parsed():
    c = bench.ClockSampler(0)
    c.parse("1965, 1965, 0x0000000000000000\n"
            "1800, 1965, 0x0000000000000004\n"     # sw_power_cap
            "[N/A], 1965, 0x0\n"                    # skipped
            "1372, 1965, 0x0000000000000048\n")     # hw_slowdown + hw_thermal_slowdown
    c.source = "test"
    s = c.summary()
    assert s["samples"] == 3 and s["sm_mhz"] == 1800.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_power_cap"]


@pytest.mark.skipif(shutil.which("nvidia-smi") is not None, reason="a GPU machine: the sampler has a source")
def test_sampler_without_a_gpu_reports_no_samples():
    with bench.ClockSampler(0) as k:
        pass
    s = k.summary()
    assert s["samples"] == 0 and s["sm_mhz"] is None and s["reasons"] == []
