"""Host-side pieces of bench.py (no GPU): the clock summary of the timed
region, the measured HBM peak and the committed ncu traffic figure it reads."""

import importlib.util
import json

import pytest

from conftest import REPO


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_module", REPO / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class _Done:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0


def _sampler(bench, lines):
    s = object.__new__(bench.ClockSampler)
    s.proc = _Done()
    s.lines = list(lines)
    return s


def test_clock_summary_takes_the_median_and_active_reasons(bench):
    lines = [
        "1965, 1965, 700.1, Not Active, Not Active, Not Active, Not Active",
        "1800, 1965, 990.0, Not Active, Not Active, Not Active, Active",
        "1965, 1965, 980.2, Not Active, Not Active, Not Active, Not Active",
        "garbage line",
        "[N/A], 1965, 0, Not Active, Not Active, Not Active, Not Active",
    ]
    out = _sampler(bench, lines).stop()
    assert out == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}


def test_clock_summary_is_none_without_samples(bench):
    assert _sampler(bench, []).stop() is None
    s = object.__new__(bench.ClockSampler)
    s.proc = None
    assert s.stop() is None


def test_measured_peak_comes_from_the_measured_file(bench):
    peak, source = bench.measured_peak_hbm()
    path = REPO / "MEASURED_PEAKS.json"
    if path.exists():
        assert source == "measured" and peak == float(json.loads(path.read_text())["hbm_gbs"])
    else:
        assert source == "fallback" and peak == bench.FALLBACK_HBM_GBS


def test_committed_ncu_traffic_figure_is_readable(bench):
    traffic = bench.ncu_traffic_per_vector(fused=True)
    assert traffic is not None and 7e6 < traffic < 2e7  # bytes per vector of one fused iteration
