"""Host logic of bench.py that needs no GPU: the clock record keeps only the
nvidia-smi samples read inside the timed region, and collects the throttle
reasons that were active there."""

import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


IDLE = "0, 1950, 1965, 300, 0x0, Not Active, Not Active, Not Active, Not Active"
CAPPED = "0, {mhz}, 1965, 990, 0x4, Not Active, Not Active, Not Active, Active"
THERMAL = "0, 1200, 1965, 990, 0x40, Not Active, Active, Not Active, Not Active"


def test_clock_summary_keeps_the_timed_window():
    b = _bench()
    c = b.ClockSampler(0)
    c.lines = [(1.0, IDLE), (2.0, CAPPED.format(mhz=1470)), (2.1, CAPPED.format(mhz=1480)),
               (2.2, "garbage"), (3.5, THERMAL)]
    c.window = [1.5, 3.0]
    s = c.summary()
    assert s == {"sm_mhz": 1475.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 2}


def test_clock_summary_reports_thermal_reasons():
    b = _bench()
    c = b.ClockSampler(0)
    c.lines = [(1.0, THERMAL), (1.1, CAPPED.format(mhz=1500))]
    c.mark_start()
    c.window[0] = 0.0
    c.mark_end()
    s = c.summary()
    assert s["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"] and s["samples"] == 2


def test_clock_summary_without_samples():
    b = _bench()
    c = b.ClockSampler(0)
    c.mark_start()
    c.mark_end()
    assert c.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
