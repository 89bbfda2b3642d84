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


def test_cpu_chi_schedule():
    b = _bench()
    for n in (1, 4, 5, 20, 100):
        s = b.cpu_chi_schedule(n)
        assert len(s) == n
        assert s.count(2048) == 1
        if n >= 4:
            assert set(s) == {256, 512, 1024, 2048}
    assert b.cpu_chi_schedule(20, n_top=2).count(2048) == 2


def test_batch_rate_weights_by_chi_counts():
    b = _bench()
    tm = {"seconds": {256: [1.0, 3.0, 2.0], 2048: [10.0]}, "flops": {256: 1e12, 2048: 8e12}}
    rate, per = b.batch_rate(tm, {256: 3, 2048: 1})
    # 3 x 1 TFLOP in 3 x 2 s (median) + 8 TFLOP in 10 s
    assert abs(rate - 11.0 / 16.0) < 1e-12
    assert per[256]["s_per_matvec"] == 2.0 and per[2048]["timed"] == 1


def test_reference_arm_never_loads_the_library():
    """The CPU arm builds its structures and FLOP counts without importing
    the package: no tenax_b200 module and no libtenax_b200.so in the
    process after a chi=256 problem is built and one oracle matvec runs."""
    import subprocess
    import sys

    code = (
        "import sys, importlib.util\n"
        f"sys.path.insert(0, {ROOT!r})\n"
        f"spec = importlib.util.spec_from_file_location('b', {os.path.join(ROOT, 'bench.py')!r})\n"
        "b = importlib.util.module_from_spec(spec); spec.loader.exec_module(b)\n"
        "hp = b.HostProblems(1)\n"
        "tm = b.time_cpu_schedule(hp, [256], warmup=0)\n"
        "assert tm['flops'][256] > 0\n"
        "assert not [m for m in sys.modules if m.startswith('tenax_b200')], 'package imported'\n"
        "maps = open('/proc/self/maps').read()\n"
        "assert 'libtenax_b200' not in maps, 'library mapped'\n"
        "print('OK')\n"
    )
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "OK" in r.stdout, r.stderr[-2000:]


def test_sector_histogram_key():
    """The autotuner's cache key: power-of-two buckets of the bond sector
    sizes of theta's outer legs, and the MPO bond dimension."""
    import types

    import numpy as np

    from tenax_b200.autotune import sector_histogram

    def leg(counts):
        return types.SimpleNamespace(charges=np.repeat(np.arange(len(counts)), counts))

    p = types.SimpleNamespace(theta=types.SimpleNamespace(indices=(leg([4, 200, 5]), None, None, leg([1, 64]))),
                              Wl=types.SimpleNamespace(indices=(types.SimpleNamespace(charges=np.zeros(26)),)))
    hist, dws = sector_histogram([p])
    assert dict(hist) == {2: 1, 8: 1, 3: 1, 0: 1, 6: 1} and dws == (26,)


def test_dram_view_of_the_dominant_kernel():
    """roofline.dram: measured DRAM bytes per launch over the stage time,
    against the HBM copy bandwidth; absent without a traffic figure."""
    b = _bench()
    v = b._dram_view(7374000000, 2.264, {"hbm_gbs": 6650.0}, "fallback")
    assert v["unit"] == "GB/s" and v["peak"] == 6650.0
    assert abs(v["achieved"] - 7374000000 / 2.264e-3 / 1e9) < 0.1
    assert abs(v["frac"] - v["achieved"] / 6650.0) < 1e-4
    assert b._dram_view(None, 2.264, {"hbm_gbs": 6650.0}, "fallback") is None
    assert b._dram_view(7374000000, 2.264, {}, "measured") is None


def test_autotune_key_names_the_library_build():
    """A schedule tuned on one build of the kernels is not reused by another:
    the cache key carries a hash of the loaded library."""
    import json
    import types

    import numpy as np

    from tenax_b200 import autotune

    leg = types.SimpleNamespace(charges=np.repeat(np.arange(3), [4, 9, 2]))
    p = types.SimpleNamespace(theta=types.SimpleNamespace(indices=(leg, None, None, leg)),
                              Wl=types.SimpleNamespace(indices=(types.SimpleNamespace(charges=np.zeros(5)),)))
    key = json.loads(autotune.cache_key([p], "bf16x3"))
    assert len(key["library"]) == 16 and key["library"] == autotune.library_id()
    assert key["schedules"] == list(autotune.SCHEDULE_SET) and key["dw"] == [5]
