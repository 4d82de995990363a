"""The algorithmic-byte model behind the V-cycle roofline entry of bench.py, counted by
hand on small hierarchies (no GPU)."""
import importlib.util
import os

import pytest

_spec = importlib.util.spec_from_file_location("bench", os.path.join(os.path.dirname(__file__), "..", "bench.py"))
bench = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(bench)


def test_two_levels_dense_coarsest():
    # fine 1000 cells, coarse 100 rows solved by the dense inverse, P with 1500 entries
    sizes = [(1000, 5800, 0), (100, 900, 1500)]
    fine = 20 * 1000 + 40 * 1000 + 2 * 40 * 1000 + 4 * 1000            # first, 1 pre, 2 post, FP64 out
    res = 40 * 1000
    restrict = 4 * 100 + 8 * 1500 + 4 * 1000 + 4 * 100
    prolong = 4 * 1000 + 8 * 1500 + 4 * 100 + 8 * 1000
    dense = 8 * 100 * 100 + 8 * 100
    assert bench.vcycle_bytes(sizes, 2, 128) == pytest.approx(fine + res + restrict + prolong + dense)


def test_three_levels_smoothed_coarsest():
    # coarsest too large for the dense inverse: it is smoothed like the middle level
    sizes = [(1000, 5800, 0), (200, 2000, 1500), (150, 1500, 400)]
    coarse_max = 100
    fine = 20 * 1000 + 40 * 1000 + 2 * 40 * 1000 + 4 * 1000
    t01 = 40 * 1000 + (4 * 200 + 8 * 1500 + 4 * 1000 + 4 * 200) + (4 * 1000 + 8 * 1500 + 4 * 200 + 8 * 1000)
    sw1 = 20 * 200 + 6 * 2000
    mid = 12 * 200 + 3 * sw1
    t12 = sw1 + (4 * 150 + 8 * 400 + 4 * 200 + 4 * 150) + (4 * 200 + 8 * 400 + 4 * 150 + 8 * 200)
    sw2 = 20 * 150 + 6 * 1500
    last = 12 * 150 + 3 * sw2
    assert bench.vcycle_bytes(sizes, 2, coarse_max) == pytest.approx(fine + t01 + mid + t12 + last)


def test_no_sweeps():
    sizes = [(1000, 5800, 0), (100, 900, 1500)]
    got = bench.vcycle_bytes(sizes, 0, 128)
    fine = 16 * 1000 + 12 * 1000
    res = 40 * 1000
    restrict = 4 * 100 + 8 * 1500 + 4 * 1000 + 4 * 100
    prolong = 4 * 1000 + 8 * 1500 + 4 * 100 + 8 * 1000
    assert got == pytest.approx(fine + res + restrict + prolong + 8 * 100 * 100 + 8 * 100)


def test_clock_summary_from_samples():
    """The clocks key of the bench line: median SM clock, highest max clock and every
    throttle reason seen Active in any sample (nvidia-smi csv, noheader, nounits)."""
    cs = bench.ClockSampler()
    assert cs.summary()["reasons"] == ["unsampled"]
    cs.samples = [["1965", "1965", "700.1", "Not Active", "Not Active", "Not Active", "Not Active"],
                  ["1950", "1965", "980.0", "Not Active", "Not Active", "Not Active", "Active"],
                  ["1980", "1965", "990.5", "Not Active", "Not Active", "Not Active", "Active"],
                  ["[N/A]", "1965", "[N/A]", "Not Active", "Active", "Not Active", "Not Active"]]
    s = cs.summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0 and s["samples"] == 4
    assert s["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]


def test_load_peaks(tmp_path):
    import json
    assert bench.load_peaks(str(tmp_path / "absent.json"))[2] == "fallback"
    p = tmp_path / "peaks.json"
    p.write_text(json.dumps({"hbm_gbs": 6543.7, "bf16_tflops": 1642.7, "bf16_tflops_sustained": 1400.0}))
    assert bench.load_peaks(str(p)) == (6543.7, 1642.7, "measured")
    p.write_text(json.dumps({"hbm_gbs": {"value": 6500.0}, "bf16_tflops": {"value": 1600.0}}))
    assert bench.load_peaks(str(p)) == (6500.0, 1600.0, "measured")
    p.write_text("{not json")
    hbm, tc, src = bench.load_peaks(str(p))
    assert (hbm, tc) == (6650.0, 1590.0) and src.startswith("fallback")
