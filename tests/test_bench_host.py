"""Host logic of bench.py that needs no GPU: the clock sampler keeps only the
samples read inside the timed window, and reports throttle reasons and the
median SM clock from them."""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import bench  # noqa: E402


class _Proc:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0

    def kill(self):
        pass


class _Thread:
    def join(self, timeout=None):
        pass


def sampler(lines):
    s = bench.ClockSampler(0)
    s.proc, s.t = _Proc(), _Thread()
    s.lines = lines
    return s


def row(sm, reasons=("Not Active",) * 4, active="0x0"):
    return "0, %d, 1965, 700.5, %s, %s" % (sm, active, ", ".join(reasons))


def test_window_drops_samples_outside_the_timed_region():
    s = sampler([(1.0, row(900)), (2.0, row(1965)), (2.1, row(1965)), (9.0, row(300))])
    s.window(1.9, 2.5)
    c = s.stop()
    assert c["sm_mhz"] == 1965.0 and c["sm_max_mhz"] == 1965.0
    assert c["samples"] == 2 and c["reasons"] == []


def test_throttle_reasons_inside_the_window_are_reported():
    hot = ("Not Active", "Active", "Not Active", "Active")
    s = sampler([(2.0, row(1500, hot, "0x24")), (5.0, row(1965))])
    s.window(1.5, 2.5)
    c = s.stop()
    assert "hw_thermal_slowdown" in c["reasons"] and "sw_power_cap" in c["reasons"]
    assert c["sm_mhz"] == 1500.0


def test_no_sample_in_the_window_falls_back_to_the_last_one():
    s = sampler([(1.0, row(1800)), (1.2, row(1965))])
    s.window(3.0, 3.1)
    c = s.stop()
    assert c["sm_mhz"] == 1965.0 and c["samples"] == 1
