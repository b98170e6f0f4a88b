"""bench.py's clock record on the CPU: the nvidia-smi samples taken inside
the timed region are summarised as the median SM clock, the maximum clock
and the throttle reasons that were active; samples outside the region are
left out unless none fall inside it; malformed lines are skipped; without
nvidia-smi the record says so."""
import bench

MAX = "1965"


def _line(sm, hw="Not Active", thermal="Not Active", sw_thermal="Not Active", cap="Not Active"):
    return f"0, {sm}, {MAX}, 700.00, 0x0000000000000000, {hw}, {thermal}, {sw_thermal}, {cap}"


class _Proc:
    def __init__(self):
        self.terminated = False

    def terminate(self):
        self.terminated = True

    def wait(self, timeout=None):
        return 0

    def kill(self):
        pass


def _sampler(lines):
    s = bench.ClockSampler(0)
    s.proc = _Proc()
    s.lines = list(lines)
    return s


def test_region_samples_only():
    s = _sampler([(0.5, _line(900, hw="Active")),
                  (1.0, _line(1965)), (1.1, _line(1950)), (1.2, _line(1900, cap="Active")),
                  (3.0, _line(800, thermal="Active"))])
    r = s.stop(1.0, 1.2)
    assert s.proc.terminated
    assert r["sm_mhz"] == 1950.0 and r["sm_max_mhz"] == 1965.0 and r["samples"] == 3
    assert r["reasons"] == ["sw_power_cap"] and r["window"] == "timed region"


def test_all_reasons_and_hex_flags():
    s = _sampler([(1.0, _line(1200, hw="Active", thermal="0x1", sw_thermal="1", cap="Active"))])
    r = s.stop()
    assert r["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_power_cap",
                            "sw_thermal_slowdown"]


def test_short_region_uses_whole_run():
    s = _sampler([(0.0, _line(1965)), (5.0, _line(1960))])
    r = s.stop(1.0, 1.001)
    assert r["samples"] == 2 and r["sm_mhz"] == 1962.5
    assert r["window"].startswith("whole run")


def test_malformed_lines_skipped():
    s = _sampler([(1.0, "[N/A]"), (1.0, "0, [N/A], 1965, 1, 0, a, b, c, d"), (1.0, _line(1800))])
    r = s.stop()
    assert r["samples"] == 1 and r["sm_mhz"] == 1800.0 and r["reasons"] == []


def test_no_nvidia_smi():
    s = bench.ClockSampler(0)
    r = s.stop()
    assert r["sm_mhz"] is None and r["reasons"] == ["nvidia-smi unavailable"]
