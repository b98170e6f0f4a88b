"""Roofline arithmetic of the bench line on the CPU: the peak comes from the
measured-peaks file (or the stated fallback), the algorithmic bytes follow
the per-unit figures of the triangle and 4-clique kernels, achieved / peak
is the reported fraction, and the DRAM traffic is read from the committed
ncu summaries for the full-size workloads only."""
import json
import os

import pytest

from gramsci_b200 import roofline

STATS = {"upper_edges": 1000, "probes": 5000, "tuples": 700, "rooted": 2100, "n_points": 300}


class _Ctx:
    def __init__(self, st):
        self.st = st

    def stats(self):
        return dict(self.st)


def test_peak_is_measured_or_fallback():
    pk = roofline.peaks()
    path = os.path.join(roofline.ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            assert pk == {"hbm_gbs": float(json.load(f)["hbm_gbs"]), "source": "measured"}
    else:
        assert pk == {"hbm_gbs": roofline.FALLBACK_HBM_GBS, "source": "fallback"}


def test_fallback_when_peaks_file_unreadable(tmp_path, monkeypatch):
    monkeypatch.setattr(roofline, "ROOT", str(tmp_path))
    assert roofline.peaks()["source"] == "fallback"
    (tmp_path / "MEASURED_PEAKS.json").write_text("{not json")
    assert roofline.peaks() == {"hbm_gbs": roofline.FALLBACK_HBM_GBS, "source": "fallback"}
    (tmp_path / "MEASURED_PEAKS.json").write_text('{"hbm_gbs": 7000}')
    assert roofline.peaks() == {"hbm_gbs": 7000.0, "source": "measured"}


def test_tri3_bytes_per_unit():
    assert roofline.tri3_bytes(STATS) == 24 * 1000 + 4 * 5000 + 30 * 700
    # linear in every unit
    double = {k: 2 * v for k, v in STATS.items()}
    assert roofline.tri3_bytes(double) == 2 * roofline.tri3_bytes(STATS)


def test_quad4_bytes_per_unit():
    assert roofline.quad4_bytes(STATS, geometric=False) == 24 * 1000 + 8 * 5000 + 17 * 2100
    assert roofline.quad4_bytes(STATS, geometric=True) == 33 * 1000 + 21 * 300


@pytest.mark.parametrize("quad", [False, True])
def test_roofline_fraction(quad):
    pk = {"hbm_gbs": 5000.0, "source": "measured"}
    q_ms = [0.5, 1.5]
    if quad:
        rf = roofline.quad4_roofline(_Ctx(STATS), q_ms, pk, geometric=True)
        b = roofline.quad4_bytes(STATS, True)
        assert rf["kernel"] == "quad4g_kernel"
    else:
        rf = roofline.tri3_roofline(_Ctx(STATS), q_ms, pk)
        b = roofline.tri3_bytes(STATS)
        assert rf["kernel"] == "tri3_kernel"
    assert rf["bound"] == "hbm" and rf["unit"] == "GB/s" and rf["peak"] == 5000.0
    assert rf["ms_per_launch"] == pytest.approx(1.0)
    assert rf["bytes_per_launch"] == b
    assert rf["achieved"] == pytest.approx(b / 1e-3 / 1e9)
    assert rf["frac"] == pytest.approx(rf["achieved"] / 5000.0)
    assert rf["traffic"] is None


@pytest.mark.parametrize("kernel,workload", [("tri3_kernel", "c2"), ("quad4g_kernel", "c3")])
def test_profiled_traffic_from_committed_summary(kernel, workload):
    path = os.path.join(roofline.ROOT, "profiles", f"{kernel}_{workload}.json")
    with open(path) as f:
        d = json.load(f)
    assert "--clock-control none" in d["command"]
    t = roofline.profiled_traffic(kernel, 1.0, workload)
    assert t == float(d["dram_bytes_read"]) + float(d["dram_bytes_write"]) and t > 0
    # the summaries hold full-size captures only
    assert roofline.profiled_traffic(kernel, 0.5, workload) is None
    assert roofline.profiled_traffic(kernel, 1.0, "nonexistent") is None


def test_fp32_binning_roofline():
    from gramsci_b200 import roofline
    # 1e9 binned directed pairs with mu bins in 1 ms on 148 SMs at 1965 MHz
    r = roofline.fp32_binning_roofline(1e9, 10, 1.0, 1965.0, 148)
    assert r["flop_per_binned_pair"] == 27
    assert abs(r["achieved"] - 27.0) < 1e-9
    assert abs(r["peak"] - 148 * 256 * 1.965e9 / 1e12) < 1e-9
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
    assert roofline.fp32_binning_roofline(1e9, 1, 1.0, 1965.0, 148)["flop_per_binned_pair"] == 11
    assert roofline.fp32_binning_roofline(1e9, 1, 1.0, None, 148) is None


def test_mark_binding_names_the_largest_fraction():
    from gramsci_b200 import roofline

    rf = {"bound": "hbm", "frac": 0.25, "issue": {"frac": 0.75}, "atomics": {"frac": 0.16}}
    roofline.mark_binding(rf)
    assert rf["binding"] == "issue" and rf["binding_frac"] == 0.75
    rf = {"kernel": "pair sweep", "fp32": {"frac": 0.07}, "issue": None}
    roofline.mark_binding(rf)
    assert rf["binding"] == "fp32"
    rf = {"bound": "hbm", "frac": 0.9, "issue": {"frac": 0.5}}
    assert roofline.mark_binding(rf)["binding"] == "hbm"
    assert "binding" not in roofline.mark_binding({"kernel": "x", "fp32": None})
