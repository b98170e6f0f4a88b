"""End to end through the `gramsci` driver: ASCII catalogues in, the
reference's result table out.  The table written by the driver (counts from
the GPU) is compared with the table the same writer produces from the CPU
oracle's N2/N3: identical layout and bin columns, values equal to the 7
digits of E14.7 (a last-digit difference is allowed only where the two FP64
sums straddle a rounding boundary of the 7th digit)."""
import subprocess

import numpy as np
import pytest

from gramsci_b200 import catalogs, host

pytestmark = pytest.mark.gpu


def _write_cat(tmp_path, name, scale):
    cat = catalogs.make(name, scale=scale)
    g, r = tmp_path / "cat.gal", tmp_path / "cat.ran"
    catalogs.write_ascii(g, cat.xyz[:cat.n_data], cat.w[:cat.n_data])
    catalogs.write_ascii(r, cat.xyz[cat.n_data:], cat.w[cat.n_data:])
    w = catalogs.normalise(cat.w, cat.n_data, cat.n_rand)
    return cat, w, str(g), str(r)


def _compare(a_path, b_path):
    a = open(a_path).read().splitlines()
    b = open(b_path).read().splitlines()
    assert len(a) == len(b)
    if a and a[0].startswith(" r1"):  # header line (2/3/4PCF tables)
        assert a[0] == b[0]
        a, b = a[1:], b[1:]
    for la, lb in zip(a, b):
        assert len(la) == len(lb)
        va = np.array([float(x) for x in la.split()])
        vb = np.array([float(x) for x in lb.split()])
        same = (va == vb) | (np.isnan(va) & np.isnan(vb))
        with np.errstate(invalid="ignore"):
            close = np.abs(va - vb) <= 1.5e-7 * np.maximum(np.abs(va), np.abs(vb))
        assert np.all(same | close), (la, lb)


@pytest.mark.parametrize("query,name,scale,nmu", [("2pcf", "c1_2pcf", 0.05, 1),
                                                   ("2pcf", "c2_3pcf", 0.01, 5),
                                                   ("3pcf", "c2_3pcf", 0.01, 5),
                                                   ("3pcf", "c2_3pcf", 0.01, 1),
                                                   ("4pcf", "c3_4pcf", 0.03, 1),
                                                   ("equi", "c2_3pcf", 0.01, 3),
                                                   ("tetra", "c3_4pcf", 0.03, 2)])
def test_cli_matches_oracle_table(tmp_path, oracle, query, name, scale, nmu):
    cat, w, g, r = _write_cat(tmp_path, name, scale)
    sp = catalogs.WORKLOADS[name]
    out = tmp_path / "gpu.out"
    cmd = [host.CLI_PATH, "-gal", g, "-ran", r, "-rmin", repr(sp["rmin"]), "-rmax", repr(sp["rmax"]),
           "-nbins", str(sp["nbins"]), "-nmu", str(nmu), "-out", str(out), f"-{query}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    G = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], nmu)
    e = host.radial_bins(sp["rmin"], sp["rmax"], sp["nbins"])
    ref = tmp_path / "oracle.out"
    if query == "2pcf":
        o = G.pcf2(w, cat.n_data)
        host.write_2pcf(str(ref), e, sp["nbins"], nmu, o["N2"], o["N3"])
    elif query == "3pcf":
        o = G.pcf3(w, cat.n_data)
        host.write_3pcf(str(ref), e, sp["nbins"], nmu, o["N2"], o["N3"])
    elif query == "4pcf":
        o = G.pcf4(w, cat.n_data)
        host.write_4pcf(str(ref), e, sp["nbins"], o["N2"], o["N3"], o["discN"], o["discR"])
    elif query == "equi":
        o = G.equi(w, cat.n_data)
        host.write_equi(str(ref), e, sp["nbins"], nmu, o["N2"], o["N3"])
    else:
        o = G.tetra(w, cat.n_data)
        host.write_tetra(str(ref), e, sp["nbins"], nmu, o["N2"], o["N3"], o["discN"], o["discR"])
    _compare(str(out), str(ref))
