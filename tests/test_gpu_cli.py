"""End to end through the `gramsci` command: ASCII catalogues in, the
reference's result table out.  The table written by the command (counts from
the GPU) is compared with the table the same writer produces from the CPU
oracle's N2/N3: identical layout and bin columns, values equal to the 7
digits of E14.7 (a last-digit difference is allowed only where the two FP64
sums straddle a rounding boundary of the 7th digit)."""
import pathlib
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
    a = pathlib.Path(a_path).read_text().splitlines()
    b = pathlib.Path(b_path).read_text().splitlines()
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


def _half_unit(v):
    """Half a unit in the 7th significant digit of E14.7 values."""
    v = np.abs(np.asarray(v, np.float64))
    with np.errstate(divide="ignore"):
        e = np.where(v > 0, np.floor(np.log10(np.where(v > 0, v, 1.0))) + 1, 0)
    return np.where(v > 0, 0.5 * 10.0 ** (e - 7), 0.0)


def _table(path):
    return np.array([[float(x) for x in l.split()] for l in pathlib.Path(path).read_text().splitlines()
                     if not l.startswith(" r1")])


@pytest.mark.parametrize("query,nmu,ncol", [("2pcf", 3, 7), ("3pcf", 1, 9), ("equi", 2, 7)])
def test_region_pipeline_equals_unsplit(tmp_path, query, nmu, ncol):
    """gramsci-decompose (2^3 subcubes) -> gramsci -cut j.loadnodes -gcol per
    region -> gramsci-resum gives the unsplit run's table, to the 8 digits
    each region table carries."""
    name = "c2_3pcf"
    cat, w, g, r = _write_cat(tmp_path, name, 0.01)
    sp = catalogs.WORKLOADS[name]
    bins = ["-rmin", repr(sp["rmin"]), "-rmax", repr(sp["rmax"]), "-nbins", str(sp["nbins"]),
            "-nmu", str(nmu)]
    full = tmp_path / "full.out"
    res = subprocess.run([host.CLI_PATH, "-gal", g, "-ran", r, *bins, "-out", str(full), f"-{query}"],
                         capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    res = subprocess.run([host.DECOMPOSE_PATH, repr(sp["rmax"]), "-gal", g, "-ran", r, "-nsplit", "2",
                          "-prefix", str(tmp_path / "reg")], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    parts = []
    for j in range(1, 9):
        out = tmp_path / f"part{j}.out"
        res = subprocess.run([host.CLI_PATH, "-cut", str(tmp_path / f"reg{j}.loadnodes"), "-gcol", *bins,
                              "-out", str(out), f"-{query}"], capture_output=True, text=True)
        assert res.returncode == 0, res.stderr
        parts.append(out)
    total = tmp_path / "total.out"
    res = subprocess.run([host.RESUM_PATH, f"-{query}", "-out", str(total), *map(str, parts)],
                         capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    a, b = _table(total), _table(full)
    assert a.shape == b.shape and a.shape[1] == ncol
    assert np.array_equal(a[:, :ncol - 3], b[:, :ncol - 3])
    # each E14.7 value carries a rounding error of at most half a unit in its
    # 7th digit: the bound is the sum of those over the parts, the total and
    # the unsplit table (FP64 summation-order differences are far smaller)
    cols = slice(ncol - 3, ncol - 1)
    bound = sum(_half_unit(_table(p)[:, cols]) for p in parts)
    bound = bound + _half_unit(a[:, cols]) + _half_unit(b[:, cols])
    err = np.abs(a[:, cols] - b[:, cols])
    assert np.all(err <= 1.01 * bound + 1e-300)
    assert np.abs(b[:, ncol - 3]).max() > 0
