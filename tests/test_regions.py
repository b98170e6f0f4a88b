"""CPU tests of the region-file tools: gramsci-decompose (the reference's
domain_decomposition program, src/domain_decomposition.f90) and
gramsci-resum (the summing step of its example script).

The reference mode is checked against a numpy restatement in single
precision (the reference declares its arrays `real`): per-region bounding
boxes, boxes grown by rmax, strict membership, buffer = 0 inside the region's
own box.  The catalogue mode is checked for its invariants: every point is a
root (buffer 0) in exactly one region, every neighbour of a root closer than
rmax is in that root's file, weights are globally normalised."""
import subprocess

import numpy as np
import pytest

from gramsci_b200 import catalogs, host


def _text(path):
    with open(path) as f:
        return f.read()


def _parse(path):
    rows = [l.split() for l in _text(path).splitlines() if l.strip()]
    if not rows:
        return np.zeros((0, 4)), np.zeros(0, int), np.zeros(0, int)
    v = np.array([[float(x) for x in r[:4]] for r in rows])
    return v, np.array([int(r[4]) for r in rows]), np.array([int(r[5]) for r in rows])


def _reference_regions(x32, w32, gal, region, rmax32):
    """domain_decomposition.f90:38-78 in float32."""
    out = {}
    for j in range(1, int(region.max()) + 1):
        m = region == j
        if m.any():
            lo, hi = x32[m].min(axis=0), x32[m].max(axis=0)
        else:
            big = np.finfo(np.float32).max
            lo, hi = np.full(3, big, np.float32), np.full(3, -big, np.float32)
        lo2 = (lo - rmax32).astype(np.float32)
        hi2 = (hi + rmax32).astype(np.float32)
        inside = np.all((x32 > lo2) & (x32 < hi2), axis=1)
        core = np.all((x32 >= lo) & (x32 <= hi), axis=1)
        out[j] = (np.nonzero(inside)[0], np.where(core[inside], 0, 1))
    return out


def test_decompose_reference_mode(tmp_path):
    rng = np.random.default_rng(3)
    n = 400
    x = rng.uniform(-50, 150, (n, 3))
    w = rng.uniform(0.5, 2.0, n)
    gal = (rng.random(n) < 0.4).astype(int)
    region = rng.integers(1, 6, n)
    region[region == 4] = 5  # region 4 is empty: its file is written, with no points
    lines = []
    for i in range(n):
        lines.append(" ".join(repr(float(v)) for v in (*x[i], w[i])) + f" {gal[i]} 0.0 {region[i]}")
        if i == 17:
            lines.append("1.0 2.0 3.0 oops 1 0.0 2")  # unreadable record: skipped
    (tmp_path / "allpoints").write_text("\n".join(lines) + "\n")
    rmax = 12.5
    nreg = host.decompose(rmax, str(tmp_path) + "/", allpoints=tmp_path / "allpoints")
    assert nreg == 5
    x32, w32 = x.astype(np.float32), w.astype(np.float32)
    ref = _reference_regions(x32, w32, gal, region, np.float32(rmax))
    for j in range(1, 6):
        v, g, b = _parse(tmp_path / f"{j}.loadnodes")
        idx, buf = ref[j]
        assert len(v) == len(idx)
        if j == 4:
            continue
        assert np.array_equal(v[:, :3].astype(np.float32), x32[idx])
        assert np.array_equal(v[:, 3].astype(np.float32), w32[idx])
        assert np.array_equal(g, gal[idx]) and np.array_equal(b, buf)


def test_decompose_catalogue_mode_invariants(tmp_path):
    cat = catalogs.make("c2_3pcf", scale=0.01)
    g, r = tmp_path / "c.gal", tmp_path / "c.ran"
    catalogs.write_ascii(g, cat.xyz[:cat.n_data], cat.w[:cat.n_data])
    catalogs.write_ascii(r, cat.xyz[cat.n_data:], cat.w[cat.n_data:])
    rmax = catalogs.WORKLOADS["c2_3pcf"]["rmax"]
    res = subprocess.run([host.DECOMPOSE_PATH, repr(rmax), "-gal", str(g), "-ran", str(r),
                          "-nsplit", "2", "-prefix", str(tmp_path / "reg")],
                         capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    key = {tuple(p): i for i, p in enumerate(map(tuple, cat.xyz))}
    n = len(key)
    assert n == cat.n
    roots = np.zeros(n, int)
    wsum = np.zeros(2)
    for j in range(1, 9):
        xyz, w, buf, nd, nr = host.read_region_gal(tmp_path / f"reg{j}.loadnodes")
        ids = np.array([key[tuple(p)] for p in xyz])
        assert np.all(ids[:nd] < cat.n_data) and np.all(ids[nd:] >= cat.n_data)
        roots[ids[buf == 0]] += 1
        wsum += [w[:nd][buf[:nd] == 0].sum(), w[nd:][buf[nd:] == 0].sum()]
        # every point within rmax of a root is in the file
        allxyz = cat.xyz
        core = xyz[buf == 0]
        if len(core):
            lo, hi = core.min(axis=0) - rmax, core.max(axis=0) + rmax
            need = np.all((allxyz > lo) & (allxyz < hi), axis=1).sum()
            assert len(xyz) >= need
    assert np.all(roots == 1)
    np.testing.assert_allclose(wsum, [1.0, -1.0], rtol=1e-12)


def test_resum_sums_tables(tmp_path):
    rng = np.random.default_rng(9)
    e = host.radial_bins(1.0, 9.0, 4)
    parts, tot2, tot3 = [], 0, 0
    for k in range(3):
        N2, N3 = rng.uniform(-1, 1, (4, 3)), rng.uniform(0.5, 1, (4, 3))
        p = tmp_path / f"t{k}"
        host.write_2pcf(str(p), e, 4, 3, N2, N3)
        parts.append(p)
        tot2, tot3 = tot2 + N2, tot3 + N3
    out = tmp_path / "sum"
    assert host.resum(2, parts, out) == 0
    lines = _text(out).splitlines()
    assert lines[0] == _text(parts[0]).splitlines()[0]
    v = np.array([[float(x) for x in l.split()] for l in lines[1:]])
    np.testing.assert_allclose(v[:, 4], tot2.ravel(), rtol=3e-7, atol=3e-7)
    np.testing.assert_allclose(v[:, 5], tot3.ravel(), rtol=3e-7)
    np.testing.assert_allclose(v[:, 6], v[:, 4] / v[:, 5], rtol=1e-6)
    # tables with different bins do not sum
    host.write_2pcf(str(tmp_path / "bad"), host.radial_bins(1.0, 10.0, 4), 4, 3, N2, N3)
    assert host.resum(2, [parts[0], tmp_path / "bad"], out) == -3


def test_resum_tetra_disc_column_is_nan(tmp_path):
    e = host.radial_bins(1.0, 9.0, 2)
    p = tmp_path / "t"
    host.write_tetra(str(p), e, 2, 1, np.ones(2), np.ones(2), np.ones((2, 6)), np.ones((2, 6)))
    assert host.resum(6, [p, p], tmp_path / "s") == 0
    v = np.array([[float(x) for x in l.split()] for l in _text(tmp_path / "s").splitlines()])
    assert np.all(v[:, 4] == 2.0) and np.all(np.isnan(v[:, 7]))


def _rows(path, header=True):
    lines = _text(path).splitlines()[1 if header else 0:]
    return np.array([[float(x) for x in l.split()] for l in lines])


@pytest.mark.parametrize("query,nmu", [(3, 1), (3, 3), (4, 1), (5, 2)])
def test_resum_other_tables(tmp_path, query, nmu):
    """gramsci-resum on 3PCF (with and without mu columns), 4PCF and -equi
    tables: header and bin columns copied, N2 and N3 summed from the tables' values,
    the ratio recomputed; the 4PCF disconnected-term columns, ratios of
    sums the tables do not hold, come out NaN."""
    rng = np.random.default_rng(query * 10 + nmu)
    nb = 3
    e = host.radial_bins(1.0, 9.0, nb)
    parts = []
    for k in range(3):
        p = tmp_path / f"t{k}"
        if query == 3:
            nc = nb * (nb + 1) * (nb + 2) // 6
            N2, N3 = rng.uniform(-1, 1, (nc, nmu)), rng.uniform(0.5, 1, (nc, nmu))
            assert host.write_3pcf(str(p), e, nb, nmu, N2, N3) == 0
        elif query == 4:
            nc = nb * (nb + 1) * (nb + 2) * (nb + 3) // 24
            N2, N3 = rng.uniform(-1, 1, (nc, nb, nb)), rng.uniform(0.5, 1, (nc, nb, nb))
            d = rng.uniform(0.5, 1, (nc, nb, nb, 6))
            assert host.write_4pcf(str(p), e, nb, N2, N3, d, d) == 0
        else:
            N2, N3 = rng.uniform(-1, 1, (nb, nmu)), rng.uniform(0.5, 1, (nb, nmu))
            assert host.write_equi(str(p), e, nb, nmu, N2, N3) == 0
        parts.append(p)
    out = tmp_path / "sum"
    assert host.resum(query, parts, out) == 0
    # the -equi table has no header line (gramsci.F90:448-458)
    hdr = query != 5
    rows = [_rows(p, hdr) for p in parts]
    got = _rows(out, hdr)
    if hdr:
        assert _text(out).splitlines()[0] == _text(parts[0]).splitlines()[0]
    # column of N2: after the bin columns (3PCF: 6 edges [+ 2 mu];
    # 4PCF: 8 edges; -equi: 2 edges + 2 mu)
    c = {3: 6 if nmu == 1 else 8, 4: 8, 5: 4}[query]
    assert got.shape == rows[0].shape
    np.testing.assert_array_equal(got[:, :c], rows[0][:, :c])
    tot = sum(r[:, c:c + 2] for r in rows)
    np.testing.assert_allclose(got[:, c:c + 2], tot, rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(got[:, c + 2], got[:, c] / got[:, c + 1], rtol=1e-6)
    if query == 4:
        assert np.all(np.isnan(got[:, c + 3:]))
