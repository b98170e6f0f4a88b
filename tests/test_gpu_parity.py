"""GPU parity: the CUDA library (through its C ABI) against the CPU oracle.

Integer work is compared bit-exactly: the graph edge set with its bins, and
the rooted pair / triangle / 4-clique counts per bin and category.  Weighted
sums are FP64 on both sides but summed in different orders; each category
sum has a single sign, so they are compared with a relative tolerance of
1e-12.  N2 mixes signs (DD - 2DR + RR), so it is compared against the sum of
absolute category sums: |N2_gpu - N2_oracle| <= 1e-12 * sum_c |catsum_c|.
"""
import numpy as np
import pytest

from gramsci_b200 import catalogs

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    den = np.maximum(np.abs(b), 1e-300)
    d = np.abs(a - b) / den
    d[(a == 0) & (b == 0)] = 0.0
    return float(d.max()) if d.size else 0.0


def _check_sums(got, ref, ncat_axis=-1):
    assert np.array_equal(got["counts"], ref["counts"])
    assert _rel(got["catsum"], ref["catsum"]) < RTOL
    scale = np.abs(ref["catsum"]).sum(axis=ncat_axis)
    assert np.all(np.abs(got["N2"] - ref["N2"]) <= RTOL * scale + 1e-300)


def _cat(name, scale, seed=None):
    cat = catalogs.make(name, scale=scale, seed=seed)
    w = catalogs.normalise(cat.w, cat.n_data, cat.n_rand)
    return cat, w, catalogs.WORKLOADS[name]


@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("name,scale", [("c1_2pcf", 0.05), ("c2_3pcf", 0.01), ("c3_4pcf", 0.05)])
def test_graph_edges_equal(gpu_ctx, oracle, name, scale, precision):
    cat, w, sp = _cat(name, scale)
    gpu_ctx.set_precision(precision)
    gpu_ctx.set_catalog(cat.xyz, w, cat.n_data)
    gpu_ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    rp, col, b, mu = gpu_ctx.graph()
    G = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    orp, ocol, ob, omu = G.csr()
    assert np.array_equal(rp, orp)
    assert np.array_equal(col, ocol)
    assert np.array_equal(b, ob)
    assert np.array_equal(mu, omu)
    gpu_ctx.set_precision("f32")


@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("name,scale,nmu", [("c1_2pcf", 0.1, 1), ("c1_2pcf", 0.1, 7),
                                            ("c5_adjoint_2pcf", 0.003, 4)])
def test_2pcf(gpu_ctx, oracle, name, scale, nmu, precision):
    cat, w, sp = _cat(name, scale)
    gpu_ctx.set_precision(precision)
    gpu_ctx.set_catalog(cat.xyz, w, cat.n_data)
    gpu_ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], nmu)
    got = gpu_ctx.count_2pcf()
    ref = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], nmu).pcf2(w, cat.n_data)
    _check_sums(got, ref)
    assert np.all(np.abs(got["N3"] - ref["N3"]) <= RTOL * np.abs(ref["N3"]) + 1e-300)
    gpu_ctx.set_precision("f32")


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_3pcf_c2(gpu_ctx, oracle, precision):
    cat, w, sp = _cat("c2_3pcf", 0.02)
    gpu_ctx.set_precision(precision)
    gpu_ctx.set_catalog(cat.xyz, w, cat.n_data)
    gpu_ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    got = gpu_ctx.count_3pcf()
    ref = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"]).pcf3(w, cat.n_data)
    _check_sums(got, ref)
    st = gpu_ctx.stats()
    assert st["rooted"] == int(ref["counts"].sum())
    gpu_ctx.set_precision("f32")


@pytest.mark.parametrize("name,scale,nmu,precision", [
    ("c2_3pcf", 0.02, 1, "f32"),          # geometric third-edge test (no mu bins)
    ("c2_3pcf", 0.02, 1, "f64"),
    ("c2_3pcf", 0.02, 5, "f32"),          # hash probes (mu bins, short rows)
    ("c5_adjoint_3pcf", 0.002, 5, "f32"),  # geometric with mu bins (long rows)
    ("c5_adjoint_3pcf", 0.002, 5, "f64")])
def test_3pcf_third_edge_modes(gpu_ctx, oracle, name, scale, nmu, precision):
    """Both ways of finding the third edge of a triangle (a hash probe of the
    rows, or the graph's membership test on the pair) give the oracle's
    counts and sums."""
    cat, w, sp = _cat(name, scale)
    gpu_ctx.set_precision(precision)
    gpu_ctx.set_catalog(cat.xyz, w, cat.n_data)
    gpu_ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], nmu)
    got = gpu_ctx.count_3pcf()
    ref = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], nmu).pcf3(w, cat.n_data)
    _check_sums(got, ref)
    assert gpu_ctx.stats()["rooted"] == int(ref["counts"].sum()) > 0
    gpu_ctx.set_precision("f32")


@pytest.mark.parametrize("mode", ["hash", "geometric"])
@pytest.mark.parametrize("query", ["3pcf", "equi", "4pcf", "4pcf_weighted", "tetra"])
def test_clique_modes(gpu_ctx, oracle, query, mode):
    """Both ways of finding the edges among a root's neighbours, forced,
    against the oracle (buffer points included)."""
    if query.startswith("4pcf") or query == "tetra":
        cat, w, sp = _cat("c3_4pcf", 0.05)
    else:
        cat, w, sp = _cat("c2_3pcf", 0.02)
    rng = np.random.default_rng(17)
    if query == "4pcf_weighted":
        w = catalogs.normalise(rng.lognormal(0, 0.3, cat.n), cat.n_data, cat.n_rand)
    buf = (rng.random(cat.n) < 0.1).astype(np.int32)
    gpu_ctx.set_clique_mode(mode)
    try:
        gpu_ctx.set_catalog(cat.xyz, w, cat.n_data, buffer=buf)
        gpu_ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
        G = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
        if query == "3pcf":
            got, ref = gpu_ctx.count_3pcf(), G.pcf3(w, cat.n_data, buffer=buf)
        elif query == "equi":
            got, ref = gpu_ctx.count_equi(), G.equi(w, cat.n_data, buffer=buf)
        elif query == "tetra":
            got, ref = gpu_ctx.count_tetra(), G.tetra(w, cat.n_data, buffer=buf)
        else:
            got, ref = gpu_ctx.count_4pcf(), G.pcf4(w, cat.n_data, buffer=buf)
        assert int(ref["counts"].sum()) > 0
        assert np.array_equal(got["counts"], ref["counts"])
        assert _rel(got["catsum"], ref["catsum"]) < RTOL
        for k in ("dcount",):
            if k in ref:
                assert np.array_equal(got[k], ref[k])
        if "dsum" in ref:
            assert _rel(got["dsum"], ref["dsum"]) < RTOL
    finally:
        gpu_ctx.set_clique_mode("auto")


def test_3pcf_unit_weights(gpu_ctx, oracle):
    cat, w, sp = _cat("c5_adjoint_3pcf", 0.002)
    w = catalogs.normalise(np.ones(cat.n), cat.n_data, cat.n_rand)
    gpu_ctx.set_catalog(cat.xyz, w, cat.n_data)
    gpu_ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    got = gpu_ctx.count_3pcf()
    ref = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"]).pcf3(w, cat.n_data)
    _check_sums(got, ref)


def test_4pcf_c3(gpu_ctx, oracle):
    cat, w, sp = _cat("c3_4pcf", 0.1)
    gpu_ctx.set_catalog(cat.xyz, w, cat.n_data)
    gpu_ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    got = gpu_ctx.count_4pcf()
    ref = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"]).pcf4(w, cat.n_data)
    assert np.array_equal(got["counts"], ref["counts"])
    assert np.array_equal(got["dcount"], ref["dcount"])
    assert _rel(got["catsum"], ref["catsum"]) < RTOL
    assert _rel(got["dsum"], ref["dsum"]) < RTOL
    assert _rel(got["discR"], ref["discR"]) < RTOL


def test_4pcf_weighted_buffer(gpu_ctx, oracle):
    cat, w, sp = _cat("c3_4pcf", 0.05)
    rng = np.random.default_rng(11)
    w = catalogs.normalise(rng.lognormal(0, 0.3, cat.n), cat.n_data, cat.n_rand)
    buf = (rng.random(cat.n) < 0.2).astype(np.int32)
    gpu_ctx.set_catalog(cat.xyz, w, cat.n_data, buffer=buf)
    gpu_ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    got = gpu_ctx.count_4pcf()
    ref = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"]).pcf4(
        w, cat.n_data, buffer=buf)
    assert np.array_equal(got["counts"], ref["counts"])
    assert np.array_equal(got["dcount"], ref["dcount"])
    assert _rel(got["catsum"], ref["catsum"]) < RTOL
    assert _rel(got["dsum"], ref["dsum"]) < RTOL


@pytest.mark.parametrize("query", ["2pcf", "3pcf"])
def test_buffer_points(gpu_ctx, oracle, query):
    cat, w, sp = _cat("c2_3pcf", 0.01)
    buf = (np.random.default_rng(5).random(cat.n) < 0.3).astype(np.int32)
    gpu_ctx.set_catalog(cat.xyz, w, cat.n_data, buffer=buf)
    gpu_ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    G = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    if query == "2pcf":
        got, ref = gpu_ctx.count_2pcf(), G.pcf2(w, cat.n_data, buffer=buf)
    else:
        got, ref = gpu_ctx.count_3pcf(), G.pcf3(w, cat.n_data, buffer=buf)
    _check_sums(got, ref)


@pytest.mark.parametrize("name,scale,nmu,weighted", [("c1_2pcf", 0.1, 3, True),
                                                      ("c4_batched", 0.003, 10, False),
                                                      ("c5_adjoint_2pcf", 0.002, 4, True)])
def test_pair_sweep_variants_agree(gpu_ctx, oracle, name, scale, nmu, weighted):
    """Every pair-sweep variant the autotuner can pick gives the oracle's
    counts (sparse and dense cells)."""
    cat, w, sp = _cat(name, scale)
    if weighted:
        w = catalogs.normalise(np.random.default_rng(1).lognormal(0, 0.3, cat.n), cat.n_data,
                               cat.n_rand)
    gpu_ctx.set_catalog(cat.xyz, w, cat.n_data)
    gpu_ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], nmu)
    ref = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], nmu).pcf2(w, cat.n_data)
    try:
        # 0-5 on cells at least rmax wide, 6 the tile sweep on them, 7 the
        # tile sweep on cells of rmax/2
        for v in range(8):
            gpu_ctx.set_autotune(v)
            _check_sums(gpu_ctx.count_2pcf(), ref)
    finally:
        gpu_ctx.set_autotune("on")


@pytest.mark.parametrize("variant", [6, 7])
@pytest.mark.parametrize("case", ["buffers_mu", "coincident_rmin0", "far_origin_weighted"])
def test_tile_sweep_edge_cases(gpu_ctx, oracle, variant, case):
    """The tile sweeps (lanes over roots, packed FP32x2 membership tests,
    approximate square roots inside the guard band) against the oracle on
    dense cells: buffer points with line-of-sight bins, coincident points
    with rmin = 0 (zero separations), and a catalogue far from the origin
    with lognormal weights (large coordinates widen the guard band)."""
    rng = np.random.default_rng(70 + variant)
    n = 6000
    nd = 2000
    if case == "far_origin_weighted":
        xyz = 1500.0 + rng.normal(0.0, 40.0, (n, 3))
    else:
        xyz = rng.normal(0.0, 25.0, (n, 3)) + np.array([300.0, -200.0, 100.0])
    if case == "coincident_rmin0":
        xyz[100:140] = xyz[100]          # 40 copies of one point
        xyz[3000:3010] = xyz[2999]
    w = catalogs.normalise(np.ones(n) if case != "far_origin_weighted"
                           else rng.lognormal(0.0, 0.5, n), nd, n - nd)
    buf = (rng.random(n) < 0.3).astype(np.int32) if case == "buffers_mu" else None
    rmin = 0.0 if case == "coincident_rmin0" else 2.0
    nmu = 7 if case == "buffers_mu" else 1
    gpu_ctx.set_catalog(xyz, w, nd, buffer=buf)
    gpu_ctx.set_bins(rmin, 20.0, 9, nmu)
    ref = oracle.Graph(xyz, rmin, 20.0, 9, nmu).pcf2(w, nd, buffer=buf)
    assert int(ref["counts"].sum()) > 100_000
    try:
        gpu_ctx.set_autotune(variant)
        _check_sums(gpu_ctx.count_2pcf(), ref)
    finally:
        gpu_ctx.set_autotune("on")


@pytest.mark.parametrize("nmu", [1, 3])
def test_equi(gpu_ctx, oracle, nmu):
    cat, w, sp = _cat("c2_3pcf", 0.02)
    gpu_ctx.set_catalog(cat.xyz, w, cat.n_data)
    gpu_ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], nmu)
    got = gpu_ctx.count_equi()
    ref = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], nmu).equi(w, cat.n_data)
    assert ref["counts"].sum() > 0
    _check_sums(got, ref)
    assert np.all(np.abs(got["N3"] - ref["N3"]) <= RTOL * np.abs(ref["N3"]) + 1e-300)


@pytest.mark.parametrize("weighted", [False, True])
def test_tetra(gpu_ctx, oracle, weighted):
    cat, w, sp = _cat("c3_4pcf", 0.1)
    if weighted:
        w = catalogs.normalise(np.random.default_rng(4).lognormal(0, 0.3, cat.n), cat.n_data,
                               cat.n_rand)
    buf = (np.random.default_rng(6).random(cat.n) < 0.1).astype(np.int32)
    gpu_ctx.set_catalog(cat.xyz, w, cat.n_data, buffer=buf)
    gpu_ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], 1)
    got = gpu_ctx.count_tetra()
    ref = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], 1).tetra(w, cat.n_data, buffer=buf)
    assert ref["counts"].sum() > 0
    assert np.array_equal(got["counts"], ref["counts"])
    assert np.array_equal(got["dcount"], ref["dcount"])
    assert _rel(got["catsum"], ref["catsum"]) < RTOL
    assert _rel(got["dsum"], ref["dsum"]) < RTOL


@pytest.mark.parametrize("query", ["graph", "2pcf", "3pcf", "4pcf"])
def test_log_bins(gpu_ctx, oracle, query):
    """-log bins: the library's FP64 path (log10 on the device, glibc's on
    the oracle side).  Both are within an ulp, so a bin could differ only for
    a separation within ~1e-15 relative of a bin edge; at these sizes the
    expected number of such edges is far below one, and the test is exact."""
    cat, w, sp = _cat("c2_3pcf", 0.01)
    rmin = 0.1 * sp["rmax"]
    gpu_ctx.set_catalog(cat.xyz, w, cat.n_data)
    gpu_ctx.set_bins(rmin, sp["rmax"], sp["nbins"], sp["nmu"], logbins=True)
    G = oracle.Graph(cat.xyz, rmin, sp["rmax"], sp["nbins"], sp["nmu"], logbins=True)
    if query == "graph":
        got, ref = gpu_ctx.graph(), G.csr()
        for a, b in zip(got, ref):
            assert np.array_equal(a, b)
        assert len(np.unique(got[2])) == sp["nbins"]
    elif query == "2pcf":
        _check_sums(gpu_ctx.count_2pcf(), G.pcf2(w, cat.n_data))
    elif query == "3pcf":
        _check_sums(gpu_ctx.count_3pcf(), G.pcf3(w, cat.n_data))
    else:
        # both 4-clique kernels (the geometric one bins its inner edges from
        # the positions, here in FP64 with log10)
        G4 = oracle.Graph(cat.xyz, rmin, sp["rmax"], 4, 1, logbins=True)
        gpu_ctx.set_bins(rmin, sp["rmax"], 4, 1, logbins=True)
        ref = G4.pcf4(w, cat.n_data)
        for mode in ("geometric", "hash"):
            gpu_ctx.set_clique_mode(mode)
            try:
                got = gpu_ctx.count_4pcf()
            finally:
                gpu_ctx.set_clique_mode("auto")
            assert int(ref["counts"].sum()) > 0
            assert np.array_equal(got["counts"], ref["counts"])
            assert np.array_equal(got["dcount"], ref["dcount"])
            assert _rel(got["catsum"], ref["catsum"]) < RTOL


def test_3pcf_without_counts_and_skewed_weights(gpu_ctx, oracle):
    """counts=False gives the same sums (the integer counts are not the
    reference's output); few galaxies against many randoms (weights 30x
    apart) keep 1e-12 because each random-count category has its own
    fixed-point scale."""
    cat, _, sp = _cat("c2_3pcf", 0.02)
    keep = np.ones(cat.n, bool)
    keep[:cat.n_data] = np.random.default_rng(8).random(cat.n_data) < 0.1
    xyz = cat.xyz[keep]
    nd = int(keep[:cat.n_data].sum())
    w = catalogs.normalise(np.random.default_rng(9).lognormal(0, 0.5, len(xyz)), nd, len(xyz) - nd)
    gpu_ctx.set_catalog(xyz, w, nd)
    gpu_ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    full = gpu_ctx.count_3pcf()
    lean = gpu_ctx.count_3pcf(counts=False)
    assert "counts" not in lean
    assert np.array_equal(full["catsum"], lean["catsum"])
    assert np.array_equal(full["N2"], lean["N2"]) and np.array_equal(full["N3"], lean["N3"])
    ref = oracle.Graph(xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"]).pcf3(w, nd)
    _check_sums(full, ref)


def test_4pcf_weighted_sums_without_counts(gpu_ctx):
    """Weighted 4PCF sums are the same whether or not the integer counts
    (not part of the reference's output) are kept."""
    cat, _, sp = _cat("c3_4pcf", 0.05)
    w = catalogs.normalise(np.random.default_rng(4).lognormal(0, 0.3, cat.n), cat.n_data,
                           cat.n_rand)
    gpu_ctx.set_catalog(cat.xyz, w, cat.n_data)
    gpu_ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    full = gpu_ctx.count_4pcf()
    lean = gpu_ctx.count_4pcf(counts=False)
    assert "counts" not in lean and int(full["counts"].sum()) > 0
    for k in ("N2", "N3", "discN", "discR", "catsum", "dsum"):
        assert np.array_equal(full[k], lean[k]), k
