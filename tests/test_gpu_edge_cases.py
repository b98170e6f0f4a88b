"""GPU edge cases against the CPU oracle: an empty catalogue, galaxies
without randoms, coincident points, a lattice whose separations and
line-of-sight cosines fall exactly on bin edges and on rmin / rmax (every
such pair goes through the FP64 recheck), and a dense blob whose rows are
longer than the triangle kernel's shared-memory capacity (its global-memory
path).  Integer counts are compared bit-exactly; weighted sums to 1e-12 of
the category sums, as in the other parity tests."""
import numpy as np
import pytest

from gramsci_b200 import api, catalogs

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _close(got, ref):
    a, b = np.asarray(got, np.float64), np.asarray(ref, np.float64)
    return np.all(np.abs(a - b) <= RTOL * np.abs(b) + 1e-300)


def _same(got, ref):
    assert np.array_equal(got["counts"], ref["counts"])
    assert _close(got["catsum"], ref["catsum"])


def test_empty_catalogue():
    with api.Context(0) as ctx:
        ctx.set_catalog(np.zeros((0, 3)), np.zeros(0), 0)
        ctx.set_bins(1.0, 10.0, 4, 2)
        for r in (ctx.count_2pcf(), ctx.count_3pcf(), ctx.count_equi()):
            assert not r["counts"].any() and not r["catsum"].any()
        ctx.set_bins(1.0, 10.0, 2, 1)
        r = ctx.count_4pcf()
        assert not r["counts"].any() and not r["dcount"].any()
        assert ctx.stats()["n_edges"] == 0


def test_galaxies_without_randoms(oracle):
    cat = catalogs.make("c2_3pcf", scale=0.02, seed=3)
    xyz = cat.xyz[:cat.n_data]
    w = catalogs.normalise(cat.w[:cat.n_data], cat.n_data, 0)
    sp = catalogs.WORKLOADS["c2_3pcf"]
    G = oracle.Graph(xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    with api.Context(0) as ctx:
        ctx.set_catalog(xyz, w, cat.n_data)
        ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
        got2, got3 = ctx.count_2pcf(), ctx.count_3pcf()
    ref2, ref3 = G.pcf2(w, cat.n_data), G.pcf3(w, cat.n_data)
    _same(got2, ref2)
    _same(got3, ref3)
    assert ref3["counts"][..., 0].sum() > 0 and not ref3["counts"][..., 1:].any()
    assert not got2["N3"].any() and not got3["N3"].any()


@pytest.mark.parametrize("rmin", [0.0, 2.0])
def test_coincident_points(oracle, rmin):
    rng = np.random.default_rng(11)
    xyz = rng.uniform(0, 60, (3000, 3))
    dup = rng.choice(3000, 300, replace=False)
    xyz = np.vstack([xyz, xyz[dup]])  # 300 points doubled: separation 0
    n_data = 1500
    w = catalogs.normalise(rng.lognormal(0, 0.3, len(xyz)), n_data, len(xyz) - n_data)
    G = oracle.Graph(xyz, rmin, 8.0, 4, 3)
    with api.Context(0) as ctx:
        ctx.set_catalog(xyz, w, n_data)
        ctx.set_bins(rmin, 8.0, 4, 3)
        _same(ctx.count_2pcf(), G.pcf2(w, n_data))
        _same(ctx.count_3pcf(), G.pcf3(w, n_data))


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_lattice_on_bin_edges(oracle, precision):
    # integer lattice: separations sqrt(k) with edges at 1, 2, 3, 4 (rmin, two
    # bin edges, rmax are all attained exactly) and cosines on mu edges
    g = np.arange(12, dtype=np.float64)
    xyz = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3) + 100.0
    n_data = len(xyz) // 2
    w = catalogs.normalise(np.ones(len(xyz)), n_data, len(xyz) - n_data)
    G = oracle.Graph(xyz, 1.0, 4.0, 3, 4)
    rp, col, b, mu = G.csr()
    with api.Context(0) as ctx:
        ctx.set_precision(precision)
        ctx.set_catalog(xyz, w, n_data)
        ctx.set_bins(1.0, 4.0, 3, 4)
        grp, gcol, gb, gmu = ctx.graph()
        assert np.array_equal(grp, rp) and np.array_equal(gcol, col)
        assert np.array_equal(gb, b) and np.array_equal(gmu, mu)
        _same(ctx.count_2pcf(), G.pcf2(w, n_data))
        _same(ctx.count_3pcf(), G.pcf3(w, n_data))
        ctx.set_bins(1.0, 4.0, 3, 1)
        G1 = oracle.Graph(xyz, 1.0, 4.0, 3, 1)
        got, ref = ctx.count_4pcf(), G1.pcf4(w, n_data)
        assert np.array_equal(got["counts"], ref["counts"])
        assert np.array_equal(got["dcount"], ref["dcount"])


def test_rows_longer_than_shared_capacity(oracle):
    # 380 points within a radius of 2 and rmax 5: every point neighbours all
    # others, so upper rows reach 379 entries, past the triangle kernel's
    # 256-entry shared staging
    rng = np.random.default_rng(5)
    v = rng.normal(size=(380, 3))
    xyz = 50.0 + 2.0 * v / np.linalg.norm(v, axis=1, keepdims=True) * rng.uniform(0.2, 1.0, (380, 1))
    n_data = 190
    w = catalogs.normalise(rng.lognormal(0, 0.3, 380), n_data, 190)
    buf = (rng.random(380) < 0.1).astype(np.int32)
    G = oracle.Graph(xyz, 0.5, 5.0, 4, 3)
    with api.Context(0) as ctx:
        ctx.set_catalog(xyz, w, n_data, buffer=buf)
        ctx.set_bins(0.5, 5.0, 4, 3)
        got = ctx.count_3pcf()
        st = ctx.stats()
        ref = G.pcf3(w, n_data, buffer=buf)
    assert st["upper_edges"] > 0 and max(np.diff(G.csr()[0])) > 256
    _same(got, ref)


@pytest.mark.parametrize("what", ["nan_coordinate", "inf_coordinate", "nan_weight", "inf_weight"])
def test_non_finite_inputs_are_refused(what):
    """A non-finite coordinate is refused by the count (the index build tests
    every coordinate); a non-finite weight by gr_set_catalog.  After the
    refusal the context counts a good catalogue as before."""
    from gramsci_b200 import _native, api, catalogs

    rng = np.random.default_rng(8)
    xyz = rng.uniform(0.0, 100.0, (300, 3))
    w = catalogs.normalise(np.ones(300), 150, 150)
    bad_xyz, bad_w = xyz.copy(), w.copy()
    if what == "nan_coordinate":
        bad_xyz[40, 2] = np.nan
    elif what == "inf_coordinate":
        bad_xyz[200, 0] = -np.inf
    elif what == "nan_weight":
        bad_w[10] = np.nan
    else:
        bad_w[250] = np.inf
    with api.Context(0) as ctx:
        ctx.set_bins(1.0, 12.0, 4, 2)
        with pytest.raises(_native.GramsciError) as e:
            ctx.set_catalog(bad_xyz, bad_w, 150)
            ctx.count_2pcf()
        assert e.value.code == _native.GR_E_ARG
        ctx.set_catalog(xyz, w, 150)
        assert int(ctx.count_2pcf()["counts"].sum()) > 0
