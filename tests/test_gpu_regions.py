"""Batched regions beyond the subcube split: caller-given region ids
(jackknife regions), independent mocks in one launch, per-region histograms
and the batched 3PCF.

Each is checked against the plain entry points and the oracle on the same
points: integer counts identical, category sums within 1e-12 relative, N2
within 1e-12 of the sum of the absolute category sums.
* Region ids: the batched total equals gr_count_2pcf on the whole
  catalogue; every region's own histogram equals gr_count_2pcf on that
  region's members with their buffer flags (and the oracle, for one region);
  the regions' histograms sum to the total.
* Mocks (overlapping in space, different sizes and normalisations): each
  mock's histogram equals that mock counted alone, so no pair joins two
  mocks; the batched 3PCF is the sum of the mocks' 3PCF.
* Batched 3PCF over a split or region ids equals the unsplit 3PCF.
"""
import numpy as np
import pytest

from gramsci_b200 import api, catalogs

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    d = np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
    d[(a == 0) & (b == 0)] = 0.0
    return float(d.max()) if d.size else 0.0


def _check(got, ref):
    assert np.array_equal(got["counts"], ref["counts"])
    assert _rel(got["catsum"], ref["catsum"]) < RTOL
    scale = np.abs(ref["catsum"]).sum(axis=-1)
    assert np.all(np.abs(got["N2"] - ref["N2"]) <= RTOL * scale + 1e-300)


def _take(d, r):
    return {k: v[..., r] for k, v in d.items()}


def _jackknife_ids(xyz, n_side, seed):
    """Spatially coherent but irregular regions: a jittered n_side^2 grid of
    columns in (x, y), region boundaries moved by up to a third of a column."""
    rng = np.random.default_rng(seed)
    lo, hi = xyz.min(0), xyz.max(0)
    edges = [np.sort(np.concatenate([[lo[d] - 1], np.linspace(lo[d], hi[d], n_side + 1)[1:-1]
                                     + rng.uniform(-1, 1, n_side - 1) * (hi[d] - lo[d]) / (3 * n_side),
                                     [hi[d] + 1]])) for d in range(2)]
    ix = np.searchsorted(edges[0], xyz[:, 0], side="right") - 1
    iy = np.searchsorted(edges[1], xyz[:, 1], side="right") - 1
    return (iy * n_side + ix).astype(np.int32), n_side * n_side


@pytest.mark.parametrize("name,scale,weighted", [("c1_2pcf", 0.3, False), ("c2_3pcf", 0.05, True),
                                                 ("c4_batched", 0.004, False)])
def test_region_ids_2pcf(oracle, name, scale, weighted):
    cat = catalogs.make(name, scale=scale)
    w = catalogs.normalise(cat.w, cat.n_data, cat.n_rand)
    sp = catalogs.WORKLOADS[name]
    ids, nreg = _jackknife_ids(cat.xyz, 3, seed=5)
    with api.Context(0) as ctx:
        ctx.set_catalog(cat.xyz, w, cat.n_data)
        ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
        whole = ctx.count_2pcf()
        ctx.set_region_ids(ids, nreg)
        total = ctx.count_2pcf_batched()
        total2 = ctx.count_2pcf_batched()  # graph replay
        per = ctx.count_2pcf_regions()
        regions = ctx.regions()
    assert len(regions) == nreg
    _check(total, whole)
    for k in total:
        assert np.array_equal(total[k], total2[k]), k
    assert np.array_equal(per["counts"].sum(axis=-1), whole["counts"])
    with api.Context(0) as ctx:
        ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
        for r, (orig, buf) in enumerate(regions):
            # own points of region r are exactly those with id r
            assert np.array_equal(np.sort(orig[buf == 0]), np.nonzero(ids == r)[0])
            nd = int(np.sum(orig < cat.n_data))
            ctx.set_catalog(cat.xyz[orig], w[orig], nd, buffer=buf)
            alone = ctx.count_2pcf()
            _check(_take(per, r), alone)
            if r == 4:
                G = oracle.Graph(cat.xyz[orig], sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
                _check(_take(per, r), G.pcf2(w[orig], nd, buffer=buf))


def _mocks(seed, sizes, box):
    rng = np.random.default_rng(seed)
    xyz, w, nds, nrs = [], [], [], []
    for nd, nr in sizes:
        g = catalogs.neyman_scott(rng, max(1, nd // 10), 10.0, 4.0, 0.0, box)[:nd]
        r = rng.uniform(0.0, box, (nr, 3))
        xyz.append(np.concatenate([g, r]))
        w.append(catalogs.normalise(rng.lognormal(0.0, 0.3, len(g) + nr), len(g), nr))
        nds.append(len(g))
        nrs.append(nr)
    return np.concatenate(xyz), np.concatenate(w), np.array(nds), np.array(nrs)


def test_mocks_2pcf_and_3pcf(oracle):
    box = 300.0
    xyz, w, nds, nrs = _mocks(9, [(3000, 9000), (1500, 6000), (4000, 4000)], box)
    rmin, rmax, nbins, nmu = 5.0, 25.0, 6, 3
    off = np.concatenate([[0], np.cumsum(nds + nrs)])
    with api.Context(0) as ctx:
        ctx.set_catalog(xyz, w, len(xyz))
        ctx.set_bins(rmin, rmax, nbins, nmu)
        ctx.set_mocks(nds, nrs)
        per = ctx.count_2pcf_regions()
        total = ctx.count_2pcf_batched()
        tri = ctx.count_3pcf_batched()
    assert np.array_equal(per["counts"].sum(axis=-1), total["counts"])
    tri_sum = None
    with api.Context(0) as ctx:
        ctx.set_bins(rmin, rmax, nbins, nmu)
        for m in range(len(nds)):
            sl = slice(off[m], off[m + 1])
            ctx.set_catalog(xyz[sl], w[sl], int(nds[m]))
            alone = ctx.count_2pcf()
            _check(_take(per, m), alone)
            t = ctx.count_3pcf()
            tri_sum = t if tri_sum is None else {k: tri_sum[k] + t[k] for k in t}
            if m == 1:
                G = oracle.Graph(xyz[sl], rmin, rmax, nbins, nmu)
                _check(_take(per, m), G.pcf2(w[sl], int(nds[m])))
    assert np.array_equal(tri["counts"], tri_sum["counts"])
    assert _rel(tri["catsum"], tri_sum["catsum"]) < 1e-11


@pytest.mark.parametrize("how", ["split", "ids"])
def test_batched_3pcf_equals_unsplit(oracle, how):
    cat = catalogs.make("c2_3pcf", scale=0.05)
    w = catalogs.normalise(cat.w, cat.n_data, cat.n_rand)
    sp = catalogs.WORKLOADS["c2_3pcf"]
    with api.Context(0) as ctx:
        ctx.set_catalog(cat.xyz, w, cat.n_data)
        ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
        whole = ctx.count_3pcf()
        if how == "split":
            ctx.set_regions(3)
        else:
            ids, nreg = _jackknife_ids(cat.xyz, 3, seed=6)
            ctx.set_region_ids(ids, nreg)
        got = ctx.count_3pcf_batched()
        # a 2PCF batched call after it (layout kept or planned again)
        pairs = ctx.count_2pcf_batched()
        pairs_whole = ctx.count_2pcf()
    _check(got, whole)
    ref = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"]).pcf3(w, cat.n_data)
    _check(got, ref)
    _check(pairs, pairs_whole)
