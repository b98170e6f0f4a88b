"""GPU parity at the configured sizes.

The other GPU parity tests shrink the catalogues (same density, smaller box),
so their coordinates stay small.  The FP32 guard band scales with the largest
coordinate (its bound is proportional to max|x| 2^-24), so these tests run
the workloads at full size, where coordinates reach 1000-2000 Mpc/h, and
compare the CUDA library with the CPU oracle on the same inputs:

* the plain 2PCF (70,000 points) and the clustered 3PCF with line-of-sight
  bins (400,000 points), in full;
* the 4PCF on the dense clustered set (120,000 points), unit and lognormal
  weights, with the disconnected pair terms, and its two 4-clique kernels
  (hash probes and the geometric pair test, heaviest roots split over
  several work items) giving identical results and gradients;
* four seeded regions of the batched catalogue (12M points, 125 regions with
  60 Mpc/h buffers), each region's members counted alone, and the per-region
  counts of all 125 regions summed against the one-launch batched count;
* the weight adjoints of the 1M + 2M point catalogue at 64 seeded weights:
  each gradient entry against central finite differences and against the
  oracle's gradient, both evaluated on the neighbourhood of that point (all
  pairs and triangles containing point k lie within rmax of it, so their
  sums, and with them the exact finite difference and gradient of entry k,
  do not depend on points farther away).

Tolerances as in the other parity tests: integer counts identical, category
sums within 1e-12 relative, N2 within 1e-12 of the sum of the absolute
category sums; gradients within 1e-12 of the largest gradient of the
oracle's, and within 1e-8 relative of the finite differences.
"""
import numpy as np
import pytest

from gramsci_b200 import api, catalogs

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _cat(name, seed=None):
    cat = catalogs.make(name, scale=1.0, seed=seed)
    w = catalogs.normalise(cat.w, cat.n_data, cat.n_rand)
    return cat, w, catalogs.WORKLOADS[name]


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    d = np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
    d[(a == 0) & (b == 0)] = 0.0
    return float(d.max()) if d.size else 0.0


def _check(got, ref, sums=("catsum",)):
    assert np.array_equal(got["counts"], ref["counts"])
    for k in sums:
        assert _rel(got[k], ref[k]) < RTOL, k
    scale = np.abs(ref["catsum"]).sum(axis=-1)
    assert np.all(np.abs(got["N2"] - ref["N2"]) <= RTOL * scale + 1e-300)


def test_full_c1_2pcf(oracle):
    cat, w, sp = _cat("c1_2pcf")
    with api.Context(0) as ctx:
        ctx.set_catalog(cat.xyz, w, cat.n_data)
        ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
        got = ctx.count_2pcf()
    ref = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"]).pcf2(w, cat.n_data)
    assert int(ref["counts"].sum()) > 1_000_000
    _check(got, ref)


def test_full_c2_3pcf(oracle):
    cat, w, sp = _cat("c2_3pcf")
    assert np.abs(cat.xyz).max() > 990.0
    with api.Context(0) as ctx:
        ctx.set_catalog(cat.xyz, w, cat.n_data)
        ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
        got = ctx.count_3pcf()
        st = ctx.stats()
    G = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    assert st["n_edges"] == G.nedges
    ref = G.pcf3(w, cat.n_data)
    assert int(ref["counts"].sum()) > 80_000_000
    _check(got, ref)


@pytest.mark.parametrize("weights", ["unit", "lognormal"])
def test_full_c3_4pcf(oracle, weights):
    cat, w, sp = _cat("c3_4pcf")
    if weights == "lognormal":
        rng = np.random.default_rng(33)
        w = catalogs.normalise(rng.lognormal(0.0, 0.3, cat.n), cat.n_data, cat.n_rand)
    with api.Context(0) as ctx:
        ctx.set_catalog(cat.xyz, w, cat.n_data)
        ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
        got = ctx.count_4pcf()
    ref = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"]).pcf4(w, cat.n_data)
    assert int(ref["counts"].sum()) > 50_000_000
    _check(got, ref, sums=("catsum", "dsum"))
    assert np.array_equal(got["dcount"], ref["dcount"])


def test_full_c4_region_subset(oracle):
    """Four seeded regions of the full batched catalogue against the oracle,
    and every region counted alone summing to the one-launch batched count."""
    import torch

    cat, w, sp = _cat("c4_batched")
    dev = torch.device("cuda:0")
    xyz_d = torch.from_numpy(cat.xyz).to(dev)
    w_d = torch.from_numpy(w).to(dev)
    with api.Context(0) as ctx:
        ctx.set_catalog(xyz_d, w_d, cat.n_data)
        ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
        ctx.set_regions(sp["nsplit"])
        batched = ctx.count_2pcf_batched()
        regions = ctx.regions()
    assert len(regions) == sp["nsplit"] ** 3
    pick = np.random.default_rng(44).choice(len(regions), size=4, replace=False)
    total = np.zeros_like(batched["counts"])
    with api.Context(0) as ctx:
        ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
        for r, (orig, buf) in enumerate(regions):
            oi = torch.from_numpy(orig.astype(np.int64)).to(dev)
            nd = int(np.sum(orig < cat.n_data))
            ctx.set_catalog(xyz_d[oi].contiguous(), w_d[oi].contiguous(), nd,
                            buffer=torch.from_numpy(buf).to(dev))
            got = ctx.count_2pcf()
            total += got["counts"]
            if r in pick:
                G = oracle.Graph(cat.xyz[orig], sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
                ref = G.pcf2(w[orig], nd, buffer=buf)
                del G
                assert int(ref["counts"].sum()) > 10_000_000, r
                assert np.abs(cat.xyz[orig]).max() > 300.0
                _check(got, ref)
    assert np.array_equal(total, batched["counts"])


@pytest.mark.parametrize("order", [2, 3])
def test_full_c5_gradients_local(oracle, order):
    import torch

    from gramsci_b200 import autograd

    name = "c5_adjoint_2pcf" if order == 2 else "c5_adjoint_3pcf"
    cat, w, sp = _cat(name)
    bins = (sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    rng = np.random.default_rng(55 + order)
    xyz_d = torch.from_numpy(cat.xyz).cuda()
    wt = torch.from_numpy(w).cuda().requires_grad_(True)
    fn = autograd.pcf2 if order == 2 else autograd.pcf3
    N2, N3 = fn(wt, xyz_d, cat.n_data, *bins)
    c2 = rng.normal(size=tuple(N2.shape))
    c3 = rng.normal(size=tuple(N3.shape))
    loss = (torch.from_numpy(c2).cuda() * N2).sum() + (torch.from_numpy(c3).cuda() * N3).sum()
    loss.backward()
    grad = wt.grad.cpu().numpy()
    assert np.all(np.isfinite(grad))
    gmax = float(np.max(np.abs(grad)))
    assert gmax > 0.0
    # 64 seeded weights: galaxies and randoms
    ks = np.concatenate([rng.choice(cat.n_data, 32, replace=False),
                         cat.n_data + rng.choice(cat.n_rand, 32, replace=False)])
    reach = sp["rmax"] * 1.01
    with api.Context(0) as ctx:
        for k in ks:
            # the neighbourhood of k, in catalogue order (galaxies first)
            sel = np.nonzero(np.max(np.abs(cat.xyz - cat.xyz[k]), axis=1) < reach)[0]
            sel = sel[np.sum((cat.xyz[sel] - cat.xyz[k]) ** 2, axis=1) < reach * reach]
            kl = int(np.searchsorted(sel, k))
            assert sel[kl] == k
            xs, ws = cat.xyz[sel], w[sel].copy()
            nd = int(np.sum(sel < cat.n_data))
            # oracle gradient entry of k on the neighbourhood
            G = oracle.Graph(xs, *bins)
            adj = G.adjoint2 if order == 2 else G.adjoint3
            g_orc = adj(ws, nd, c2, c3)[kl]
            # central finite difference on the GPU (multilinear: exact up to rounding)
            h = abs(ws[kl])
            loss_pm = []
            for sgn in (1.0, -1.0):
                wp = ws.copy()
                wp[kl] += sgn * h
                ctx.set_catalog(xs, wp, nd)
                ctx.set_bins(*bins)
                r = ctx.count_2pcf() if order == 2 else ctx.count_3pcf()
                loss_pm.append(float(np.sum(c2 * r["N2"]) + np.sum(c3 * r["N3"])))
            fd = (loss_pm[0] - loss_pm[1]) / (2 * h)
            # the 128-bit fixed-point gradients quantise every term at one
            # scale for the whole catalogue: their error bound is relative to
            # the largest gradient, as in the other adjoint tests
            assert abs(grad[k] - g_orc) <= RTOL * gmax, (k, grad[k], g_orc)
            assert abs(grad[k] - fd) <= 1e-8 * max(abs(fd), 1e-300), (k, grad[k], fd)


def test_full_c3_clique_modes_identical():
    """The hash-probe and the geometric 4-clique kernels at full size, where
    the roots are taken longest row first and the heaviest rows are split
    over several work items: identical counts, sums and weight gradients,
    unit and lognormal weights."""
    cat, w, sp = _cat("c3_4pcf")
    rng = np.random.default_rng(34)
    wl = catalogs.normalise(rng.lognormal(0.0, 0.3, cat.n), cat.n_data, cat.n_rand)
    out, grads = {}, {}
    with api.Context(0) as ctx:
        ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
        for wname, ww in (("unit", w), ("lognormal", wl)):
            ctx.set_catalog(cat.xyz, ww, cat.n_data)
            for mode in ("hash", "geometric"):
                ctx.set_clique_mode(mode)
                r = ctx.count_4pcf()
                out[(wname, mode)] = r
                if wname == "lognormal":
                    cot = [np.random.default_rng(35).normal(size=r[k].shape)
                           for k in ("N2", "N3", "discN", "discR")]
                    grads[mode] = ctx.adjoint_4pcf(*cot)
    for wname in ("unit", "lognormal"):
        a, b = out[(wname, "hash")], out[(wname, "geometric")]
        assert set(a) == set(b)
        for k in a:
            assert np.array_equal(a[k], b[k]), (wname, k)
    assert int(out[("unit", "geometric")]["counts"].sum()) > 50_000_000
    assert np.array_equal(grads["hash"], grads["geometric"])
