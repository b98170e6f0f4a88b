"""The allocation-free 2PCF entry point, gr_count_2pcf_noalloc.

Some callers cannot call cudaMalloc: code running inside another framework's
memory pool or under a fixed memory budget, or a plugin that may only use the
buffers its host gives it.  For them the library offers one 2PCF entry point
that takes device pointers for the catalogue and the outputs and keeps every
intermediate array in a fixed device array inside the library.

These tests call it through the C ABI.  Two calls run back to back on the
shared array: a larger catalogue first, then a smaller one with a different
bounding box, bin count and mu binning, so a cell table or histogram left
over from the first call would show in the second.  Each result is checked
against the CPU oracle (integer counts identical, weighted sums within 1e-12
relative) and against the allocating entry point gr_count_2pcf (identical:
both convert the same fixed-point sums with one rounding).  The refusals
(sizes beyond the limits, non-finite inputs, rmax <= rmin) and the empty
catalogue are covered too.  The file is named to run last, so that a run
stopping at the first failure has run every other test already.
"""
import ctypes

import numpy as np
import pytest

from gramsci_b200 import _native, api, catalogs
from oracle import oracle

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _outputs(nbins, nmu, dev):
    import torch

    nbm = nbins * nmu
    return (torch.full((nbm * 4,), -1, dtype=torch.int64, device=dev),
            torch.full((nbm * 4,), np.nan, dtype=torch.float64, device=dev),
            torch.full((nbm,), np.nan, dtype=torch.float64, device=dev),
            torch.full((nbm,), np.nan, dtype=torch.float64, device=dev))


def _call(lib, d_xyz, d_w, n_data, n_rand, rmin, rmax, nbins, nmu, outs):
    counts, catsum, N2, N3 = outs
    return lib.gr_count_2pcf_noalloc(_ptr(d_xyz), _ptr(d_w), n_data, n_rand, rmin, rmax, nbins,
                                     nmu, _ptr(counts), _ptr(catsum), _ptr(N2), _ptr(N3), None)


def _host(outs, nbins, nmu):
    counts, catsum, N2, N3 = (t.cpu().numpy() for t in outs)
    return dict(counts=counts.reshape(4, nmu, nbins).transpose(),
                catsum=catsum.reshape(4, nmu, nbins).transpose(),
                N2=N2.reshape(nmu, nbins).transpose(), N3=N3.reshape(nmu, nbins).transpose())


def test_noalloc_matches_oracle_on_two_calls_with_different_geometry():
    import torch

    dev = torch.device("cuda:0")
    lib = _native.load()
    # a larger clustered catalogue (about 20k points, box 1000, lognormal
    # weights) and then a smaller one in a shifted, smaller box with other bins
    big = catalogs.make("c2_3pcf", scale=0.05, seed=7)
    rng = np.random.default_rng(11)
    ns, nr = 1500, 3000
    small_xyz = np.concatenate([rng.uniform(-250.0, -50.0, (ns, 3)),
                                rng.uniform(-250.0, -50.0, (nr, 3))])
    small_w = rng.lognormal(0.0, 0.5, ns + nr)
    cases = [
        (big.xyz, catalogs.normalise(big.w, big.n_data, big.n_rand), big.n_data, big.n_rand,
         5.0, 25.0, 8, 5),
        (small_xyz, catalogs.normalise(small_w, ns, nr), ns, nr, 2.0, 31.0, 5, 3),
    ]
    assert max(c[2] + c[3] for c in cases) <= _native.GR_NOALLOC_MAX_POINTS
    for call, (xyz, w, nd, nrr, rmin, rmax, nbins, nmu) in enumerate(cases):
        ref = oracle.Graph(xyz, rmin, rmax, nbins, nmu).pcf2(w, nd)
        with api.Context(0) as ctx:
            ctx.set_catalog(xyz, w, nd)
            ctx.set_bins(rmin, rmax, nbins, nmu)
            alloc = ctx.count_2pcf()
        d_xyz = torch.from_numpy(np.ascontiguousarray(xyz)).to(dev)
        d_w = torch.from_numpy(w).to(dev)
        outs = _outputs(nbins, nmu, dev)
        assert _call(lib, d_xyz, d_w, nd, nrr, rmin, rmax, nbins, nmu, outs) == _native.GR_OK
        torch.cuda.synchronize()
        got = _host(outs, nbins, nmu)
        assert int(ref["counts"].sum()) > 0, call
        assert np.array_equal(got["counts"], ref["counts"]), call
        den = np.maximum(np.abs(ref["catsum"]), 1e-300)
        assert np.max(np.abs(got["catsum"] - ref["catsum"]) / den) < RTOL, call
        scale = np.abs(ref["catsum"]).sum(axis=-1)
        assert np.all(np.abs(got["N2"] - ref["N2"]) <= RTOL * scale + 1e-300), call
        assert np.all(np.abs(got["N3"] - ref["N3"]) <= RTOL * np.abs(ref["N3"]) + 1e-300), call
        for k in ("counts", "catsum", "N2", "N3"):
            assert np.array_equal(got[k], alloc[k]), (call, k)


def test_noalloc_empty_catalogue_gives_zeros():
    import torch

    dev = torch.device("cuda:0")
    lib = _native.load()
    d = torch.zeros(3, dtype=torch.float64, device=dev)
    outs = _outputs(4, 2, dev)
    assert _call(lib, d, d, 0, 0, 1.0, 5.0, 4, 2, outs) == _native.GR_OK
    torch.cuda.synchronize()
    got = _host(outs, 4, 2)
    assert np.all(got["counts"] == 0)
    for k in ("catsum", "N2", "N3"):
        assert np.all(got[k] == 0.0), k


def test_noalloc_rejects_bad_inputs_and_sizes_beyond_its_limits():
    import torch

    lib = _native.load()
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(3)
    xyz = rng.uniform(0.0, 100.0, (200, 3))
    w = catalogs.normalise(np.ones(200), 100, 100)
    outs = _outputs(4, 1, dev)
    # a NaN coordinate and an infinite weight are found by the bounds pass
    bad_xyz = xyz.copy()
    bad_xyz[17, 1] = np.nan
    bad_w = w.copy()
    bad_w[150] = np.inf
    for x, ww in ((bad_xyz, w), (xyz, bad_w)):
        d_xyz = torch.from_numpy(x).to(dev)
        d_w = torch.from_numpy(ww).to(dev)
        assert _call(lib, d_xyz, d_w, 100, 100, 1.0, 10.0, 4, 1, outs) == _native.GR_E_ARG
    d_xyz = torch.from_numpy(xyz).to(dev)
    d_w = torch.from_numpy(w).to(dev)
    # rmax <= rmin, negative rmin, bins out of range
    for rmin, rmax, nb, nm in ((5.0, 5.0, 4, 1), (6.0, 5.0, 4, 1), (-1.0, 5.0, 4, 1),
                               (1.0, 5.0, 0, 1), (1.0, 5.0, 4, 128)):
        assert _call(lib, d_xyz, d_w, 100, 100, rmin, rmax, nb, nm, outs) == _native.GR_E_ARG
    # the stated limits
    n = _native.GR_NOALLOC_MAX_POINTS + 1
    big_xyz = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    big_w = torch.ones(n, dtype=torch.float64, device=dev)
    assert _call(lib, big_xyz, big_w, n, 0, 1.0, 2.0, 4, 1, outs) == _native.GR_E_CAPACITY
    assert _call(lib, d_xyz, d_w, 10, 0, 1.0, 2.0, 127, 127, outs) == _native.GR_E_CAPACITY
    # the library still works after the refusals
    outs = _outputs(4, 1, dev)
    assert _call(lib, d_xyz, d_w, 100, 100, 1.0, 10.0, 4, 1, outs) == _native.GR_OK
    torch.cuda.synchronize()
    ref = oracle.Graph(xyz, 1.0, 10.0, 4, 1).pcf2(w, 100)
    assert np.array_equal(_host(outs, 4, 1)["counts"], ref["counts"])
