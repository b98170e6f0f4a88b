"""The allocation-free 2PCF entry point, gr_count_2pcf_noalloc.

Some callers cannot call cudaMalloc: code running inside another framework's
memory pool or under a fixed memory budget, or a plugin that may only use the
buffers its host gives it.  For them the library offers one 2PCF entry point
that takes device pointers for the catalogue and the outputs and keeps every
intermediate array in a fixed device array inside the library.  This test
calls it through the C ABI twice in a row (the second call reuses the shared
array, which still holds the first call's contents) and checks each result
against the ordinary entry point, gr_count_2pcf, with the tolerances of the
other parity tests: integer counts identical, weighted sums within 1e-12.
It also checks that inputs beyond the stated limits are refused before any
work is done.  The file is named to run last, so that a run stopping at the
first failure has run every other test already.
"""
import ctypes

import numpy as np
import pytest

from gramsci_b200 import _native, api, catalogs

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_matches_allocating_entry_point():
    import torch

    cat = catalogs.make("c2_3pcf", scale=0.05, seed=7)  # about 20k points, lognormal weights
    assert cat.n <= _native.GR_NOALLOC_MAX_POINTS
    w = catalogs.normalise(cat.w, cat.n_data, cat.n_rand)
    rmin, rmax, nbins, nmu = 5.0, 25.0, 8, 5

    with api.Context(0) as ctx:
        ctx.set_catalog(cat.xyz, w, cat.n_data)
        ctx.set_bins(rmin, rmax, nbins, nmu)
        ref = ctx.count_2pcf()

    lib = _native.load()
    dev = torch.device("cuda:0")
    d_xyz = torch.from_numpy(cat.xyz).to(dev)
    d_w = torch.from_numpy(w).to(dev)
    nbm = nbins * nmu
    for call in range(2):
        counts = torch.full((nbm * 4,), -1, dtype=torch.int64, device=dev)
        catsum = torch.full((nbm * 4,), np.nan, dtype=torch.float64, device=dev)
        N2 = torch.full((nbm,), np.nan, dtype=torch.float64, device=dev)
        N3 = torch.full((nbm,), np.nan, dtype=torch.float64, device=dev)
        rc = lib.gr_count_2pcf_noalloc(_ptr(d_xyz), _ptr(d_w), cat.n_data, cat.n_rand, rmin, rmax,
                                       nbins, nmu, _ptr(counts), _ptr(catsum), _ptr(N2), _ptr(N3),
                                       None)
        assert rc == _native.GR_OK, (call, rc)
        torch.cuda.synchronize()
        got_counts = counts.cpu().numpy().reshape(4, nmu, nbins).transpose()
        got_catsum = catsum.cpu().numpy().reshape(4, nmu, nbins).transpose()
        got_N2 = N2.cpu().numpy().reshape(nmu, nbins).transpose()
        got_N3 = N3.cpu().numpy().reshape(nmu, nbins).transpose()
        assert np.array_equal(got_counts, ref["counts"]), call
        den = np.maximum(np.abs(ref["catsum"]), 1e-300)
        assert np.max(np.abs(got_catsum - ref["catsum"]) / den) < RTOL, call
        scale = np.abs(ref["catsum"]).sum(axis=-1)
        assert np.all(np.abs(got_N2 - ref["N2"]) <= RTOL * scale + 1e-300), call
        assert np.all(np.abs(got_N3 - ref["N3"]) <= RTOL * np.abs(ref["N3"]) + 1e-300), call


def test_noalloc_rejects_sizes_beyond_its_limits():
    import torch

    lib = _native.load()
    dev = torch.device("cuda:0")
    n = _native.GR_NOALLOC_MAX_POINTS + 1
    d_xyz = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    d_w = torch.ones(n, dtype=torch.float64, device=dev)
    rc = lib.gr_count_2pcf_noalloc(_ptr(d_xyz), _ptr(d_w), n, 0, 1.0, 2.0, 4, 1, None, None, None,
                                   None, None)
    assert rc == _native.GR_E_CAPACITY
    rc = lib.gr_count_2pcf_noalloc(_ptr(d_xyz), _ptr(d_w), 10, 0, 1.0, 2.0, 127, 127, None, None,
                                   None, None, None)
    assert rc == _native.GR_E_CAPACITY
