"""Batched regions (the 5^3-region workload at reduced scale): the 2PCF of all regions in
one graph-replayed launch equals the 2PCF of the whole catalogue and the sum
of the regions run one launch at a time (integer counts bit-exact, weighted
sums within 1e-12), on the density-ramped Neyman-Scott catalogue."""
import numpy as np
import pytest

from gramsci_b200 import catalogs

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def _close(a, b):
    den = np.maximum(np.abs(b), 1e-300)
    d = np.abs(a - b) / den
    d[(a == 0) & (b == 0)] = 0
    return float(d.max())


@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("nsplit", [2, 3])
def test_batched_equals_unsplit_and_region_sum(gpu_ctx, weighted, nsplit):
    cat = catalogs.make("c4_batched", scale=0.004)
    sp = catalogs.WORKLOADS["c4_batched"]
    raw = np.random.default_rng(3).lognormal(0, 0.3, cat.n) if weighted else cat.w
    w = catalogs.normalise(raw, cat.n_data, cat.n_rand)
    gpu_ctx.set_catalog(cat.xyz, w, cat.n_data)
    gpu_ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    whole = gpu_ctx.count_2pcf()
    gpu_ctx.set_regions(nsplit)
    first = gpu_ctx.count_2pcf_batched()   # plans, runs, captures
    again = gpu_ctx.count_2pcf_batched()   # graph replay
    regions = gpu_ctx.regions()
    assert len(regions) == nsplit ** 3
    for b in (first, again):
        assert np.array_equal(b["counts"], whole["counts"])
        assert _close(b["catsum"], whole["catsum"]) < RTOL
    # every point is a root in exactly one region
    roots = np.concatenate([o[bf == 0] for o, bf in regions])
    assert np.array_equal(np.sort(roots), np.arange(cat.n))
    # one launch per region, summed
    tot_c = np.zeros_like(whole["counts"])
    tot_s = np.zeros_like(whole["catsum"])
    for o, bf in regions:
        if len(o) == 0:
            continue
        gpu_ctx.set_catalog(cat.xyz[o], w[o], int(np.sum(o < cat.n_data)), buffer=bf)
        r = gpu_ctx.count_2pcf()
        tot_c += r["counts"]
        tot_s += r["catsum"]
    assert np.array_equal(tot_c, whole["counts"])
    assert _close(tot_s, whole["catsum"]) < 1e-11
    gpu_ctx.set_regions(0)
