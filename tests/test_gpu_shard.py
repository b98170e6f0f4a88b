"""Slab shards of one catalogue counted one after the other on one GPU
(gramsci_b200/shard.py without the all-reduce): the shards' histograms,
each counted through the C ABI with its halo points flagged as buffer
points, add up to one call on the whole catalogue (integer counts
identical, sums within 1e-12 relative) and to the oracle.  This is the
split a multi-GPU run of one catalogue makes, one shard per rank."""
import numpy as np
import pytest

from gramsci_b200 import catalogs, shard

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _close(got, ref, key):
    got, ref = np.asarray(got), np.asarray(ref)
    if np.issubdtype(ref.dtype, np.integer):
        assert np.array_equal(got, ref), key
    else:
        scale = max(float(np.abs(ref).max()), 1e-300)
        assert float(np.abs(got - ref).max()) <= RTOL * scale, key


@pytest.mark.parametrize("name,scale,world", [
    ("c1_2pcf", 0.1, 3),
    ("c2_3pcf", 0.05, 4),
    ("c3_4pcf", 0.05, 2),
])
def test_shards_add_up_to_the_catalogue(gpu_ctx, oracle, name, scale, world):
    cat = catalogs.make(name, scale)
    sp = catalogs.WORKLOADS[name]
    kind = sp["query"]
    w = catalogs.normalise(cat.w, cat.n_data, cat.n_rand)
    ctx = gpu_ctx
    ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    ctx.set_catalog(cat.xyz, w, cat.n_data)
    full = getattr(ctx, "count_" + kind)()
    total = None
    for r in range(world):
        sx, sw, snd, sb, _ = shard.shard(cat.xyz, w, cat.n_data, r, world, sp["rmax"])
        ctx.set_catalog(sx, sw, snd, buffer=sb)
        part = getattr(ctx, "count_" + kind)()
        total = part if total is None else {k: total[k] + part[k] for k in total}
    for k in full:
        _close(total[k], full[k], k)
    g = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    ref = getattr(g, "pcf" + kind[0])(w, cat.n_data)
    for k in ref:
        _close(total[k], ref[k], k)
