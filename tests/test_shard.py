"""CPU tests of the slab sharding of one catalogue over several ranks
(gramsci_b200/shard.py): the partition of the roots, the completeness of the
Rmax halos, and that the rooted histograms of the shards (counted with the
oracle, buffer points as in src/gramsci.F90:363, 476, 672) add up to those of
the whole catalogue.  The world-size-2 test runs the all-reduce over gloo
ranks, each counting its shard with the oracle."""
import os
import socket

import numpy as np
import pytest
from scipy.spatial import cKDTree

from gramsci_b200 import catalogs, shard
from oracle import oracle as orc


def _catalogue(name, scale, seed=None):
    cat = catalogs.make(name, scale, seed)
    sp = catalogs.WORKLOADS[name]
    w = catalogs.normalise(cat.w, cat.n_data, cat.n_rand)
    return cat, w, sp


@pytest.mark.parametrize("world", [1, 2, 3, 5])
def test_roots_partition_and_halos_are_complete(world):
    cat, w, sp = _catalogue("c2_3pcf", 0.01)
    rmax = sp["rmax"]
    roots = np.zeros(cat.n, int)
    tree = cKDTree(cat.xyz)
    for r in range(world):
        sx, sw, snd, sb, idx = shard.shard(cat.xyz, w, cat.n_data, r, world, rmax)
        assert np.all(np.diff(idx) > 0)  # catalogue order
        assert np.array_equal(sx, cat.xyz[idx]) and np.array_equal(sw, w[idx])
        assert snd == np.count_nonzero(idx < cat.n_data)
        assert set(np.unique(sb)) <= {0, 1}
        own = idx[sb == 0]
        roots[own] += 1
        # every point closer than rmax to a root of the shard is in the shard
        near = tree.query_ball_point(cat.xyz[own], rmax)
        need = np.unique(np.concatenate([np.asarray(v, int) for v in near])) if len(own) else []
        assert np.isin(need, idx).all()
    assert np.all(roots == 1)


def test_catalogue_buffer_points_stay_buffer():
    cat, w, sp = _catalogue("c1_2pcf", 0.01)
    buf = (np.arange(cat.n) % 7 == 0).astype(np.int32)
    for r in range(3):
        _, _, _, sb, idx = shard.shard(cat.xyz, w, cat.n_data, r, 3, sp["rmax"], buffer=buf)
        assert np.all(sb[buf[idx] == 1] == 1)


def test_slab_edges_and_arguments():
    e = shard.slab_edges(np.arange(100.0), 4)
    assert e[0] == -np.inf and e[-1] == np.inf and np.all(np.diff(e) > 0)
    assert np.array_equal(shard.slab_edges(np.arange(10.0), 1), [-np.inf, np.inf])
    xyz = np.zeros((4, 3))
    xyz[:, 2] = [0, 10, 20, 30]
    assert shard.slab_axis(xyz) == 2
    with pytest.raises(ValueError):
        shard.shard(xyz, np.ones(4), 2, 2, 2, 1.0)
    with pytest.raises(ValueError):
        shard.shard(xyz, np.ones(3), 2, 0, 2, 1.0)
    with pytest.raises(ValueError):
        shard.shard(xyz, np.ones(4), 2, 0, 2, 0.0)
    # an empty catalogue gives empty shards
    sx, sw, snd, sb, idx = shard.shard(np.zeros((0, 3)), np.zeros(0), 0, 1, 2, 5.0)
    assert sx.shape == (0, 3) and snd == 0 and sb.size == 0


def _oracle_counts(kind, xyz, w, n_data, sp, buffer=None):
    g = orc.Graph(xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    return getattr(g, "pcf" + kind[0])(w, n_data, buffer)


def _check_sum(parts, full):
    for k in full:
        tot = sum(p[k] for p in parts)
        if np.issubdtype(np.asarray(full[k]).dtype, np.integer):
            assert np.array_equal(tot, full[k]), k
        else:
            scale = max(np.abs(full[k]).max(), 1e-300)
            assert np.abs(tot - full[k]).max() <= 1e-12 * scale, k


@pytest.mark.parametrize("name,kind,scale,world", [
    ("c1_2pcf", "2pcf", 0.02, 3),
    ("c2_3pcf", "3pcf", 0.01, 4),
    ("c3_4pcf", "4pcf", 0.01, 2),
])
def test_shard_histograms_add_up(name, kind, scale, world):
    cat, w, sp = _catalogue(name, scale)
    full = _oracle_counts(kind, cat.xyz, w, cat.n_data, sp)
    parts = []
    for r in range(world):
        sx, sw, snd, sb, _ = shard.shard(cat.xyz, w, cat.n_data, r, world, sp["rmax"])
        parts.append(_oracle_counts(kind, sx, sw, snd, sp, sb))
    _check_sum(parts, full)


class _OracleCounter:
    """Stands in for a device context in the gloo test: the oracle counts
    the catalogue it was given."""

    def __init__(self, sp):
        self.sp = sp

    def set_catalog(self, xyz, w, n_data, buffer=None):
        self.args = (xyz, w, n_data, buffer)

    def count_3pcf(self):
        xyz, w, n_data, buffer = self.args
        return _oracle_counts("3pcf", xyz, w, n_data, self.sp, buffer)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    cat, w, sp = _catalogue("c2_3pcf", 0.01)
    got = shard.count(_OracleCounter(sp), "3pcf", cat.xyz, w, cat.n_data, rank, world, sp["rmax"])
    out[rank] = {k: np.asarray(v).copy() for k, v in got.items()}
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_allreduce_gloo():
    import torch.multiprocessing as mp

    world = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    cat, w, sp = _catalogue("c2_3pcf", 0.01)
    full = _oracle_counts("3pcf", cat.xyz, w, cat.n_data, sp)
    for r in range(world):
        _check_sum([res[r]], full)
    for k in full:
        assert np.array_equal(res[0][k], res[1][k])
