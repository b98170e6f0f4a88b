"""GPU tests of graph persistence and reuse: gr_graph_save / gr_graph_load
(the build-once, query-many "graph database") and GR_OPT_KEEP_GRAPH.

A loaded graph must give the same counts as a fresh build (and as the
oracle); any mismatch between the file and the context (bins, coordinates,
damaged bytes) is refused on the host before anything reaches the device."""
import pathlib

import numpy as np
import pytest

from gramsci_b200 import api, catalogs
from gramsci_b200._native import GramsciError

pytestmark = pytest.mark.gpu


def _setup(ctx, name, scale, nmu=None, seed=None):
    cat = catalogs.make(name, scale=scale, seed=seed)
    w = catalogs.normalise(cat.w, cat.n_data, cat.n_rand)
    sp = catalogs.WORKLOADS[name]
    ctx.set_catalog(cat.xyz, w, cat.n_data)
    ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"] if nmu is None else nmu)
    return cat, w, sp


def _same(a, b):
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_save_load_roundtrip(tmp_path, oracle):
    path = tmp_path / "c2.csr"
    with api.Context(0) as ctx:
        cat, w, sp = _setup(ctx, "c2_3pcf", 0.02)
        fresh3 = ctx.count_3pcf()
        fresh2 = ctx.count_2pcf()
        ctx.graph_save(path)
    with api.Context(0) as ctx:
        _setup(ctx, "c2_3pcf", 0.02)
        ctx.graph_load(path)
        got3 = ctx.count_3pcf()
        assert ctx.stats()["ms_graph"] < 0.05  # no graph build
        _same(got3, fresh3)
        _same(ctx.count_2pcf(), fresh2)
        _same(ctx.count_equi(), ctx.count_equi())
        rp, col, b, mu = ctx.graph()
        G = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
        orp, ocol, ob, omu = G.csr()
        assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
        assert np.array_equal(b, ob) and np.array_equal(mu, omu)
        ref = G.pcf3(w, cat.n_data)
        assert np.array_equal(got3["counts"], ref["counts"])


def test_save_load_4pcf(tmp_path):
    path = tmp_path / "c3.csr"
    with api.Context(0) as ctx:
        _setup(ctx, "c3_4pcf", 0.05)
        fresh = ctx.count_4pcf()
        fresh_t = ctx.count_tetra()
        ctx.graph_save(path)
        _setup(ctx, "c3_4pcf", 0.05)
        ctx.graph_load(path)
        _same(ctx.count_4pcf(), fresh)
        _same(ctx.count_tetra(), fresh_t)


def test_load_refuses_mismatches(tmp_path):
    path = tmp_path / "g.csr"
    with api.Context(0) as ctx:
        cat, w, sp = _setup(ctx, "c2_3pcf", 0.01)
        ctx.graph_save(path)
        # other bins
        ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"] + 1, sp["nmu"])
        with pytest.raises(GramsciError) as e:
            ctx.graph_load(path)
        assert e.value.code == -1
        # other coordinates (one point moved)
        xyz = cat.xyz.copy()
        xyz[5, 0] += 1e-9
        ctx.set_catalog(xyz, w, cat.n_data)
        ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
        with pytest.raises(GramsciError):
            ctx.graph_load(path)
        # damaged payload
        ctx.set_catalog(cat.xyz, w, cat.n_data)
        raw = bytearray(pathlib.Path(path).read_bytes())
        raw[200] ^= 0x40
        bad = tmp_path / "bad.csr"
        bad.write_bytes(bytes(raw))
        with pytest.raises(GramsciError):
            ctx.graph_load(bad)
        # truncated file
        bad.write_bytes(bytes(raw[:100]))
        with pytest.raises(GramsciError):
            ctx.graph_load(bad)
        # the good file still loads and counts
        ctx.graph_load(path)
        assert ctx.count_3pcf()["counts"].sum() > 0


def test_keep_graph_reuses_and_invalidates(oracle):
    with api.Context(0) as ctx:
        ctx.set_keep_graph(True)
        cat, w, sp = _setup(ctx, "c2_3pcf", 0.01)
        a = ctx.count_3pcf()
        b = ctx.count_3pcf()
        assert ctx.stats()["ms_graph"] < 0.05
        _same(a, b)
        # a new catalogue invalidates the kept graph
        cat2, w2, _ = _setup(ctx, "c2_3pcf", 0.01, seed=123)
        got = ctx.count_3pcf()
        ref = oracle.Graph(cat2.xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"]).pcf3(w2, cat2.n_data)
        assert np.array_equal(got["counts"], ref["counts"])
        # precision change invalidates too, and f64 gives the same graph
        ctx.set_precision("f64")
        _same(ctx.count_3pcf(), got)
        ctx.set_keep_graph(False)
