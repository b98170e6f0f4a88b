"""Known-answer configurations (tests/golden/known_answers.json, made by
tests/golden/make_golden.py from geometry alone) against the oracle (CPU)
and against the CUDA library (GPU).  The 4PCF answers of the tetrahedron
case pin the oracle; the library's 4PCF is held to the oracle by the GPU
parity tests."""
import json
import os

import numpy as np
import pytest

from gramsci_b200 import catalogs

with open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")) as _f:
    CASES = json.load(_f)


def _prep(c):
    xyz = np.array(c["xyz"], np.float64)
    n = len(xyz)
    w = catalogs.normalise(np.array(c["w"], np.float64), c["n_data"], n - c["n_data"])
    return xyz, w


def _check(c, counts2, counts3=None, N2_3=None):
    exp2 = np.zeros_like(counts2)
    for k, v in c["counts2"].items():
        b, m, cat = map(int, k.split(","))
        exp2[b - 1, m - 1, cat] = v
    assert np.array_equal(counts2, exp2), c["name"]
    if counts3 is not None and "counts3" in c:
        exp3 = np.zeros_like(counts3)
        for k, v in c["counts3"].items():
            cfg, m, nr = map(int, k.split(","))
            exp3[cfg - 1, m - 1, nr] = v
        assert np.array_equal(counts3, exp3), c["name"]
    if N2_3 is not None and "N2_3" in c:
        for k, v in c["N2_3"].items():
            cfg, m = map(int, k.split(","))
            assert abs(N2_3[cfg - 1, m - 1] - v) <= c.get("rtol", 1e-15) * abs(v)


def _check4(c, r4):
    """4PCF known answers: counts by number of randoms, N2, disconnected-term
    counts (term 1-6, randoms in the pair) and discN sums; every entry not
    listed is 0."""
    exp = np.zeros_like(r4["counts"])
    for k, v in c["counts4"].items():
        cfg, d1, d2, nr = map(int, k.split(","))
        exp[cfg - 1, d1 - 1, d2 - 1, nr] = v
    assert np.array_equal(r4["counts"], exp), c["name"]
    exp = np.zeros_like(r4["dcount"])
    for k, v in c["dcount4"].items():
        cfg, d1, d2, t, npr = map(int, k.split(","))
        exp[cfg - 1, d1 - 1, d2 - 1, t - 1, npr] = v
    assert np.array_equal(r4["dcount"], exp), c["name"]
    for key, got in (("N2_4", r4["N2"]), ("discN4", r4["discN"])):
        exp = np.zeros_like(got)
        for k, v in c[key].items():
            exp[tuple(int(x) - 1 for x in k.split(","))] = v
        np.testing.assert_allclose(got, exp, rtol=c["rtol"], atol=0)
    assert not r4["N3"].any() and not r4["discR"].any()


def _check_special(c, eq, te):
    """-equi and -tetra known answers: counts by number of randoms, N2 and
    (-tetra) discN; N3 and discR are 0 in these cases."""
    exp = np.zeros_like(eq["counts"])
    for k, v in c["counts_equi"].items():
        b, m, nr = map(int, k.split(","))
        exp[b - 1, m - 1, nr] = v
    assert np.array_equal(eq["counts"], exp), c["name"]
    exp = np.zeros_like(te["counts"])
    for k, v in c["counts_tetra"].items():
        b, nr = map(int, k.split(","))
        exp[b - 1, nr] = v
    assert np.array_equal(te["counts"], exp), c["name"]
    for entries, got in ((c["N2_equi"], eq["N2"]), (c["N2_tetra"], te["N2"]),
                         (c["discN_tetra"], te["discN"])):
        exp = np.zeros_like(got)
        for k, v in entries.items():
            exp[tuple(int(x) - 1 for x in k.split(","))] = v
        np.testing.assert_allclose(got, exp, rtol=c["rtol"], atol=0)
    assert not eq["N3"].any() and not te["N3"].any() and not te["discR"].any()


@pytest.mark.parametrize("c", CASES, ids=[c["name"] for c in CASES])
def test_oracle_known_answers(oracle, c):
    xyz, w = _prep(c)
    G = oracle.Graph(xyz, c["rmin"], c["rmax"], c["nbins"], c["nmu"])
    r2 = G.pcf2(w, c["n_data"])
    r3 = G.pcf3(w, c["n_data"]) if c["n_data"] >= 3 else None
    _check(c, r2["counts"], r3["counts"] if r3 else None, r3["N2"] if r3 else None)
    if "counts4" in c:
        _check4(c, G.pcf4(w, c["n_data"]))
    if "counts_equi" in c:
        _check_special(c, G.equi(w, c["n_data"]), G.tetra(w, c["n_data"]))
    if "log_case" in c:
        lc = dict(c, **c["log_case"])
        GL = oracle.Graph(xyz, lc["rmin"], lc["rmax"], lc["nbins"], lc["nmu"], logbins=True)
        _check(lc, GL.pcf2(w, c["n_data"])["counts"])
        rp, col, b, mu = GL.csr()
        for k, (eb, em) in lc["edges"].items():
            i, j = map(int, k.split(","))
            e = rp[i] + list(col[rp[i]:rp[i + 1]]).index(j)
            assert (b[e], mu[e]) == (eb, em), k
    if "buffer_case" in c:
        bc = dict(c, **c["buffer_case"])
        buf = np.array(bc["buffer"], np.int32)
        nd = c["n_data"]
        r3b = G.pcf3(w, nd, buffer=buf)
        _check(bc, G.pcf2(w, nd, buffer=buf)["counts"], r3b["counts"], r3b["N2"])
        if "counts4" in bc:
            _check4(bc, G.pcf4(w, nd, buffer=buf))
    if "grad2" in c:
        nd, nb, nm = c["n_data"], c["nbins"], c["nmu"]
        r4 = G.pcf4(w, nd)
        got = [G.adjoint2(w, nd, np.ones((nb, nm))),
               G.adjoint3(w, nd, np.ones((oracle.ncfg3(nb), nm))),
               G.adjoint4(w, nd, np.ones_like(r4["N2"]))]
        for k, g in zip(("grad2", "grad3", "grad4"), got):
            np.testing.assert_allclose(g, c[k], rtol=c["rtol"], atol=1e-15, err_msg=k)
    if "edges" in c:
        rp, col, b, mu = G.csr()
        for k, (eb, em) in c["edges"].items():
            i, j = map(int, k.split(","))
            row = list(col[rp[i]:rp[i + 1]])
            e = rp[i] + row.index(j)
            assert (b[e], mu[e]) == (eb, em), k


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("c", CASES, ids=[c["name"] for c in CASES])
def test_gpu_known_answers(gpu_ctx, c, precision):
    xyz, w = _prep(c)
    gpu_ctx.set_precision(precision)
    gpu_ctx.set_catalog(xyz, w, c["n_data"])
    gpu_ctx.set_bins(c["rmin"], c["rmax"], c["nbins"], c["nmu"])
    r2 = gpu_ctx.count_2pcf()
    r3 = gpu_ctx.count_3pcf()
    _check(c, r2["counts"], r3["counts"], r3["N2"])
    if "edges" in c:
        rp, col, b, mu = gpu_ctx.graph()
        for k, (eb, em) in c["edges"].items():
            i, j = map(int, k.split(","))
            row = list(col[rp[i]:rp[i + 1]])
            e = rp[i] + row.index(j)
            assert (b[e], mu[e]) == (eb, em), k
    gpu_ctx.set_precision("f32")
