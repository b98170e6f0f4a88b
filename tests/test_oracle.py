"""CPU tests of the oracle: the oracle is pinned by independent brute-force
enumerations written here in numpy/Python, by hand-derived configurations
(tests/golden), and by agreement of its two range searches (uniform grid and
kd-tree restatement of the reference's search)."""
import itertools
import math

import numpy as np
import pytest

from gramsci_b200 import catalogs


def brute_edges(xyz, rmin, rmax, nbins, nmu, logbins=False):
    """Reference predicate written independently: all ordered pairs.  Log
    bins take floor((log10 r - log10 rmin) / delta) + 1 with delta =
    (log10 rmax - log10 rmin) / nbins (gramsci.F90:136-139, :334-335)."""
    n = len(xyz)
    if logbins:
        inv_dr = 1.0 / ((math.log10(rmax) - math.log10(rmin)) / nbins)
    else:
        inv_dr = 1.0 / ((rmax - rmin) / nbins)
    mu_scale = 0.5 * nmu
    E = {}
    for i in range(n):
        for j in range(n):
            if i == j:
                continue
            d = xyz[j] - xyz[i]
            sd = d[0] * d[0]
            sd = sd + d[1] * d[1]
            sd = sd + d[2] * d[2]
            if sd > rmax * rmax or (rmin > 0 and sd <= rmin * rmin):
                continue
            r = math.sqrt(sd)
            if r <= rmin or r >= rmax:
                continue
            t = (math.log10(r) - math.log10(rmin)) * inv_dr if logbins else (r - rmin) * inv_dr
            b = min(int(math.floor(t)) + 1, nbins)
            m = 1
            if nmu >= 2:
                mid = 0.5 * (xyz[i] + xyz[j])
                s = xyz[i] - xyz[j]
                th = mid[0] * s[0]
                th = th + mid[1] * s[1]
                th = th + mid[2] * s[2]
                nm = mid[0] * mid[0]
                nm = nm + mid[1] * mid[1]
                nm = nm + mid[2] * mid[2]
                ns = s[0] * s[0]
                ns = ns + s[1] * s[1]
                ns = ns + s[2] * s[2]
                th = th / (math.sqrt(nm) * math.sqrt(ns))
                m = min(max(int(math.floor((th + 1.0) * mu_scale)) + 1, 1), nmu)
            E[(i, j)] = (b, m)
    return E


def small_catalogue(n_data, n_rand, box, seed):
    rng = np.random.default_rng(seed)
    g = catalogs.neyman_scott(rng, max(1, n_data // 5), 5.0, box / 20, 0.0, box)[:n_data]
    r = rng.uniform(0, box, size=(n_rand, 3))
    xyz = np.concatenate([g, r])
    w = catalogs.normalise(rng.lognormal(0, 0.3, len(xyz)), len(g), n_rand)
    return xyz, w, len(g)


@pytest.mark.parametrize("nmu", [1, 4])
@pytest.mark.parametrize("method", ["grid", "kdtree"])
def test_graph_matches_brute_force(oracle, nmu, method):
    xyz, w, nd = small_catalogue(40, 60, 100.0, 1)
    G = oracle.Graph(xyz, 3.0, 30.0, 6, nmu, method=method)
    rp, col, b, mu = G.csr()
    E = brute_edges(xyz, 3.0, 30.0, 6, nmu)
    got = {}
    for i in range(len(xyz)):
        row = col[rp[i]:rp[i + 1]]
        assert np.all(np.diff(row) > 0), "rows must be sorted by id"
        for k in range(rp[i], rp[i + 1]):
            got[(i, int(col[k]))] = (int(b[k]), int(mu[k]))
    assert got == E


@pytest.mark.parametrize("nmu", [1, 3])
@pytest.mark.parametrize("method", ["grid", "kdtree"])
def test_log_bin_graph_matches_brute_force(oracle, nmu, method):
    xyz, w, nd = small_catalogue(40, 60, 100.0, 4)
    G = oracle.Graph(xyz, 1.5, 40.0, 7, nmu, logbins=True, method=method)
    rp, col, b, mu = G.csr()
    E = brute_edges(xyz, 1.5, 40.0, 7, nmu, logbins=True)
    got = {(i, int(col[k])): (int(b[k]), int(mu[k]))
           for i in range(len(xyz)) for k in range(rp[i], rp[i + 1])}
    assert got == E
    # log bins differ from linear ones on this range
    lin = brute_edges(xyz, 1.5, 40.0, 7, nmu)
    assert lin.keys() == E.keys() and any(lin[e][0] != E[e][0] for e in E)


def test_grid_and_kdtree_agree(oracle):
    cat = catalogs.make("c2_3pcf", scale=0.01)
    a = oracle.Graph(cat.xyz, 5, 25, 8, 5, method="grid").csr()
    b = oracle.Graph(cat.xyz, 5, 25, 8, 5, method="kdtree").csr()
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_rmin_zero_and_duplicates(oracle):
    xyz = np.array([[0, 0, 0], [0, 0, 0], [1, 0, 0], [0, 2, 0], [50, 50, 50]], float)
    G = oracle.Graph(xyz, 0.0, 3.0, 3, 1)
    rp, col, b, mu = G.csr()
    # duplicates (d = 0) are never neighbours: rmin < d is strict
    assert list(col[rp[0]:rp[1]]) == [2, 3]
    assert list(col[rp[1]:rp[2]]) == [2, 3]
    assert rp[5] - rp[4] == 0


def _brute_counts(xyz, w, nd, rmin, rmax, nbins, nmu, normal, buffer=None, logbins=False):
    E = brute_edges(xyz, rmin, rmax, nbins, nmu, logbins=logbins)
    n = len(xyz)
    nb = {i: sorted(j for (a, j) in E if a == i) for i in range(n)}
    rnd = lambda i: i >= nd  # noqa: E731
    c2 = np.zeros((nbins, nmu, 4), np.int64)
    for (i, j), (b, m) in E.items():
        if buffer is not None and buffer[i]:
            continue
        c2[b - 1, m - 1, 2 * rnd(i) + rnd(j)] += 1
    from oracle import oracle as O

    nc = O.ncfg3(nbins)
    c3 = np.zeros((nc, nmu, 4), np.int64)
    s3 = np.zeros((nc, nmu, 4))
    for i in range(n):
        if buffer is not None and buffer[i]:
            continue
        for a, c in itertools.combinations(nb[i], 2):
            if (a, c) not in E:
                continue
            b1, m1 = E[(i, a)]
            b2, m2 = E[(i, c)]
            b3 = E[(a, c)][0]
            cfg = O.bintable3(b1, b2, b3, nbins)
            m = normal[m1 - 1, m2 - 1] if nmu >= 2 else 1
            k = rnd(i) + rnd(a) + rnd(c)
            c3[cfg - 1, m - 1, k] += 1
            s3[cfg - 1, m - 1, k] += w[i] * w[a] * w[c]
    return c2, c3, s3


@pytest.mark.parametrize("logbins", [False, True])
@pytest.mark.parametrize("nmu", [1, 3])
def test_2pcf_3pcf_match_brute_force(oracle, nmu, logbins):
    xyz, w, nd = small_catalogue(30, 45, 60.0, 2)
    buf = (np.arange(len(xyz)) % 7 == 3).astype(np.int32)
    normal = oracle.normal_table(nmu)
    c2, c3, s3 = _brute_counts(xyz, w, nd, 2.0, 20.0, 5, nmu, normal, buffer=buf, logbins=logbins)
    G = oracle.Graph(xyz, 2.0, 20.0, 5, nmu, logbins=logbins)
    r2 = G.pcf2(w, nd, buffer=buf)
    r3 = G.pcf3(w, nd, buffer=buf)
    assert np.array_equal(r2["counts"], c2)
    assert np.array_equal(r3["counts"], c3)
    assert np.allclose(r3["catsum"], s3, rtol=1e-13, atol=0)
    # N3 is minus the all-random sum (gramsci.F90:495-497)
    assert np.allclose(r3["N3"], -r3["catsum"][:, :, 3], rtol=1e-13, atol=1e-300)


@pytest.mark.parametrize("logbins", [False, True])
@pytest.mark.parametrize("with_buffer", [False, True])
def test_4pcf_matches_brute_force(oracle, with_buffer, logbins):
    xyz, w, nd = small_catalogue(25, 25, 30.0, 3)
    buf = (np.arange(len(xyz)) % 5 == 2).astype(np.int32) if with_buffer else None
    nbins = 3
    E = brute_edges(xyz, 1.0, 12.0, nbins, 1, logbins=logbins)
    n = len(xyz)
    nbrs = {i: sorted(j for (a, j) in E if a == i) for i in range(n)}
    nc = oracle.ncfg4(nbins)
    cnt = np.zeros((nc, nbins, nbins, 5), np.int64)
    dcnt = np.zeros((nc, nbins, nbins, 6, 4), np.int64)
    n2 = np.zeros((nc, nbins, nbins))
    n3 = np.zeros((nc, nbins, nbins))
    dn = np.zeros((nc, nbins, nbins, 6))
    dr = np.zeros((nc, nbins, nbins, 6))
    gate = [3, 3, 1, 0, 0, 0]
    pu = [0, 0, 0, 1, 3, 3]
    pv = [1, 2, 3, 2, 2, 1]
    for i in range(n):
        if len(nbrs[i]) <= 3 or (buf is not None and buf[i]):
            continue
        for a, b, c in itertools.combinations(nbrs[i], 3):
            if (a, b) not in E or (b, c) not in E or (a, c) not in E:
                continue
            cfg = oracle.bintable4(E[(i, a)][0], E[(a, b)][0], E[(b, c)][0], E[(i, c)][0], nbins)
            if cfg <= 0:
                continue
            d1, d2 = E[(i, b)][0], E[(a, c)][0]
            v = [i, a, b, c]
            r = [x >= nd for x in v]
            cnt[cfg - 1, d1 - 1, d2 - 1, sum(r)] += 1
            # N2 takes every clique's weight product, N3 the all-random ones
            # (gramsci.F90:704-707)
            wp = w[i] * w[a] * w[b] * w[c]
            n2[cfg - 1, d1 - 1, d2 - 1] += wp
            if all(r):
                n3[cfg - 1, d1 - 1, d2 - 1] += wp
            for t in range(6):
                if r[gate[t]]:
                    npr = r[pu[t]] + r[pv[t]]
                    dcnt[cfg - 1, d1 - 1, d2 - 1, t, npr] += 1
                    # discN takes the pair's weight product when the gate
                    # vertex is a random, discR when the pair is too
                    # (gramsci.F90:752-818)
                    pw = w[v[pu[t]]] * w[v[pv[t]]]
                    dn[cfg - 1, d1 - 1, d2 - 1, t] += pw
                    if npr == 2:
                        dcnt[cfg - 1, d1 - 1, d2 - 1, t, 3] += 1
                        dr[cfg - 1, d1 - 1, d2 - 1, t] += pw
    G = oracle.Graph(xyz, 1.0, 12.0, nbins, 1, logbins=logbins)
    r4 = G.pcf4(w, nd, buffer=buf)
    assert cnt.sum() > 0
    assert np.array_equal(r4["counts"], cnt)
    assert np.array_equal(r4["dcount"], dcnt)
    scale = np.abs(n2).max()
    np.testing.assert_allclose(r4["N2"], n2, rtol=1e-12, atol=1e-13 * scale)
    np.testing.assert_allclose(r4["N3"], n3, rtol=1e-12, atol=1e-13 * scale)
    dscale = np.abs(dn).max()
    assert dscale > 0
    np.testing.assert_allclose(r4["discN"], dn, rtol=1e-12, atol=1e-13 * dscale)
    np.testing.assert_allclose(r4["discR"], dr, rtol=1e-12, atol=1e-13 * dscale)


def test_bintables(oracle):
    # 3PCF: symmetric, ranks 1..C(n+2,3) in lexicographic order of i<=j<=k
    n = 5
    rank = 0
    for i in range(1, n + 1):
        for j in range(i, n + 1):
            for k in range(j, n + 1):
                rank += 1
                for p in itertools.permutations((i, j, k)):
                    assert oracle.bintable3(*p, n) == rank
    assert rank == oracle.ncfg3(n)
    # 4PCF: canonical entries only
    rank = 0
    for t in itertools.product(range(1, n + 1), repeat=4):
        if list(t) == sorted(t):
            rank += 1
    assert rank == oracle.ncfg4(n)
    assert oracle.bintable4(1, 1, 1, 1, n) == 1
    assert oracle.bintable4(n, n, n, n, n) == oracle.ncfg4(n)
    assert oracle.bintable4(2, 1, 3, 4, n) == 0


def test_find_normal_table(oracle):
    # find_normal is symmetric in its arguments only up to rounding; the
    # table is indexed [mu(k1)-1, mu(k2)-1] with k1 < k2 in id order.
    differ = []
    for nmu in range(2, 128):
        t0 = oracle.normal_table(nmu, 0)
        t1 = oracle.normal_table(nmu, 1)
        assert t0.min() >= 1 and t0.max() <= nmu
        assert t1.min() >= 1 and t1.max() <= nmu
        if not np.array_equal(t0, t1):
            differ.append(nmu)
            # a contraction choice moves a handful of entries by one bin
            assert np.abs(t0 - t1).max() == 1 and (t0 != t1).sum() <= 16
    # Up to nmu = 21 (the workloads use 1..10) the separate-operation and the
    # FMA-contracted evaluation give the same table, so the reference build's
    # contraction choice cannot change a 3PCF mu bin there.
    assert min(differ) == 22
    # mu bins symmetric about the centre give the largest normal value
    t = oracle.normal_table(5, 0)
    assert t[2, 2] == 5 or t[2, 2] >= t[0, 0]


def test_normalise_matches_reference_rule(oracle):
    rng = np.random.default_rng(0)
    w = rng.lognormal(0, 0.3, 1000)
    a = catalogs.normalise(w, 400, 600)
    b = oracle.normalise(w, 400, 600)
    assert np.array_equal(a, b)
    assert abs(a[:400].sum() - 1) < 1e-12 and abs(a[400:].sum() + 1) < 1e-12


@pytest.mark.parametrize("with_buffer", [False, True])
def test_adjoint_2pcf_matches_finite_differences(oracle, with_buffer):
    xyz, w, nd = small_catalogue(30, 40, 60.0, 4)
    buf = (np.arange(len(w)) % 4 == 1).astype(np.int32) if with_buffer else None
    G = oracle.Graph(xyz, 2.0, 20.0, 4, 3)
    rng = np.random.default_rng(9)
    cot2 = rng.normal(size=(4, 3))
    cot3 = rng.normal(size=(4, 3))
    g = G.adjoint2(w, nd, cot2, cot3, buffer=buf)

    def L(wv):
        r = G.pcf2(wv, nd, buffer=buf)
        return float((cot2 * r["N2"]).sum() + (cot3 * r["N3"]).sum())

    for k in rng.choice(len(w), 8, replace=False):
        h = 1e-3 * abs(w[k])
        wp, wm = w.copy(), w.copy()
        wp[k] += h
        wm[k] -= h
        fd = (L(wp) - L(wm)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-8 * max(abs(fd), abs(g[k]), 1e-30)


@pytest.mark.parametrize("with_buffer", [False, True])
def test_adjoint_3pcf_matches_finite_differences(oracle, with_buffer):
    xyz, w, nd = small_catalogue(30, 40, 50.0, 5)
    buf = (np.arange(len(w)) % 4 == 1).astype(np.int32) if with_buffer else None
    nb, nm = 3, 2
    G = oracle.Graph(xyz, 2.0, 20.0, nb, nm)
    rng = np.random.default_rng(10)
    nc = oracle.ncfg3(nb)
    cot2 = rng.normal(size=(nc, nm))
    cot3 = rng.normal(size=(nc, nm))
    g = G.adjoint3(w, nd, cot2, cot3, buffer=buf)

    def L(wv):
        r = G.pcf3(wv, nd, buffer=buf)
        return float((cot2 * r["N2"]).sum() + (cot3 * r["N3"]).sum())

    for k in rng.choice(len(w), 8, replace=False):
        h = 1e-3 * abs(w[k])
        wp, wm = w.copy(), w.copy()
        wp[k] += h
        wm[k] -= h
        fd = (L(wp) - L(wm)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-7 * max(abs(fd), abs(g[k]), 1e-30)


def test_adjoint_4pcf_matches_finite_differences(oracle):
    """All four cotangent terms (N2, N3, discN, discR), buffer roots
    included.  The sums are multilinear in the weights, so central
    differences carry only rounding error."""
    xyz, w, nd = small_catalogue(25, 25, 30.0, 3)
    nb = 3
    G = oracle.Graph(xyz, 1.0, 12.0, nb, 1)
    rng = np.random.default_rng(12)
    buf = (rng.random(len(w)) < 0.15).astype(np.int32)
    nc = oracle.ncfg4(nb)
    c2, c3 = rng.normal(size=(nc, nb, nb)), rng.normal(size=(nc, nb, nb))
    cN, cR = rng.normal(size=(nc, nb, nb, 6)), rng.normal(size=(nc, nb, nb, 6))
    g = G.adjoint4(w, nd, c2, c3, cN, cR, buffer=buf)

    def L(wv):
        r = G.pcf4(wv, nd, buffer=buf)
        return float((c2 * r["N2"]).sum() + (c3 * r["N3"]).sum() + (cN * r["discN"]).sum()
                     + (cR * r["discR"]).sum())

    assert np.count_nonzero(g) > len(w) // 4
    gmax = np.abs(g).max()
    for k in rng.choice(np.flatnonzero(g), 10, replace=False):
        h = 0.5 * abs(w[k])
        wp, wm = w.copy(), w.copy()
        wp[k] += h
        wm[k] -= h
        fd = (L(wp) - L(wm)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-10 * gmax, (k, fd, g[k])


@pytest.mark.parametrize("nm,with_buffer", [(2, False), (1, False), (1, True)])
def test_equi_and_tetra_match_brute_force(oracle, nm, with_buffer):
    """-equi / -tetra (gramsci.F90:402-660): same-bin triangles and 4-cliques,
    counts and weighted sums, against an independent enumeration."""
    xyz, w, nd = small_catalogue(30, 30, 30.0, 6)
    nb = 3
    buf = (np.arange(len(xyz)) % 6 == 1).astype(np.int32) if with_buffer else None
    E = brute_edges(xyz, 1.0, 12.0, nb, nm)
    n = len(xyz)
    nbrs = {i: sorted(j for (a, j) in E if a == i) for i in range(n)}
    normal = oracle.normal_table(nm)
    rnd = lambda i: i >= nd  # noqa: E731
    ce = np.zeros((nb, nm, 4), np.int64)
    e2, e3 = np.zeros((nb, nm)), np.zeros((nb, nm))
    ct = np.zeros((nb, 5), np.int64)
    t2, t3 = np.zeros(nb), np.zeros(nb)
    dn, dr = np.zeros((nb, 6)), np.zeros((nb, 6))
    for i in range(n):
        if buf is not None and buf[i]:
            continue
        for a, c in itertools.combinations(nbrs[i], 2):
            b = E[(i, a)][0]
            if E[(i, c)][0] != b or E.get((a, c), (0,))[0] != b:
                continue
            m = normal[E[(i, a)][1] - 1, E[(i, c)][1] - 1] if nm >= 2 else 1
            ce[b - 1, m - 1, rnd(i) + rnd(a) + rnd(c)] += 1
            e2[b - 1, m - 1] += w[i] * w[a] * w[c]
            # without mu bins N3 takes minus the all-random products
            # (gramsci.F90:430-433); with them only N2 is summed
            if nm == 1 and rnd(i) and rnd(a) and rnd(c):
                e3[b - 1, 0] -= w[i] * w[a] * w[c]
        for a, b2, c in itertools.combinations(nbrs[i], 3):
            b = E[(i, a)][0]
            if not all(E.get(e, (0,))[0] == b for e in [(i, b2), (i, c), (a, b2), (b2, c), (a, c)]):
                continue
            ct[b - 1, sum(rnd(x) for x in (i, a, b2, c))] += 1
            p4 = w[i] * w[a] * w[b2] * w[c]
            t2[b - 1] += p4
            if all(rnd(x) for x in (i, a, b2, c)):
                t3[b - 1] += p4
            # the six disconnected terms: (gate, the two other vertices of
            # the triple product), term t at index t-1 (:581-628)
            for t, (gate, u, v) in enumerate([(c, i, a), (c, i, b2), (a, i, c),
                                              (i, a, b2), (i, c, b2), (i, c, a)]):
                if rnd(gate):
                    pw = w[gate] * w[u] * w[v]
                    dn[b - 1, t] += pw
                    if rnd(u) and rnd(v):
                        dr[b - 1, t] += pw
    G = oracle.Graph(xyz, 1.0, 12.0, nb, nm)
    e = G.equi(w, nd, buffer=buf)
    t = G.tetra(w, nd, buffer=buf)
    assert ce.sum() > 0 and ct.sum() > 0
    assert np.array_equal(e["counts"], ce)
    assert np.array_equal(t["counts"], ct)
    for got, ref in ((e["N2"], e2), (e["N3"], e3), (t["N2"], t2), (t["N3"], t3),
                     (t["discN"], dn), (t["discR"], dr)):
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-14 * max(np.abs(ref).max(), 1e-300))
    if nm >= 2:
        # with mu bins the reference sums only N2 for -equi
        assert np.all(e["N3"] == 0)


def test_empty_single_and_all_buffer_catalogues(oracle):
    for xyz in (np.zeros((0, 3)), np.array([[1.0, 2.0, 3.0]])):
        n = len(xyz)
        G = oracle.Graph(xyz, 1.0, 10.0, 3, 2)
        assert np.array_equal(G.csr()[0], np.zeros(n + 1, np.int64))
        w = np.full(n, 1.0)
        for r in (G.pcf2(w, n), G.pcf3(w, n), G.pcf4(w, n)):
            assert not r["N2"].any() and not r["N3"].any() and not r["counts"].any()
    xyz, w, nd = small_catalogue(30, 30, 40.0, 5)
    G = oracle.Graph(xyz, 1.0, 12.0, 3, 2)
    allbuf = np.ones(len(xyz), np.int32)
    assert G.pcf3(w, nd)["counts"].sum() > 0
    for r in (G.pcf2(w, nd, buffer=allbuf), G.pcf3(w, nd, buffer=allbuf),
              G.pcf4(w, nd, buffer=allbuf)):
        assert not r["N2"].any() and not r["counts"].any()


def test_galaxies_only_have_no_random_terms(oracle):
    xyz, w, nd = small_catalogue(60, 0, 40.0, 6)
    G = oracle.Graph(xyz, 1.0, 12.0, 3, 1)
    r2, r3, r4 = G.pcf2(w, nd), G.pcf3(w, nd), G.pcf4(w, nd)
    assert r2["counts"][..., 0].sum() > 0 and r3["counts"][..., 0].sum() > 0
    for r in (r2, r3, r4):
        assert not r["N3"].any() and not r["counts"][..., 1:].any()
    assert not r4["discN"].any() and not r4["discR"].any()


@pytest.mark.parametrize("method", ["grid", "kdtree"])
def test_thread_count_does_not_change_results(oracle, method):
    """The reference arm runs the oracle on every host thread: the graph and
    the integer counts do not depend on the thread count, and the sums
    only to rounding."""
    cat = catalogs.make("c2_3pcf", scale=0.01)
    w = catalogs.normalise(cat.w, cat.n_data, cat.n_rand)
    sp = catalogs.WORKLOADS["c2_3pcf"]
    args = (cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    G1 = oracle.Graph(*args, method=method, threads=1)
    G4 = oracle.Graph(*args, method=method, threads=4)
    for x, y in zip(G1.csr(), G4.csr()):
        assert np.array_equal(x, y)
    a, b = G1.pcf3(w, cat.n_data), G4.pcf3(w, cat.n_data)
    assert a["counts"].sum() > 0 and np.array_equal(a["counts"], b["counts"])
    np.testing.assert_allclose(a["catsum"], b["catsum"], rtol=1e-12, atol=1e-15 * np.abs(a["catsum"]).max())
