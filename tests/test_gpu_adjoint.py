"""Weight adjoints on the GPU (the adjoint workload at reduced scale: Neyman-Scott
galaxies with lognormal weights plus uniform randoms, same number density).

* against the oracle's gradient (long double accumulation on the CPU):
  |g_gpu - g_oracle| <= 1e-12 * max|g_oracle| elementwise;
* against FP64 central finite differences of the GPU forward pass on 64
  seeded weights, through the torch.autograd.Function: relative 1e-8.  The
  counts are multilinear in the weights (a point appears at most once per
  pair or triangle), so central differences carry no truncation error for
  any step; a step of half the weight keeps the FP64 cancellation in
  L(w+h) - L(w-h) far below the tolerance;
* through the weight normalisation with torch autograd.

The 4PCF adjoint (all four cotangent terms N2, N3, discN, discR) is checked
the same two ways on the 4PCF workload (Neyman-Scott galaxies, 4 bins) at
reduced scale, with lognormal weights and with buffer points.
"""
import numpy as np
import pytest

from gramsci_b200 import api, catalogs

pytestmark = pytest.mark.gpu


def _cat(name, scale, seed=None):
    cat = catalogs.make(name, scale=scale, seed=seed)
    w = catalogs.normalise(cat.w, cat.n_data, cat.n_rand)
    return cat, w, catalogs.WORKLOADS[name]


@pytest.mark.parametrize("order,name,scale,mode", [(2, "c5_adjoint_2pcf", 0.003, "auto"),
                                                   (3, "c5_adjoint_3pcf", 0.002, "auto"),
                                                   (3, "c2_3pcf", 0.01, "auto"),
                                                   (3, "c2_3pcf", 0.01, "hash")])
def test_adjoint_matches_oracle(gpu_ctx, oracle, order, name, scale, mode):
    gpu_ctx.set_clique_mode(mode)
    try:
        _adjoint_matches_oracle(gpu_ctx, oracle, order, name, scale)
    finally:
        gpu_ctx.set_clique_mode("auto")


def _adjoint_matches_oracle(gpu_ctx, oracle, order, name, scale):
    cat, w, sp = _cat(name, scale)
    rng = np.random.default_rng(order)
    gpu_ctx.set_catalog(cat.xyz, w, cat.n_data)
    gpu_ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    G = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    if order == 2:
        shape = (sp["nbins"], sp["nmu"])
        c2, c3 = rng.normal(size=shape), rng.normal(size=shape)
        g = gpu_ctx.adjoint_2pcf(c2, c3)
        ref = G.adjoint2(w, cat.n_data, c2, c3)
    else:
        shape = (oracle.ncfg3(sp["nbins"]), sp["nmu"])
        c2, c3 = rng.normal(size=shape), rng.normal(size=shape)
        gpu_ctx.count_3pcf()  # the adjoint reuses this graph
        g = gpu_ctx.adjoint_3pcf(c2, c3)
        ref = G.adjoint3(w, cat.n_data, c2, c3)
    assert np.abs(ref).max() > 0
    assert np.all(np.abs(g - ref) <= 1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("case", ["lognormal", "buffer", "unit_partial", "hash"])
def test_adjoint_4pcf_matches_oracle(gpu_ctx, oracle, case):
    cat = catalogs.make("c3_4pcf", scale=0.05)
    sp = catalogs.WORKLOADS["c3_4pcf"]
    rng = np.random.default_rng(40 + len(case))
    raw = np.ones(cat.n) if case == "unit_partial" else rng.lognormal(0, 0.3, cat.n)
    w = catalogs.normalise(raw, cat.n_data, cat.n_rand)
    buf = (rng.random(cat.n) < 0.2).astype(np.int32) if case == "buffer" else None
    gpu_ctx.set_catalog(cat.xyz, w, cat.n_data, buffer=buf)
    gpu_ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    nb = sp["nbins"]
    nc = oracle.ncfg4(nb)
    c2, c3 = rng.normal(size=(nc, nb, nb)), rng.normal(size=(nc, nb, nb))
    cN, cR = rng.normal(size=(nc, nb, nb, 6)), rng.normal(size=(nc, nb, nb, 6))
    if case == "unit_partial":
        c3, cR = None, None
        gpu_ctx.count_4pcf()  # the adjoint reuses this graph
    if case == "hash":
        gpu_ctx.set_clique_mode("hash")
    try:
        g = gpu_ctx.adjoint_4pcf(c2, c3, cN, cR)
    finally:
        gpu_ctx.set_clique_mode("auto")
    G = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    ref = G.adjoint4(w, cat.n_data, c2, c3, cN, cR, buffer=buf)
    assert np.count_nonzero(ref) > cat.n // 10
    assert np.all(np.abs(g - ref) <= 1e-12 * np.abs(ref).max())
    if buf is not None:
        # buffer points are never roots but still carry gradient as members
        assert np.count_nonzero(g[buf == 1]) > 0


def test_autograd_4pcf_matches_finite_differences():
    import torch

    from gramsci_b200 import autograd

    cat = catalogs.make("c3_4pcf", scale=0.02, seed=23)
    sp = catalogs.WORKLOADS["c3_4pcf"]
    rng = np.random.default_rng(104)
    w = catalogs.normalise(rng.lognormal(0, 0.3, cat.n), cat.n_data, cat.n_rand)
    dev = torch.device("cuda:0")
    xyz = torch.from_numpy(cat.xyz).to(dev)
    wt = torch.tensor(w, dtype=torch.float64, device=dev, requires_grad=True)
    args = (cat.n_data, sp["rmin"], sp["rmax"], sp["nbins"])
    outs = autograd.pcf4(wt, xyz, *args)
    cots = [torch.tensor(rng.normal(size=o.shape), device=dev) for o in outs]
    L = sum((c * o).sum() for c, o in zip(cots, outs))
    (g,) = torch.autograd.grad(L, wt)
    g = g.cpu().numpy()

    def loss(wv):
        o = autograd.pcf4(torch.tensor(wv, dtype=torch.float64, device=dev), xyz, *args)
        return float(sum((c * x).sum() for c, x in zip(cots, o)))

    nz = np.flatnonzero(g)
    assert len(nz) >= 32
    for k in rng.choice(nz, 32, replace=False):
        h = 0.5 * abs(w[k])
        wp, wm = w.copy(), w.copy()
        wp[k] += h
        wm[k] -= h
        fd = (loss(wp) - loss(wm)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-8 * max(abs(fd), abs(g[k])), (k, fd, g[k])


@pytest.mark.parametrize("order", [2, 3])
def test_autograd_matches_finite_differences(order):
    import torch

    from gramsci_b200 import autograd

    name = "c5_adjoint_2pcf" if order == 2 else "c5_adjoint_3pcf"
    cat, w, sp = _cat(name, 0.001, seed=21)
    dev = torch.device("cuda:0")
    xyz = torch.from_numpy(cat.xyz).to(dev)
    wt = torch.tensor(w, dtype=torch.float64, device=dev, requires_grad=True)
    f = autograd.pcf2 if order == 2 else autograd.pcf3
    args = (cat.n_data, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    N2, N3 = f(wt, xyz, *args)
    rng = np.random.default_rng(100 + order)
    c2 = torch.tensor(rng.normal(size=N2.shape), device=dev)
    c3 = torch.tensor(rng.normal(size=N3.shape), device=dev)
    L = (c2 * N2).sum() + (c3 * N3).sum()
    (g,) = torch.autograd.grad(L, wt)
    g = g.cpu().numpy()

    def loss(wv):
        a, b = f(torch.tensor(wv, dtype=torch.float64, device=dev), xyz, *args)
        return float((c2 * a).sum() + (c3 * b).sum())

    idx = rng.choice(len(w), 64, replace=False)
    for k in idx:
        h = 0.5 * abs(w[k])
        wp, wm = w.copy(), w.copy()
        wp[k] += h
        wm[k] -= h
        fd = (loss(wp) - loss(wm)) / (2 * h)
        scale = max(abs(fd), abs(g[k]), 1e-300)
        assert abs(fd - g[k]) <= 1e-8 * scale or (abs(fd) < 1e-30 and abs(g[k]) < 1e-30), (k, fd, g[k])


def test_autograd_through_normalisation():
    import torch

    from gramsci_b200 import autograd

    cat, _, sp = _cat("c5_adjoint_2pcf", 0.001, seed=22)
    dev = torch.device("cuda:0")
    xyz = torch.from_numpy(cat.xyz).to(dev)
    raw = torch.tensor(cat.w, dtype=torch.float64, device=dev, requires_grad=True)
    w = autograd.normalise(raw, cat.n_data)
    N2, N3 = autograd.pcf2(w, xyz, cat.n_data, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    N2.sum().backward()
    g = raw.grad.cpu().numpy()
    # the normalised galaxy weights sum to one whatever the raw weights, so
    # scaling all raw galaxy weights leaves N2 unchanged: zero directional
    # derivative along the raw galaxy weights
    d = float(np.dot(g[:cat.n_data], cat.w[:cat.n_data]))
    assert abs(d) <= 1e-9 * np.abs(g[:cat.n_data] * cat.w[:cat.n_data]).sum()
