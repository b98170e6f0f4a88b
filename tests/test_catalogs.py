"""The seeded synthetic workloads: sizes and distributions as the benchmark
configurations describe them, determinism, and the constant number density
that ``scale`` keeps (so neighbour counts per point match at reduced scale)."""
import numpy as np
import pytest

from gramsci_b200 import catalogs


def test_sizes_of_the_full_workloads():
    c1 = catalogs.make("c1_2pcf")
    assert (c1.n_data, c1.n_rand) == (20000, 50000)
    assert np.all(c1.w == 1.0) and c1.xyz.min() >= 0.0 and c1.xyz.max() <= 1000.0
    c2 = catalogs.make("c2_3pcf")
    assert c2.n_rand == 300000 and abs(c2.n_data - 100000) < 1500  # 10,000 x Poisson(10)
    assert abs(np.std(np.log(c2.w)) - 0.3) < 0.01                  # lognormal(0, 0.3)
    c3 = catalogs.make("c3_4pcf")
    assert c3.n_rand == 90000 and abs(c3.n_data - 30000) < 800    # 1,500 x Poisson(20)
    assert c3.meta["box"] == 300.0 and np.all(c3.w == 1.0)


def test_seeds_and_scale():
    a = catalogs.make("c2_3pcf", scale=0.05)
    b = catalogs.make("c2_3pcf", scale=0.05)
    c = catalogs.make("c2_3pcf", scale=0.05, seed=77)
    assert np.array_equal(a.xyz, b.xyz) and np.array_equal(a.w, b.w)
    assert not np.array_equal(a.xyz[:10], c.xyz[:10])
    full = catalogs.make("c2_3pcf")
    dens_full = full.n_rand / full.meta["box"] ** 3
    dens_small = a.n_rand / a.meta["box"] ** 3
    assert abs(dens_small / dens_full - 1.0) < 1e-3


def test_batched_catalogue_ramp():
    cat = catalogs.make("c4_batched", scale=0.02)
    box = cat.meta["box"]
    x = cat.xyz[:cat.n_data, 0]
    inner = (x > 0.0) & (x < box)
    lo = np.count_nonzero(inner & (x < 0.1 * box))
    hi = np.count_nonzero(inner & (x > 0.9 * box))
    # parent density 1 + 7u along x (u in [0, 1]): the last tenth of the box
    # holds (1 + 7 * 0.95) / (1 + 7 * 0.05) = 5.7 times the galaxies of the first
    assert 4.0 < hi / lo < 7.0
    assert cat.n_rand == 160000


@pytest.mark.parametrize("name", ["c1_2pcf", "c2_3pcf", "c5_adjoint_3pcf"])
def test_normalise_follows_the_reference_rule(name):
    cat = catalogs.make(name, scale=0.01)
    w = catalogs.normalise(cat.w, cat.n_data, cat.n_rand)
    assert np.all(w[:cat.n_data] > 0) and np.all(w[cat.n_data:] < 0)
    assert abs(w[:cat.n_data].sum() - 1.0) < 1e-12 and abs(w[cat.n_data:].sum() + 1.0) < 1e-12


def test_torch_normalise_matches_and_differentiates():
    """autograd.normalise (torch, differentiable) equals catalogs.normalise,
    and its Jacobian is the quotient rule of w_k / sum(w) per catalogue."""
    import torch

    from gramsci_b200 import autograd

    rng = np.random.default_rng(5)
    nd, nr = 4, 3
    raw = rng.lognormal(0, 0.3, nd + nr)
    t = torch.tensor(raw, dtype=torch.float64, requires_grad=True)
    out = autograd.normalise(t, nd)
    np.testing.assert_allclose(out.detach().numpy(), catalogs.normalise(raw, nd, nr), rtol=1e-15)
    J = torch.autograd.functional.jacobian(lambda x: autograd.normalise(x, nd), t).numpy()
    for lo, hi, sign in ((0, nd, 1.0), (nd, nd + nr, -1.0)):
        S = raw[lo:hi].sum()
        for i in range(lo, hi):
            for k in range(lo, hi):
                exp = sign * ((i == k) / S - raw[i] / S ** 2)
                assert abs(J[i, k] - exp) <= 1e-14 * max(1.0, abs(exp)), (i, k)
        # no coupling between the two catalogues
        other = [k for k in range(nd + nr) if not lo <= k < hi]
        assert np.all(J[lo:hi][:, other] == 0)
