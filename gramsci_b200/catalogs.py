"""Seeded synthetic catalogues for the benchmark and parity workloads.

The reference reads ASCII catalogues of ``x y z w`` records (src/gramsci.F90:
1364-1388).  Here catalogues are generated in memory with numpy's seeded
``default_rng`` and can be written in that same ASCII layout.  Positions and
weights are FP64.

Workloads (sizes are the full ones; ``scale`` shrinks the point counts and the
box volume together so the number density, hence the neighbour counts per
point, stays the same):

* ``c1_2pcf``   20,000 uniform galaxies + 50,000 uniform randoms in [0,1000]^3,
                unit weights, rmin 10, rmax 50, 10 bins, nmu 1.
* ``c2_3pcf``   Neyman-Scott galaxies (10,000 parents, Poisson(10) children,
                Gaussian sigma 4) + 300,000 randoms in [0,1000]^3, lognormal
                (0, 0.3) weights, rmin 5, rmax 25, 8 bins, nmu 5.
* ``c3_4pcf``   Neyman-Scott (1,500 parents, Poisson(20), sigma 3) + 90,000
                randoms in [0,300]^3, unit weights, rmin 2, rmax 12, 4 bins.
* ``c4_batched`` Neyman-Scott with parent density rising linearly along x by a
                factor 8 (about 4,000,000 galaxies) + 8,000,000 randoms in
                [0,2000]^3, rmin 10, rmax 60, 12 bins, nmu 10, 5^3 regions.
* ``c5_adjoint`` Neyman-Scott (sigma 5, about 1,000,000 galaxies, lognormal
                weights) + 2,000,000 randoms in [0,1000]^3; weighted 2PCF
                (10, 40, 10 bins, nmu 4) and weighted 3PCF (10, 30, 6 bins).
"""
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Catalogue:
    """Galaxies first, then randoms, as the reference orders them."""

    xyz: np.ndarray          # (N, 3) float64
    w: np.ndarray            # (N,) float64, raw (un-normalised) weights
    n_data: int
    n_rand: int
    buffer: np.ndarray = None  # (N,) int32 0/1 or None
    meta: dict = field(default_factory=dict)

    @property
    def n(self):
        return self.n_data + self.n_rand


def uniform(rng, n, lo, hi):
    return rng.uniform(lo, hi, size=(n, 3))


def neyman_scott(rng, n_parents, mean_children, sigma, lo, hi, ramp=None):
    """Poisson parents in the box, Poisson(mean) children with isotropic
    Gaussian offsets.  ``ramp`` = max/min ratio of a parent density rising
    linearly along x (inverse-CDF sampling), or None for uniform parents."""
    L = hi - lo
    parents = rng.uniform(lo, hi, size=(n_parents, 3))
    if ramp is not None and ramp != 1.0:
        # p(u) proportional to 1 + (ramp-1) u on [0,1]
        a = ramp - 1.0
        u = rng.uniform(0.0, 1.0, size=n_parents)
        x01 = (-1.0 + np.sqrt(1.0 + a * (a + 2.0) * u)) / a
        parents[:, 0] = lo + L * x01
    nchild = rng.poisson(mean_children, size=n_parents)
    pid = np.repeat(np.arange(n_parents), nchild)
    pts = parents[pid] + rng.normal(0.0, sigma, size=(pid.size, 3))
    return pts


def _lognormal(rng, n, sigma=0.3):
    return rng.lognormal(0.0, sigma, size=n)


WORKLOADS = {
    "c1_2pcf": dict(rmin=10.0, rmax=50.0, nbins=10, nmu=1, query="2pcf"),
    "c2_3pcf": dict(rmin=5.0, rmax=25.0, nbins=8, nmu=5, query="3pcf"),
    "c3_4pcf": dict(rmin=2.0, rmax=12.0, nbins=4, nmu=1, query="4pcf"),
    "c4_batched": dict(rmin=10.0, rmax=60.0, nbins=12, nmu=10, query="2pcf", nsplit=5),
    "c5_adjoint_2pcf": dict(rmin=10.0, rmax=40.0, nbins=10, nmu=4, query="2pcf"),
    "c5_adjoint_3pcf": dict(rmin=10.0, rmax=30.0, nbins=6, nmu=1, query="3pcf"),
}


def make(name, scale=1.0, seed=None):
    """Build the catalogue of a named workload.  ``scale`` in (0, 1] shrinks
    the counts by ``scale`` and the box edge by ``scale ** (1/3)``."""
    s = float(scale)
    e = s ** (1.0 / 3.0)
    if name == "c1_2pcf":
        rng = np.random.default_rng(1 if seed is None else seed)
        L = 1000.0 * e
        g = uniform(rng, int(round(20000 * s)), 0.0, L)
        r = uniform(rng, int(round(50000 * s)), 0.0, L)
        wg, wr = np.ones(len(g)), np.ones(len(r))
    elif name == "c2_3pcf":
        rng = np.random.default_rng(2 if seed is None else seed)
        L = 1000.0 * e
        g = neyman_scott(rng, int(round(10000 * s)), 10.0, 4.0, 0.0, L)
        r = uniform(rng, int(round(300000 * s)), 0.0, L)
        wg, wr = _lognormal(rng, len(g)), _lognormal(rng, len(r))
    elif name == "c3_4pcf":
        rng = np.random.default_rng(3 if seed is None else seed)
        L = 300.0 * e
        g = neyman_scott(rng, int(round(1500 * s)), 20.0, 3.0, 0.0, L)
        r = uniform(rng, int(round(90000 * s)), 0.0, L)
        wg, wr = np.ones(len(g)), np.ones(len(r))
    elif name == "c4_batched":
        rng = np.random.default_rng(4 if seed is None else seed)
        L = 2000.0 * e
        g = neyman_scott(rng, int(round(400000 * s)), 10.0, 5.0, 0.0, L, ramp=8.0)
        r = uniform(rng, int(round(8000000 * s)), 0.0, L)
        wg, wr = np.ones(len(g)), np.ones(len(r))
    elif name in ("c5_adjoint", "c5_adjoint_2pcf", "c5_adjoint_3pcf"):
        rng = np.random.default_rng(5 if seed is None else seed)
        L = 1000.0 * e
        g = neyman_scott(rng, int(round(100000 * s)), 10.0, 5.0, 0.0, L)
        r = uniform(rng, int(round(2000000 * s)), 0.0, L)
        wg, wr = _lognormal(rng, len(g)), np.ones(len(r))
    else:
        raise KeyError(name)
    xyz = np.concatenate([g, r]).astype(np.float64)
    w = np.concatenate([wg, wr]).astype(np.float64)
    cat = Catalogue(xyz=np.ascontiguousarray(xyz), w=w, n_data=len(g), n_rand=len(r),
                    meta=dict(name=name, scale=s, box=L))
    return cat


def normalise(w, n_data, n_rand):
    """Signed normalised weights as the reference forms them after reading
    (src/gramsci.F90:1390-1391): galaxy weights over their sum, random weights
    negated over theirs.  Sums are left to right."""
    w = np.asarray(w, np.float64)
    out = np.empty_like(w)
    # np.cumsum accumulates strictly left to right (no pairwise summation)
    sg = float(np.cumsum(w[:n_data])[-1]) if n_data else 0.0
    sr = float(np.cumsum(w[n_data:n_data + n_rand])[-1]) if n_rand else 0.0
    out[:n_data] = w[:n_data] / sg if n_data else w[:n_data]
    out[n_data:n_data + n_rand] = -1.0 * w[n_data:n_data + n_rand] / sr if n_rand else 0.0
    return out


def write_ascii(path, xyz, w):
    """Write ``x y z w`` records, one point per line, full FP64 precision."""
    a = np.column_stack([np.asarray(xyz, np.float64).reshape(-1, 3), np.asarray(w, np.float64)])
    np.savetxt(path, a, fmt="%.17g")
