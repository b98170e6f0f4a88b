"""Triangle rows of every length: a sparse background with a tight clump of
1,100 points, so that upper rows run from a few entries to more than 1,024.
Rows up to 256 entries take the main launch, longer rows up to 1,024 the
second (geometric) launch, and the longest the global-memory path; the 3PCF
counts, sums and the weight adjoint equal the oracle's."""
import numpy as np
import pytest

from gramsci_b200 import catalogs

pytestmark = pytest.mark.gpu

RMIN, RMAX, NBINS = 0.5, 10.0, 4


def _catalogue():
    rng = np.random.default_rng(41)
    bg = rng.uniform(0.0, 60.0, (2000, 3))
    d = rng.normal(size=(1100, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    clump = 30.0 + d * (2.0 * rng.random(1100) ** (1.0 / 3.0))[:, None]
    xyz = np.vstack([bg, clump])
    n_data = 1500
    w = catalogs.normalise(rng.lognormal(0, 0.3, len(xyz)), n_data, len(xyz) - n_data)
    return xyz, w, n_data


@pytest.mark.parametrize("nmu", [1, 3])
def test_3pcf_long_rows(gpu_ctx, oracle, nmu):
    xyz, w, nd = _catalogue()
    gpu_ctx.set_catalog(xyz, w, nd)
    gpu_ctx.set_bins(RMIN, RMAX, NBINS, nmu)
    got = gpu_ctx.count_3pcf()
    G = oracle.Graph(xyz, RMIN, RMAX, NBINS, nmu)
    ref = G.pcf3(w, nd)
    assert np.array_equal(got["counts"], ref["counts"])
    scale = np.abs(ref["catsum"]).max()
    assert np.all(np.abs(got["catsum"] - ref["catsum"]) <= 1e-12 * scale)
    rp = G.csr()[0]
    assert np.diff(rp).max() > 1024  # the longest rows exceed both launches' capacity
    if nmu == 1:
        rng = np.random.default_rng(42)
        c2 = rng.normal(size=got["N2"].shape)
        c3 = rng.normal(size=got["N3"].shape)
        g = gpu_ctx.adjoint_3pcf(c2, c3)
        gr = G.adjoint3(w, nd, c2, c3)
        assert np.all(np.abs(g - gr) <= 1e-12 * np.abs(gr).max())
