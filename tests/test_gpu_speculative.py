"""Rebuilds without host waits (3PCF and 2PCF): a count of a catalogue seen before
takes the grid of the last bounding box and fills the graph in the scratch
area as it is, and a device flag sends the call round again with waits when
the bounding box changed or the scratch area was too small.  Every case is
checked against the oracle: repeated counts of one catalogue, another
catalogue of the same size and bounding box (the captured rebuild of the
previous call replayed), a denser catalogue with the same bounding box
(scratch too small), and a catalogue with another bounding box (grid
changed)."""
import numpy as np
import pytest

from gramsci_b200 import api, catalogs

pytestmark = pytest.mark.gpu

RMIN, RMAX, NBINS, NMU = 5.0, 25.0, 8, 5


def _with_corners(rng, interior, box):
    corners = np.array([[x, y, z] for x in (0.0, box) for y in (0.0, box) for z in (0.0, box)])
    return np.vstack([corners, interior])


def _check(ctx, oracle, xyz, n_data, rng):
    n = len(xyz)
    w = catalogs.normalise(rng.lognormal(0, 0.3, n), n_data, n - n_data)
    ctx.set_catalog(xyz, w, n_data)
    ref = oracle.Graph(xyz, RMIN, RMAX, NBINS, NMU).pcf3(w, n_data)
    for _ in range(2):
        got = ctx.count_3pcf()
        assert np.array_equal(got["counts"], ref["counts"])
        scale = np.abs(ref["catsum"]).max()
        assert np.all(np.abs(got["catsum"] - ref["catsum"]) <= 1e-12 * scale)
    assert int(ref["counts"].sum()) > 0


def test_repeats_and_scratch_overflow(oracle):
    rng = np.random.default_rng(31)
    box = 300.0
    a = _with_corners(rng, rng.uniform(0.0, box, (2992, 3)), box)
    a2 = _with_corners(rng, rng.uniform(0.0, box, (2992, 3)), box)  # same box and size
    b = _with_corners(rng, rng.uniform(100.0, 200.0, (2992, 3)), box)  # same box, dense
    with api.Context(0) as ctx:
        ctx.set_bins(RMIN, RMAX, NBINS, NMU)
        _check(ctx, oracle, a, 1000, rng)
        # other points, same configuration: the captured rebuild of the
        # previous call is replayed
        _check(ctx, oracle, a2, 1000, rng)
        _check(ctx, oracle, b, 1000, rng)
        _check(ctx, oracle, a, 1000, rng)


def test_changed_bounding_box(oracle):
    rng = np.random.default_rng(32)
    a = rng.uniform(0.0, 300.0, (3000, 3))
    c = rng.uniform(0.0, 360.0, (3000, 3))
    with api.Context(0) as ctx:
        ctx.set_bins(RMIN, RMAX, NBINS, NMU)
        _check(ctx, oracle, a, 1000, rng)
        _check(ctx, oracle, c, 1000, rng)
        _check(ctx, oracle, a, 1000, rng)


def _check2(ctx, oracle, xyz, n_data, rng):
    n = len(xyz)
    w = catalogs.normalise(rng.lognormal(0, 0.3, n), n_data, n - n_data)
    ctx.set_catalog(xyz, w, n_data)
    ref = oracle.Graph(xyz, RMIN, RMAX, NBINS, NMU).pcf2(w, n_data)
    for _ in range(2):
        got = ctx.count_2pcf()
        assert np.array_equal(got["counts"], ref["counts"])
        scale = np.abs(ref["catsum"]).max()
        assert np.all(np.abs(got["catsum"] - ref["catsum"]) <= 1e-12 * scale)
    assert int(ref["counts"].sum()) > 0


def test_2pcf_rebuilds(oracle):
    """The 2PCF takes the grid of the last bounding box too: repeats, another
    catalogue of the same size and box (the captured index replayed), a
    changed box, on a sparse grid and on a dense one (cells of rmax/2)."""
    rng = np.random.default_rng(33)
    a = _with_corners(rng, rng.uniform(0.0, 300.0, (2992, 3)), 300.0)
    a2 = _with_corners(rng, rng.uniform(0.0, 300.0, (2992, 3)), 300.0)
    c = rng.uniform(0.0, 360.0, (3000, 3))
    d = _with_corners(rng, rng.uniform(0.0, 150.0, (19992, 3)), 150.0)
    d2 = _with_corners(rng, rng.uniform(0.0, 150.0, (19992, 3)), 150.0)
    with api.Context(0) as ctx:
        ctx.set_bins(RMIN, RMAX, NBINS, NMU)
        for xyz in (a, a2, c, a, d, d2, d):
            _check2(ctx, oracle, xyz, len(xyz) // 3, rng)


def test_mixed_calls_keep_their_rebuilds_apart(oracle):
    """2PCF and 3PCF counts, bin and precision changes interleaved on one
    context (each kind keeps its own captured rebuild, keyed by what it
    reads): every result against the oracle."""
    rng = np.random.default_rng(34)
    a = _with_corners(rng, rng.uniform(0.0, 300.0, (2992, 3)), 300.0)
    b = _with_corners(rng, rng.uniform(0.0, 300.0, (2992, 3)), 300.0)
    n_data = 1000
    with api.Context(0) as ctx:
        for xyz, bins, prec in ((a, (RMIN, RMAX, NBINS, NMU), "f32"),
                                (b, (RMIN, RMAX, NBINS, NMU), "f32"),
                                (b, (4.0, 20.0, 6, 3), "f32"),
                                (a, (4.0, 20.0, 6, 3), "f64"),
                                (a, (RMIN, RMAX, NBINS, NMU), "f32")):
            ctx.set_precision(prec)
            ctx.set_bins(*bins)
            w = catalogs.normalise(rng.lognormal(0, 0.3, len(xyz)), n_data, len(xyz) - n_data)
            ctx.set_catalog(xyz, w, n_data)
            G = oracle.Graph(xyz, *bins)
            ref2, ref3 = G.pcf2(w, n_data), G.pcf3(w, n_data)
            for _ in range(2):
                for got, ref in ((ctx.count_3pcf(), ref3), (ctx.count_2pcf(), ref2)):
                    assert np.array_equal(got["counts"], ref["counts"])
                    scale = np.abs(ref["catsum"]).max()
                    assert np.all(np.abs(got["catsum"] - ref["catsum"]) <= 1e-12 * scale)
