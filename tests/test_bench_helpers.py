"""bench.py's CPU-side helpers: the parity record printed beside the GPU
numbers (counts identical or not, relative error of the category sums per
bin, N2 against the sum of absolute category sums) and the seeded sub-cube
that bounds the CPU baselines (inner roots, a buffer shell of rmax)."""
import numpy as np

import bench
from gramsci_b200 import catalogs


def _result(rng, shape):
    counts = rng.integers(1, 100, size=shape + (4,))
    catsum = rng.uniform(1e-6, 1e-3, size=shape + (4,)) * np.array([1, -1, -1, 1])
    return {"counts": counts, "catsum": catsum, "N2": catsum.sum(axis=-1), "N3": catsum[..., 3]}


def test_parity_record_identical_and_perturbed():
    rng = np.random.default_rng(1)
    ref = _result(rng, (8, 5))
    same = bench.parity_record(ref, ref)
    assert same["counts_exact"] and same["max_rel_catsum"] == 0.0 and same["max_rel_N2"] == 0.0
    assert len(same["per_bin_max_rel"]) == 40 and max(same["per_bin_max_rel"]) == 0.0
    got = {k: v.copy() for k, v in ref.items()}
    got["catsum"][3, 2, 1] *= 1 + 1e-10
    got["counts"][0, 0, 0] += 1
    rec = bench.parity_record(got, ref)
    assert not rec["counts_exact"]
    assert abs(rec["max_rel_catsum"] - 1e-10) < 1e-12
    # bin (3, 2) in Fortran order: index 3 + 8 * 2
    per = rec["per_bin_max_rel"]
    assert per[3 + 8 * 2] > 0 and sum(1 for x in per if x > 0) == 1


def test_subcube_marks_the_shell_as_buffer():
    cat = catalogs.make("c1_2pcf", scale=0.2)
    w = catalogs.normalise(cat.w, cat.n_data, cat.n_rand)
    xs, ws, bs, nd, centre = bench.subcube(cat, w, 50.0, 200.0, seed=3)
    d = np.abs(xs - np.array(centre)).max(axis=1)
    assert np.all(d < 150.0)
    assert np.array_equal(bs == 0, d < 100.0)
    # galaxies first, in catalogue order
    assert nd == int(np.sum(ws > 0)) and np.all(ws[:nd] > 0) and np.all(ws[nd:] < 0)
    assert 0 < bs.sum() < len(bs)
