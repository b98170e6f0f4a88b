"""CPU tests of the `gramsci` command's host side (libgramsci_host.so):
option parsing as the reference's parseOptions does it, list-directed
catalogue reading, weight normalisation, radial bin edges and the E14.7
output records."""
import os

import numpy as np
import pytest

from gramsci_b200 import catalogs, host


@pytest.mark.parametrize("v,s", [
    (1.0, " 0.1000000E+01"), (-0.5, "-0.5000000E+00"), (0.0, " 0.0000000E+00"),
    (123456789.0, " 0.1234568E+09"), (9.99999996, " 0.1000000E+02"), (0.1, " 0.1000000E+00"),
    (1e-300, " 0.1000000-299"), (1e100, " 0.1000000+101"), (float("nan"), "           NaN"),
    (float("inf"), "      Infinity"), (-float("inf"), "     -Infinity"),
    (-2.124343822e-07, "-0.2124344E-06"),
])
def test_e14_7(v, s):
    assert host.format_e14_7(v) == s


def test_options_defaults_and_six_character_match():
    o = host.parse_args(["-gal", "g", "-ran", "r", "-rmin", "1d1", "-rmax", "5.0E1", "-nbins_x",
                         "10", "-nmu", "4", "-2pcf", "-3pcf"])
    assert o.error == 0 and not o.help
    assert (o.gal, o.ran, o.out) == (b"g", b"r", b"result.txt")
    assert (o.rmin, o.rmax, o.nbins, o.nmu, o.rsd) == (10.0, 50.0, 10, 4, 1)
    assert (o.two_pcf, o.three_pcf, o.four_pcf, o.rancat) == (1, 1, 0, 1)


def test_options_errors():
    assert host.parse_args(["-gal", "g", "-rmin", "1"]).help == 1  # fewer than 6 arguments
    o = host.parse_args(["-gal", "g", "-ran", "r", "-rmin", "1", "-bogus", "-2pcf"])
    assert o.error == 1 and b"unknown option -bogus ignored" in o.message
    o = host.parse_args(["-gal", "g", "-ran", "r", "-rmin", "one", "-2pcf"])
    assert o.error == 2
    o = host.parse_args(["-gal", "g", "-ran", "r", "-nbins", "2.5", "-2pcf"])
    assert o.error == 2
    o = host.parse_args(["-cut", "3.loadnodes", "-rmin", "1", "-rmax", "2", "-2pcf"])
    assert o.cut_mode == 1 and o.out == b"3.loadnodes"


def test_read_catalogue_list_directed(tmp_path):
    g = tmp_path / "g.txt"
    g.write_text("1 2 3 1.0\n4.0d0, 5, 6, 2\n\n7 8\n9 3 extra ignored\n")
    r = tmp_path / "r.txt"
    r.write_text("0 0 0 1\n1 1 1 1\n")
    xyz, w, nd, nr = host.read_catalogue(str(g), str(r))
    # the blank line and the split record count as one value-read each, as
    # gfortran's list-directed count loop sees them
    assert (nd, nr) == (4, 2)
    assert np.array_equal(xyz[:3], [[1, 2, 3], [4, 5, 6], [7, 8, 9]])
    assert np.array_equal(w[:3], [1.0, 2.0, 3.0])
    assert np.array_equal(xyz[4:], [[0, 0, 0], [1, 1, 1]])


def test_read_catalogue_roundtrip(tmp_path):
    cat = catalogs.make("c1_2pcf", scale=0.01)
    gp, rp = tmp_path / "g", tmp_path / "r"
    catalogs.write_ascii(gp, cat.xyz[:cat.n_data], cat.w[:cat.n_data])
    catalogs.write_ascii(rp, cat.xyz[cat.n_data:], cat.w[cat.n_data:])
    xyz, w, nd, nr = host.read_catalogue(str(gp), str(rp))
    assert (nd, nr) == (cat.n_data, cat.n_rand)
    assert np.array_equal(xyz, cat.xyz) and np.array_equal(w, cat.w)


def test_radial_bins():
    e = host.radial_bins(10.0, 50.0, 10)
    assert np.array_equal(e, 10.0 + np.arange(11) * 40.0 / 10)
    el = host.radial_bins(1.0, 100.0, 2, logbins=True)
    assert np.allclose(el, [1.0, 10.0, 100.0], rtol=1e-15)


def test_writers_layout(tmp_path):
    nb, nm = 3, 2
    e = host.radial_bins(1.0, 10.0, nb)
    N2 = np.arange(nb * nm, dtype=float).reshape(nb, nm, order="F") + 1
    N3 = np.full((nb, nm), 2.0)
    p = tmp_path / "o2"
    assert host.write_2pcf(str(p), e, nb, nm, N2, N3) == 0
    lines = p.read_text().splitlines()
    assert lines[0] == " r1 min, r1 max, r2 min, r2 max, NN, RR, 2pcf (xi)"
    assert len(lines) == 1 + nb * nm
    # row order: radial bin outer, mu bin inner; columns 15 characters apart
    assert lines[1] == " ".join(host.format_e14_7(v) for v in
                                [1.0, 4.0, -1.0, 0.0, N2[0, 0], 2.0, N2[0, 0] / 2.0])
    assert lines[2].split()[2:4] == [host.format_e14_7(0.0).strip(), host.format_e14_7(1.0).strip()]
    nc = nb * (nb + 1) * (nb + 2) // 6
    p3 = tmp_path / "o3"
    assert host.write_3pcf(str(p3), e, nb, 1, np.ones((nc, 1)), np.ones((nc, 1))) == 0
    l3 = p3.read_text().splitlines()
    assert len(l3) == 1 + nc and len(l3[1].split()) == 9
    p3m = tmp_path / "o3m"
    assert host.write_3pcf(str(p3m), e, nb, nm, np.ones((nc, nm)), np.ones((nc, nm))) == 0
    l3m = p3m.read_text().splitlines()
    assert len(l3m) == 1 + nc * nm and len(l3m[1].split()) == 11
    nc4 = nb * (nb + 1) * (nb + 2) * (nb + 3) // 24
    p4 = tmp_path / "o4"
    z = np.ones((nc4, nb, nb))
    assert host.write_4pcf(str(p4), e, nb, z, z, np.ones((nc4, nb, nb, 6)), np.ones((nc4, nb, nb, 6))) == 0
    l4 = p4.read_text().splitlines()
    assert len(l4) == 1 + nc4 * nb * nb and len(l4[1].split()) == 14


def test_cli_help_and_unknown_option():
    import subprocess

    r = subprocess.run([host.CLI_PATH, "-help"], capture_output=True, text=True)
    assert r.returncode == 0 and "usage" in r.stdout
    r = subprocess.run([host.CLI_PATH, "-gal", "a", "-ran", "b", "-rmin", "1", "-what", "-2pcf"],
                       capture_output=True, text=True)
    assert r.returncode == 0 and "unknown option -what ignored" in r.stdout
    r = subprocess.run([host.CLI_PATH, "-gal", "a", "-ran", "b", "-rmin", "x", "-rmax", "2"],
                       capture_output=True, text=True)
    assert r.returncode == 2


def test_cli_without_gpu_fails_loudly(tmp_path):
    """On a host without a CUDA device the command stops with status 1 and
    names the cause; no table is written (there is no host fallback)."""
    import subprocess

    import torch

    if torch.cuda.is_available():
        pytest.skip("needs a host without a GPU")
    g, r, out = tmp_path / "g", tmp_path / "r", tmp_path / "out"
    g.write_text("1 2 3 1\n4 5 6 1\n")
    r.write_text("1 2 4 1\n4 5 7 1\n")
    res = subprocess.run([host.CLI_PATH, "-gal", str(g), "-ran", str(r), "-rmin", "1", "-rmax", "10",
                          "-nbins", "3", "-2pcf", "-out", str(out)],
                         capture_output=True, text=True, timeout=120)
    assert res.returncode == 1
    assert "gr_create failed (-3): no usable CUDA device" in res.stderr
    assert not out.exists()


def test_tables_read_by_the_reference_harness(tmp_path):
    """The reference's own test harness reads result tables with
    np.loadtxt(out, skiprows=1) and averages columns 4 / 5 (2PCF, N2 / N3)
    and 6 / 7 (3PCF) (tests/run_correlation_tests.py:24-40).  Tables written
    here parse the same way, with the ratio column NaN or Infinity where
    N3 is 0, and the column means agree with the histograms to E14.7's 7
    digits."""
    rng = np.random.default_rng(4)
    e = host.radial_bins(1.0, 30.0, 10)
    N2, N3 = rng.uniform(1e-8, 1e-6, (10, 10)), rng.uniform(1e-8, 1e-6, (10, 10))
    N3[0, 0] = 0.0
    N2[1, 1] = N3[1, 1] = 0.0
    p2 = tmp_path / "tmp_2pcf.out"
    assert host.write_2pcf(str(p2), e, 10, 10, N2, N3) == 0
    t2 = np.loadtxt(p2, skiprows=1)
    assert t2.shape == (100, 7)
    np.testing.assert_allclose(np.mean(t2[:, 4]), N2.mean(), rtol=1e-7)
    np.testing.assert_allclose(np.mean(t2[:, 5]), N3.mean(), rtol=1e-7)
    assert np.isinf(t2[0, 6]) and np.isnan(t2[11, 6])
    e6 = host.radial_bins(1.0, 30.0, 6)
    nc = 6 * 7 * 8 // 6
    M2, M3 = rng.uniform(1e-13, 1e-11, (nc, 1)), rng.uniform(1e-13, 1e-11, (nc, 1))
    p3 = tmp_path / "tmp_3pcf.out"
    assert host.write_3pcf(str(p3), e6, 6, 1, M2, M3) == 0
    t3 = np.loadtxt(p3, skiprows=1)
    assert t3.shape == (nc, 9)
    np.testing.assert_allclose(np.mean(t3[:, 6]), M2.mean(), rtol=1e-7)
    np.testing.assert_allclose(np.mean(t3[:, 7]), M3.mean(), rtol=1e-7)


def _e14_7_model(v):
    """Fortran E14.7 of a finite double with a two-digit exponent, from the
    exact decimal value: 0.ddddddd x 10^e with 0.1 <= mantissa < 1, rounded
    to nearest, right-aligned in 14 characters."""
    from decimal import ROUND_HALF_EVEN, Decimal

    if v == 0.0:
        return " 0.0000000E+00"
    d = abs(Decimal(v))
    e = d.adjusted() + 1  # d = m * 10^e with 0.1 <= m < 1
    m = (d.scaleb(-e)).quantize(Decimal("1e-7"), rounding=ROUND_HALF_EVEN)
    if m >= 1:
        m, e = Decimal("0.1000000"), e + 1
    body = f"{m:.7f}E{'+' if e >= 0 else '-'}{abs(e):02d}"
    return ("-" if v < 0 else "") + body.rjust(13 if v < 0 else 14)


def test_e14_7_matches_exact_decimal_model():
    rng = np.random.default_rng(7)
    vals = rng.uniform(-1, 1, 4000) * 10.0 ** rng.integers(-95, 95, 4000)
    # values next to a rounding boundary of the 7th digit and to a power of 10
    vals = np.concatenate([vals, [9.99999995, 9.9999999499999, 0.99999995, 1.00000005e-3,
                                  -9.99999996e50, 1e-99, 9.99999e98]])
    for v in vals:
        assert host.format_e14_7(float(v)) == _e14_7_model(float(v)), repr(v)


def test_read_catalogue_number_forms_roundtrip(tmp_path):
    """17-significant-digit values in the forms list-directed input takes
    (plain, E or D exponent, lower or upper case) and with space, comma or
    tab separators read back bit-exactly."""
    rng = np.random.default_rng(9)
    n = 600
    vals = rng.uniform(-1, 1, (n, 4)) * 10.0 ** rng.integers(-30, 30, (n, 4))
    forms = [lambda x: f"{x:.17g}", lambda x: f"{x:.16E}", lambda x: f"{x:.16e}".replace("e", "d"),
             lambda x: f"{x:.16E}".replace("E", "D")]
    seps = [" ", ", ", "\t", "   "]
    lines = []
    for i, row in enumerate(vals):
        f, s = forms[i % len(forms)], seps[(i // len(forms)) % len(seps)]
        lines.append(s.join(f(float(x)) for x in row))
    g, r = tmp_path / "g", tmp_path / "r"
    g.write_text("\n".join(lines[:400]) + "\n")
    r.write_text("\n".join(lines[400:]) + "\n")
    xyz, w, nd, nr = host.read_catalogue(str(g), str(r))
    assert (nd, nr) == (400, 200)
    assert np.array_equal(xyz, vals[:, :3]) and np.array_equal(w, vals[:, 3])
