"""The C headers as a C or cgo user includes them: both compile as C99 and
C++11 with warnings as errors, and a C program linked against the two
in-tree libraries calls entry points that need no GPU (version string,
argument rejection, radial bin edges, the table number format)."""
import os
import shutil
import subprocess

import pytest

from gramsci_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.dirname(_native.LIB_PATH)
HEADERS = ["gramsci_cuda.h", "gramsci_host.h"]

pytestmark = pytest.mark.skipif(shutil.which("gcc") is None or shutil.which("g++") is None,
                                reason="needs gcc and g++")

PROGRAM = r"""
#include <stdio.h>
#include <string.h>
#include "gramsci_cuda.h"
#include "gramsci_host.h"

int main(void) {
    double e[4];
    char s[16];
    if (strstr(gr_version(), "sm_100a") == NULL) return 1;
    if (gr_destroy(NULL) != GR_E_ARG) return 2;
    grh_radial_bins(1.0, 4.0, 3, 0, e);
    if (e[0] != 1.0 || e[1] != 2.0 || e[2] != 3.0 || e[3] != 4.0) return 3;
    grh_format_e14_7(0.5, s);
    printf("[%s]\n", s);
    return 0;
}
"""


@pytest.mark.parametrize("header", HEADERS)
@pytest.mark.parametrize("lang,std", [("c", "-std=c99"), ("c++", "-std=c++11")])
def test_header_compiles(header, lang, std):
    cc = "gcc" if lang == "c" else "g++"
    r = subprocess.run([cc, std, "-Wall", "-Wextra", "-Werror", "-pedantic", "-fsyntax-only",
                        "-x", lang, os.path.join(INC, header)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_c_program_links_and_runs(tmp_path):
    src = tmp_path / "bind.c"
    exe = tmp_path / "bind"
    src.write_text(PROGRAM)
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", INC, str(src), "-o", str(exe),
                        "-L", LIBDIR, "-lgramsci_cuda", "-lgramsci_host",
                        "-Wl,-rpath," + LIBDIR], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.returncode, r.stderr)
    line = r.stdout.strip()
    # table numbers are written in Fortran's E14.7 form
    assert line == "[ 0.5000000E+00]"
