"""C ABI checks that need no GPU: the library loads and exports every entry
point declared in include/gramsci_cuda.h, and the ctypes binding declares
exactly those."""
import ctypes
import os
import re

import pytest
import torch

from gramsci_b200 import _native

HEADER = _native.HEADER


def declared():
    with open(HEADER) as f:
        src = f.read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gr_[a-z0-9_]+)\s*\(", src)))


def test_header_declarations_bound():
    names = declared()
    assert "gr_count_3pcf" in names and "gr_create" in names
    assert sorted(_native.SIGNATURES) == names


def test_library_exports_every_symbol():
    lib = ctypes.CDLL(_native.LIB_PATH)
    for name in declared():
        assert hasattr(lib, name), name


def test_version_string():
    assert "sm_100a" in _native.load().gr_version().decode()


def test_null_context_is_rejected():
    lib = _native.load()
    assert lib.gr_destroy(None) == _native.GR_E_ARG
    assert lib.gr_set_bins(None, 1.0, 2.0, 3, 1, 0) == _native.GR_E_ARG
    assert lib.gr_count_3pcf(None, None, None, None, None) == _native.GR_E_ARG


def test_library_is_in_tree():
    assert os.path.dirname(_native.LIB_PATH).endswith(os.path.join("gramsci_b200", "lib"))


def test_missing_library_raises(tmp_path, monkeypatch):
    monkeypatch.setattr(_native, "_lib", None)
    with pytest.raises(ImportError, match="missing"):
        _native.load(str(tmp_path / "libgramsci_cuda.so"))


@pytest.mark.skipif(torch.cuda.is_available(), reason="needs a host without a GPU")
def test_no_device_fails_loudly():
    """Without a CUDA device a context cannot be made: the counts are never
    computed by a host fallback."""
    from gramsci_b200 import api

    with pytest.raises(_native.GramsciError, match="gr_create"):
        api.Context(0)


def test_header_constants_match_binding():
    with open(HEADER) as f:
        defs = dict(re.findall(r"^#define (GR_[A-Z0-9_]+) \(?(-?\d+)\)?", f.read(), flags=re.M))
    assert {"GR_OK", "GR_E_CUDA", "GR_OPT_CLIQUE_MODE", "GR_NOALLOC_MAX_BINS"} <= set(defs)
    for name, v in defs.items():
        assert getattr(_native, name) == int(v), name


class _FakeLib:
    """Records gr_set_option calls; every call succeeds."""

    def __init__(self):
        self.calls = []

    def gr_set_option(self, h, key, value):
        self.calls.append((key, value))
        return 0


def test_option_setters_pass_header_keys():
    from gramsci_b200 import api

    ctx = object.__new__(api.Context)
    ctx._lib, ctx._h = _FakeLib(), None
    ctx.set_precision("f64")
    ctx.set_autotune("off")
    ctx.set_autotune(3)
    ctx.set_keep_graph(True)
    ctx.set_clique_mode("geometric")
    ctx.set_clique_mode("hash")
    assert ctx._lib.calls == [(_native.GR_OPT_PRECISION, 1), (_native.GR_OPT_AUTOTUNE, 0),
                              (_native.GR_OPT_AUTOTUNE, 5), (_native.GR_OPT_KEEP_GRAPH, 1),
                              (_native.GR_OPT_CLIQUE_MODE, 2), (_native.GR_OPT_CLIQUE_MODE, 1)]
    assert (_native.GR_OPT_KEEP_GRAPH, _native.GR_OPT_CLIQUE_MODE) == (4, 5)
