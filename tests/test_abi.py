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


def _prototypes():
    with open(HEADER) as f:
        src = re.sub(r"/\*.*?\*/", "", f.read(), flags=re.S)
    src = re.sub(r"^\s*#.*$", "", src, flags=re.M)
    out = {}
    for ret, name, args in re.findall(r"([A-Za-z_][\w\s\*]*?)\b(gr_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;",
                                      src, flags=re.S):
        params = [] if args.strip() in ("", "void") else [a.strip() for a in args.split(",")]
        types = [" ".join(re.match(r"(.*?)\w+$", p, flags=re.S).group(1).split()) for p in params]
        out[name] = (" ".join(ret.split()), types)
    return out


def _kind_c(t):
    t = t.replace("const ", "").replace(" *", "*").strip()
    if t.endswith("*"):
        return "ptr"
    return {"int": ("int", 4), "int32_t": ("int", 4), "int64_t": ("int", 8),
            "double": ("float", 8)}[t]


def _kind_ctypes(c):
    if c in (ctypes.c_void_p, ctypes.c_char_p) or hasattr(c, "_type_") and isinstance(c._type_, type):
        return "ptr"
    kind = "float" if c in (ctypes.c_double, ctypes.c_float) else "int"
    return (kind, ctypes.sizeof(c))


def test_binding_signatures_match_prototypes():
    """Every ctypes signature agrees with its C prototype: pointers for
    pointers, and scalars of the same kind and width (a narrower integer
    here would silently truncate a size)."""
    protos = _prototypes()
    assert sorted(protos) == sorted(_native.SIGNATURES)
    for name, (ret, types) in protos.items():
        res, argtypes = _native.SIGNATURES[name]
        assert [_kind_c(t) for t in types] == [_kind_ctypes(a) for a in argtypes], name
        assert _kind_c(ret) == _kind_ctypes(res), name


def _struct_cases():
    from gramsci_b200 import host

    return [("gramsci_cuda.h", "gr_stats", _native.GrStats),
            ("gramsci_host.h", "grh_options", host.Options)]


@pytest.mark.parametrize("header,cname,cls", _struct_cases(), ids=["gr_stats", "grh_options"])
def test_struct_layout(tmp_path, header, cname, cls):
    """The C compiler's layout of a struct crossing the ABI (size and every
    field offset) equals the ctypes structure's."""
    import shutil
    import subprocess

    if shutil.which("gcc") is None:
        pytest.skip("needs gcc")
    fields = [f for f, _ in cls._fields_]
    prog = (f"#include <stdio.h>\n#include <stddef.h>\n#include \"{header}\"\n"
            f"int main(void) {{\n  printf(\"%zu\\n\", sizeof({cname}));\n"
            + "".join(f"  printf(\"%zu\\n\", offsetof({cname}, {f}));\n" for f in fields)
            + "  return 0;\n}\n")
    (tmp_path / "s.c").write_text(prog)
    r = subprocess.run(["gcc", "-std=c99", "-I", os.path.dirname(HEADER), str(tmp_path / "s.c"),
                        "-o", str(tmp_path / "s")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    vals = [int(x) for x in subprocess.run([str(tmp_path / "s")], capture_output=True,
                                           text=True).stdout.split()]
    assert vals[0] == ctypes.sizeof(cls)
    assert vals[1:] == [getattr(cls, f).offset for f in fields]
