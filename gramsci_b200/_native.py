"""ctypes binding of libgramsci_cuda.so (include/gramsci_cuda.h).

The library is built in-tree (gramsci_b200/lib/libgramsci_cuda.so, see
gramsci_b200/build.py).  There is no CPU fallback: importing the binding
without the library raises, and every call that fails on the device raises
GramsciError with the library's message.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libgramsci_cuda.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "gramsci_cuda.h")

GR_OK = 0
GR_E_ARG = -1
GR_E_CAPACITY = -2
GR_E_CUDA = -3
GR_E_TIMEOUT = -4
GR_E_UNSUPPORTED = -5
GR_OPT_PRECISION = 1
GR_OPT_TIMEOUT_MS = 2
GR_OPT_AUTOTUNE = 3
GR_OPT_KEEP_GRAPH = 4
GR_OPT_CLIQUE_MODE = 5


class GramsciError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"gramsci error {code}: {msg}")
        self.code = code


class GrStats(ctypes.Structure):
    _fields_ = [
        ("ms_index", ctypes.c_double),
        ("ms_graph", ctypes.c_double),
        ("ms_query", ctypes.c_double),
        ("ms_total", ctypes.c_double),
        ("n_points", ctypes.c_int64),
        ("n_edges", ctypes.c_int64),
        ("tuples", ctypes.c_int64),
        ("rooted", ctypes.c_int64),
        ("fp64_rechecks", ctypes.c_int64),
        ("candidates", ctypes.c_int64),
        ("kernel_launches", ctypes.c_int64),
        ("probes", ctypes.c_int64),
        ("upper_edges", ctypes.c_int64),
    ]


_d = ctypes.POINTER(ctypes.c_double)
_i32 = ctypes.POINTER(ctypes.c_int32)
_i64 = ctypes.POINTER(ctypes.c_int64)
_u8 = ctypes.POINTER(ctypes.c_uint8)
_vp = ctypes.c_void_p
_ctx = ctypes.c_void_p

# name -> (restype, argtypes); every entry point of include/gramsci_cuda.h
SIGNATURES = {
    "gr_version": (ctypes.c_char_p, []),
    "gr_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int]),
    "gr_destroy": (ctypes.c_int, [_ctx]),
    "gr_last_error": (ctypes.c_char_p, [_ctx]),
    "gr_set_stream": (ctypes.c_int, [_ctx, _vp]),
    "gr_set_catalog": (ctypes.c_int, [_ctx, _vp, _vp, _vp, ctypes.c_int64, ctypes.c_int64]),
    "gr_set_catalog_dev": (ctypes.c_int, [_ctx, _vp, _vp, _vp, ctypes.c_int64, ctypes.c_int64]),
    "gr_set_bins": (ctypes.c_int, [_ctx, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
                                   ctypes.c_int32, ctypes.c_int32]),
    "gr_set_option": (ctypes.c_int, [_ctx, ctypes.c_int32, ctypes.c_int64]),
    "gr_count_2pcf": (ctypes.c_int, [_ctx, _vp, _vp, _vp, _vp]),
    "gr_count_3pcf": (ctypes.c_int, [_ctx, _vp, _vp, _vp, _vp]),
    "gr_count_4pcf": (ctypes.c_int, [_ctx, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gr_count_equi": (ctypes.c_int, [_ctx, _vp, _vp, _vp, _vp]),
    "gr_count_tetra": (ctypes.c_int, [_ctx, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gr_graph_build": (ctypes.c_int, [_ctx]),
    "gr_graph_save": (ctypes.c_int, [_ctx, ctypes.c_char_p]),
    "gr_graph_load": (ctypes.c_int, [_ctx, ctypes.c_char_p]),
    "gr_graph_nedges": (ctypes.c_int, [_ctx, _i64]),
    "gr_graph_export": (ctypes.c_int, [_ctx, _vp, _vp, _vp, _vp]),
    "gr_get_stats": (ctypes.c_int, [_ctx, ctypes.POINTER(GrStats)]),
    "gr_adjoint_2pcf": (ctypes.c_int, [_ctx, _vp, _vp, _vp]),
    "gr_set_regions": (ctypes.c_int, [_ctx, ctypes.c_int32]),
    "gr_count_2pcf_batched": (ctypes.c_int, [_ctx, _vp, _vp, _vp, _vp]),
    "gr_set_region_ids": (ctypes.c_int, [_ctx, _vp, ctypes.c_int32]),
    "gr_set_mocks": (ctypes.c_int, [_ctx, ctypes.c_int32, _vp, _vp]),
    "gr_count_2pcf_regions": (ctypes.c_int, [_ctx, _vp, _vp, _vp, _vp]),
    "gr_count_3pcf_batched": (ctypes.c_int, [_ctx, _vp, _vp, _vp, _vp]),
    "gr_regions_info": (ctypes.c_int, [_ctx, _vp, _vp]),
    "gr_regions_export": (ctypes.c_int, [_ctx, _vp, _vp, _vp]),
    "gr_adjoint_3pcf": (ctypes.c_int, [_ctx, _vp, _vp, _vp]),
    "gr_adjoint_4pcf": (ctypes.c_int, [_ctx, _vp, _vp, _vp, _vp, _vp]),
    "gr_count_2pcf_noalloc": (ctypes.c_int, [_vp, _vp, ctypes.c_int64, ctypes.c_int64,
                                             ctypes.c_double, ctypes.c_double, ctypes.c_int32,
                                             ctypes.c_int32, _vp, _vp, _vp, _vp, _vp]),
}
GR_NOALLOC_MAX_POINTS = 32768
GR_NOALLOC_MAX_BINS = 4096

_lib = None


def load(path=LIB_PATH):
    """Load the library (once).  Raises if it is missing: there is no
    fallback implementation."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing; build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "or `make -C gramsci_b200/csrc`")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(lib, ctx, rc):
    if rc != GR_OK:
        msg = lib.gr_last_error(ctx)
        raise GramsciError(rc, msg.decode() if msg else "")
    return rc
