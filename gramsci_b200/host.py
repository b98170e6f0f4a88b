"""ctypes binding of libgramsci_host.so (include/gramsci_host.h): option
parsing, catalogue reading, weight normalisation and output writers of the
`gramsci` command.  None of these needs a GPU."""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libgramsci_host.so")
CLI_PATH = os.path.join(HERE, "bin", "gramsci")
DECOMPOSE_PATH = os.path.join(HERE, "bin", "gramsci-decompose")
RESUM_PATH = os.path.join(HERE, "bin", "gramsci-resum")


class Options(ctypes.Structure):
    _fields_ = [("gal", ctypes.c_char * 2048), ("ran", ctypes.c_char * 2048),
                ("out", ctypes.c_char * 2048), ("cut", ctypes.c_char * 2048),
                ("rmin", ctypes.c_double), ("rmax", ctypes.c_double),
                ("nbins", ctypes.c_int32), ("nmu", ctypes.c_int32),
                ("rsd", ctypes.c_int32), ("logbins", ctypes.c_int32), ("cut_mode", ctypes.c_int32),
                ("mpi", ctypes.c_int32), ("rancat", ctypes.c_int32),
                ("two_pcf", ctypes.c_int32), ("three_pcf", ctypes.c_int32),
                ("four_pcf", ctypes.c_int32), ("equi", ctypes.c_int32), ("tetra", ctypes.c_int32),
                ("gcol", ctypes.c_int32),
                ("help", ctypes.c_int32), ("error", ctypes.c_int32),
                ("message", ctypes.c_char * 256)]


_lib = None
_d = ctypes.POINTER(ctypes.c_double)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; run `make -C gramsci_b200/csrc`")
        L = ctypes.CDLL(LIB_PATH)
        L.grh_parse_args.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p),
                                     ctypes.POINTER(Options)]
        L.grh_read_catalogue.argtypes = [ctypes.c_char_p, ctypes.c_char_p,
                                         ctypes.POINTER(_d), ctypes.POINTER(_d),
                                         ctypes.POINTER(ctypes.c_int64),
                                         ctypes.POINTER(ctypes.c_int64)]
        L.grh_free.argtypes = [ctypes.c_void_p]
        L.grh_normalise.argtypes = [_d, ctypes.c_int64, ctypes.c_int64]
        L.grh_radial_bins.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int32,
                                      ctypes.c_int32, _d]
        L.grh_format_e14_7.argtypes = [ctypes.c_double, ctypes.c_char_p]
        for name in ("grh_write_2pcf", "grh_write_3pcf"):
            getattr(L, name).argtypes = [ctypes.c_char_p, _d, ctypes.c_int32, ctypes.c_int32, _d, _d]
        L.grh_write_4pcf.argtypes = [ctypes.c_char_p, _d, ctypes.c_int32, _d, _d, _d, _d]
        L.grh_write_equi.argtypes = [ctypes.c_char_p, _d, ctypes.c_int32, ctypes.c_int32, _d, _d]
        L.grh_write_tetra.argtypes = [ctypes.c_char_p, _d, ctypes.c_int32, ctypes.c_int32, _d, _d,
                                      _d, _d]
        _lib = L
    return _lib


def parse_args(args):
    argv = (ctypes.c_char_p * (len(args) + 1))(b"gramsci", *[a.encode() for a in args])
    o = Options()
    load().grh_parse_args(len(args) + 1, argv, ctypes.byref(o))
    return o


def read_catalogue(gal, ran=None):
    xyz = _d()
    w = _d()
    nd = ctypes.c_int64()
    nr = ctypes.c_int64()
    rc = load().grh_read_catalogue(gal.encode(), ran.encode() if ran else None, ctypes.byref(xyz),
                                   ctypes.byref(w), ctypes.byref(nd), ctypes.byref(nr))
    if rc:
        raise OSError(f"grh_read_catalogue failed ({rc})")
    n = nd.value + nr.value
    a = np.ctypeslib.as_array(xyz, shape=(max(3 * n, 1),))[:3 * n].reshape(n, 3).copy()
    b = np.ctypeslib.as_array(w, shape=(max(n, 1),))[:n].copy()
    load().grh_free(ctypes.cast(xyz, ctypes.c_void_p))
    load().grh_free(ctypes.cast(w, ctypes.c_void_p))
    return a, b, nd.value, nr.value


def format_e14_7(v):
    buf = ctypes.create_string_buffer(16)
    load().grh_format_e14_7(float(v), buf)
    return buf.value.decode()


def radial_bins(rmin, rmax, nbins, logbins=False):
    e = np.zeros(nbins + 1)
    load().grh_radial_bins(rmin, rmax, nbins, int(bool(logbins)), e.ctypes.data_as(_d))
    return e


def _flat(a):
    return np.ascontiguousarray(np.asarray(a, np.float64).T.ravel())


def write_2pcf(path, edges, nbins, nmu, N2, N3):
    e, a, b = _flat(edges), _flat(N2), _flat(N3)
    return load().grh_write_2pcf(path.encode(), e.ctypes.data_as(_d), nbins, nmu,
                                 a.ctypes.data_as(_d), b.ctypes.data_as(_d))


def write_3pcf(path, edges, nbins, nmu, N2, N3):
    e, a, b = _flat(edges), _flat(N2), _flat(N3)
    return load().grh_write_3pcf(path.encode(), e.ctypes.data_as(_d), nbins, nmu,
                                 a.ctypes.data_as(_d), b.ctypes.data_as(_d))


def write_4pcf(path, edges, nbins, N2, N3, discN, discR):
    e, a, b, c, d = _flat(edges), _flat(N2), _flat(N3), _flat(discN), _flat(discR)
    return load().grh_write_4pcf(path.encode(), e.ctypes.data_as(_d), nbins, a.ctypes.data_as(_d),
                                 b.ctypes.data_as(_d), c.ctypes.data_as(_d), d.ctypes.data_as(_d))


def write_equi(path, edges, nbins, nmu, N2, N3):
    e, a, b = _flat(edges), _flat(N2), _flat(N3)
    return load().grh_write_equi(path.encode(), e.ctypes.data_as(_d), nbins, nmu,
                                 a.ctypes.data_as(_d), b.ctypes.data_as(_d))


def write_tetra(path, edges, nbins, nmu, N2, N3, discN, discR):
    e, a, b, c, d = _flat(edges), _flat(N2), _flat(N3), _flat(discN), _flat(discR)
    return load().grh_write_tetra(path.encode(), e.ctypes.data_as(_d), nbins, nmu,
                                  a.ctypes.data_as(_d), b.ctypes.data_as(_d), c.ctypes.data_as(_d),
                                  d.ctypes.data_as(_d))


def decompose(rmax, prefix, allpoints=None, gal=None, ran=None, nsplit=0):
    """grh_decompose: region files <prefix>j.loadnodes; returns the count."""
    L = load()
    L.grh_decompose.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_double,
                                ctypes.c_int32, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int32)]
    n = ctypes.c_int32(0)
    enc = lambda s: None if s is None else str(s).encode()
    rc = L.grh_decompose(enc(allpoints), enc(gal), enc(ran), float(rmax), int(nsplit),
                         str(prefix).encode(), ctypes.byref(n))
    if rc:
        raise OSError(f"grh_decompose failed ({rc})")
    return n.value


def resum(query, inputs, out):
    """grh_resum; query 2/3/4 (N-point), 5 (-equi), 6 (-tetra).  Returns rc."""
    L = load()
    arr = (ctypes.c_char_p * len(inputs))(*[str(p).encode() for p in inputs])
    L.grh_resum.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_char_p),
                            ctypes.c_char_p]
    return L.grh_resum(int(query), len(inputs), arr, str(out).encode())


def read_region_gal(path):
    """grh_read_region_gal: (xyz (N,3), w, buffer, n_data, n_rand)."""
    L = load()
    xyz, w = _d(), _d()
    buf = ctypes.POINTER(ctypes.c_int32)()
    nd, nr = ctypes.c_int64(0), ctypes.c_int64(0)
    L.grh_read_region_gal.argtypes = [ctypes.c_char_p, ctypes.POINTER(_d), ctypes.POINTER(_d),
                                      ctypes.POINTER(ctypes.POINTER(ctypes.c_int32)),
                                      ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]
    if L.grh_read_region_gal(str(path).encode(), ctypes.byref(xyz), ctypes.byref(w), ctypes.byref(buf),
                             ctypes.byref(nd), ctypes.byref(nr)):
        raise OSError(f"cannot read {path}")
    n = nd.value + nr.value
    out = (np.ctypeslib.as_array(xyz, (3 * n,)).reshape(n, 3).copy() if n else np.zeros((0, 3)),
           np.ctypeslib.as_array(w, (n,)).copy() if n else np.zeros(0),
           np.ctypeslib.as_array(buf, (n,)).copy() if n else np.zeros(0, np.int32), nd.value, nr.value)
    L.grh_free.argtypes = [ctypes.c_void_p]
    for p in (xyz, w, buf):
        L.grh_free(ctypes.cast(p, ctypes.c_void_p))
    return out
