"""ctypes front end of the CPU oracle (oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
CPU-baseline leg of bench.py, never by the gramsci_b200 package.  See the
header of oracle.cpp for what the oracle restates and for its parity status
(unpinned against reference outputs: no Fortran compiler is available to
build the reference).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_d = ctypes.POINTER(ctypes.c_double)
_i32 = ctypes.POINTER(ctypes.c_int32)
_i64 = ctypes.POINTER(ctypes.c_int64)
_u8 = ctypes.POINTER(ctypes.c_uint8)


def build():
    """Compile liboracle.so in place (g++ with OpenMP, strict IEEE)."""
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
            os.path.join(_HERE, "oracle.cpp")
        ):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_graph_new.restype = ctypes.c_void_p
        L.orc_graph_new.argtypes = [_d, ctypes.c_int64, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                    ctypes.c_int32, ctypes.c_int32]
        L.orc_graph_free.argtypes = [ctypes.c_void_p]
        L.orc_graph_nedges.restype = ctypes.c_int64
        L.orc_graph_nedges.argtypes = [ctypes.c_void_p]
        L.orc_graph_copy.argtypes = [ctypes.c_void_p, _i64, _i32, _u8, _u8]
        L.orc_edge_eval.restype = ctypes.c_int32
        L.orc_edge_eval.argtypes = [_d, _d, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
                                    ctypes.c_int32, ctypes.c_int32, _i32]
        L.orc_normal_table.argtypes = [ctypes.c_int32, ctypes.c_int32, _i32]
        L.orc_bintable3.restype = ctypes.c_int32
        L.orc_bintable3.argtypes = [ctypes.c_int32] * 4
        L.orc_bintable4.restype = ctypes.c_int32
        L.orc_bintable4.argtypes = [ctypes.c_int32] * 5
        L.orc_normalise.argtypes = [_d, ctypes.c_int64, ctypes.c_int64]
        L.orc_2pcf.argtypes = [ctypes.c_void_p, _d, _i32, ctypes.c_int64, _d, _d, _i64, _d]
        L.orc_3pcf.argtypes = [ctypes.c_void_p, _d, _i32, ctypes.c_int64, _i32, _d, _d, _i64, _d]
        L.orc_4pcf.argtypes = [ctypes.c_void_p, _d, _i32, ctypes.c_int64, _d, _d, _d, _d, _i64,
                               _d, _i64, _d]
        L.orc_equi.argtypes = [ctypes.c_void_p, _d, _i32, ctypes.c_int64, _i32, _d, _d, _i64, _d]
        L.orc_tetra.argtypes = [ctypes.c_void_p, _d, _i32, ctypes.c_int64, _d, _d, _d, _d, _i64, _d,
                                _i64, _d]
        L.orc_adjoint_2pcf.argtypes = [ctypes.c_void_p, _d, _i32, ctypes.c_int64, _d, _d, _d]
        L.orc_adjoint_3pcf.argtypes = [ctypes.c_void_p, _d, _i32, ctypes.c_int64, _i32, _d, _d, _d]
        L.orc_adjoint_4pcf.argtypes = [ctypes.c_void_p, _d, _i32, ctypes.c_int64, _d, _d, _d, _d,
                                       _d]
        L.orc_max_threads.restype = ctypes.c_int32
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def ncfg3(nbins):
    return nbins * (nbins + 1) * (nbins + 2) // 6


def ncfg4(nbins):
    return nbins * (nbins + 1) * (nbins + 2) * (nbins + 3) // 24


class Graph:
    """Neighbour graph of a catalogue: rows sorted by 0-based point index."""

    def __init__(self, xyz, rmin, rmax, nbins, nmu=1, logbins=False, method="grid", threads=0):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        self.n = xyz.shape[0]
        self.nbins, self.nmu = int(nbins), int(nmu)
        self.rmin, self.rmax = float(rmin), float(rmax)
        self._xyz = xyz
        m = {"grid": 0, "kdtree": 1}[method]
        self._h = lib().orc_graph_new(_p(xyz, _d), self.n, self.rmin, self.rmax, self.nbins,
                                      self.nmu, int(bool(logbins)), m, int(threads))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_graph_free(self._h)
            self._h = None

    @property
    def nedges(self):
        return int(lib().orc_graph_nedges(self._h))

    def csr(self):
        E = self.nedges
        row_ptr = np.zeros(self.n + 1, np.int64)
        col = np.zeros(E, np.int32)
        b = np.zeros(E, np.uint8)
        mu = np.zeros(E, np.uint8)
        lib().orc_graph_copy(self._h, _p(row_ptr, _i64), _p(col, _i32), _p(b, _u8), _p(mu, _u8))
        return row_ptr, col, b, mu

    # -- queries ---------------------------------------------------------
    def pcf2(self, w, n_data, buffer=None):
        w = np.ascontiguousarray(w, np.float64)
        buf = None if buffer is None else np.ascontiguousarray(buffer, np.int32)
        nb, nm = self.nbins, self.nmu
        N2 = np.zeros(nb * nm)
        N3 = np.zeros(nb * nm)
        counts = np.zeros(nb * nm * 4, np.int64)
        catsum = np.zeros(nb * nm * 4)
        lib().orc_2pcf(self._h, _p(w, _d), _p(buf, _i32), int(n_data), _p(N2, _d), _p(N3, _d),
                       _p(counts, _i64), _p(catsum, _d))
        f = lambda a, *s: a.reshape(s[::-1]).transpose()  # Fortran layout
        return dict(N2=f(N2, nb, nm), N3=f(N3, nb, nm), counts=f(counts, nb, nm, 4),
                    catsum=f(catsum, nb, nm, 4))

    def pcf3(self, w, n_data, buffer=None, normal_variant=0):
        w = np.ascontiguousarray(w, np.float64)
        buf = None if buffer is None else np.ascontiguousarray(buffer, np.int32)
        nb, nm = self.nbins, self.nmu
        nc = ncfg3(nb)
        tab = normal_table(nm, normal_variant)
        N2 = np.zeros(nc * nm)
        N3 = np.zeros(nc * nm)
        counts = np.zeros(nc * nm * 4, np.int64)
        catsum = np.zeros(nc * nm * 4)
        lib().orc_3pcf(self._h, _p(w, _d), _p(buf, _i32), int(n_data),
                       _p(np.ascontiguousarray(tab.T.ravel()), _i32), _p(N2, _d), _p(N3, _d),
                       _p(counts, _i64), _p(catsum, _d))
        f = lambda a, *s: a.reshape(s[::-1]).transpose()
        return dict(N2=f(N2, nc, nm), N3=f(N3, nc, nm), counts=f(counts, nc, nm, 4),
                    catsum=f(catsum, nc, nm, 4))

    def pcf4(self, w, n_data, buffer=None):
        w = np.ascontiguousarray(w, np.float64)
        buf = None if buffer is None else np.ascontiguousarray(buffer, np.int32)
        nb = self.nbins
        nc = ncfg4(nb)
        nbin = nc * nb * nb
        N2 = np.zeros(nbin)
        N3 = np.zeros(nbin)
        dN = np.zeros(nbin * 6)
        dR = np.zeros(nbin * 6)
        counts = np.zeros(nbin * 5, np.int64)
        catsum = np.zeros(nbin * 5)
        dcount = np.zeros(nbin * 24, np.int64)
        dsum = np.zeros(nbin * 24)
        lib().orc_4pcf(self._h, _p(w, _d), _p(buf, _i32), int(n_data), _p(N2, _d), _p(N3, _d),
                       _p(dN, _d), _p(dR, _d), _p(counts, _i64), _p(catsum, _d),
                       _p(dcount, _i64), _p(dsum, _d))
        f = lambda a, *s: a.reshape(s[::-1]).transpose()
        return dict(N2=f(N2, nc, nb, nb), N3=f(N3, nc, nb, nb), discN=f(dN, nc, nb, nb, 6),
                    discR=f(dR, nc, nb, nb, 6), counts=f(counts, nc, nb, nb, 5),
                    catsum=f(catsum, nc, nb, nb, 5), dcount=f(dcount, nc, nb, nb, 6, 4),
                    dsum=f(dsum, nc, nb, nb, 6, 4))

    def equi(self, w, n_data, buffer=None, normal_variant=0):
        w = np.ascontiguousarray(w, np.float64)
        buf = None if buffer is None else np.ascontiguousarray(buffer, np.int32)
        nb, nm = self.nbins, self.nmu
        tab = normal_table(nm, normal_variant)
        N2, N3 = np.zeros(nb * nm), np.zeros(nb * nm)
        counts = np.zeros(nb * nm * 4, np.int64)
        catsum = np.zeros(nb * nm * 4)
        lib().orc_equi(self._h, _p(w, _d), _p(buf, _i32), int(n_data),
                       _p(np.ascontiguousarray(tab.T.ravel()), _i32), _p(N2, _d), _p(N3, _d),
                       _p(counts, _i64), _p(catsum, _d))
        f = lambda a, *s: a.reshape(s[::-1]).transpose()
        return dict(N2=f(N2, nb, nm), N3=f(N3, nb, nm), counts=f(counts, nb, nm, 4),
                    catsum=f(catsum, nb, nm, 4))

    def tetra(self, w, n_data, buffer=None):
        w = np.ascontiguousarray(w, np.float64)
        buf = None if buffer is None else np.ascontiguousarray(buffer, np.int32)
        nb = self.nbins
        N2, N3 = np.zeros(nb), np.zeros(nb)
        dN, dR = np.zeros(nb * 6), np.zeros(nb * 6)
        counts = np.zeros(nb * 5, np.int64)
        catsum = np.zeros(nb * 5)
        dcount = np.zeros(nb * 30, np.int64)
        dsum = np.zeros(nb * 30)
        lib().orc_tetra(self._h, _p(w, _d), _p(buf, _i32), int(n_data), _p(N2, _d), _p(N3, _d),
                        _p(dN, _d), _p(dR, _d), _p(counts, _i64), _p(catsum, _d), _p(dcount, _i64),
                        _p(dsum, _d))
        f = lambda a, *s: a.reshape(s[::-1]).transpose()
        return dict(N2=N2, N3=N3, discN=f(dN, nb, 6), discR=f(dR, nb, 6), counts=f(counts, nb, 5),
                    catsum=f(catsum, nb, 5), dcount=f(dcount, nb, 6, 5), dsum=f(dsum, nb, 6, 5))

    def adjoint2(self, w, n_data, cot2, cot3=None, buffer=None):
        w = np.ascontiguousarray(w, np.float64)
        buf = None if buffer is None else np.ascontiguousarray(buffer, np.int32)
        c2 = np.ascontiguousarray(np.asarray(cot2, np.float64).T.ravel())
        c3 = None if cot3 is None else np.ascontiguousarray(np.asarray(cot3, np.float64).T.ravel())
        g = np.zeros(self.n)
        lib().orc_adjoint_2pcf(self._h, _p(w, _d), _p(buf, _i32), int(n_data), _p(c2, _d),
                               _p(c3, _d), _p(g, _d))
        return g

    def adjoint3(self, w, n_data, cot2, cot3=None, buffer=None, normal_variant=0):
        w = np.ascontiguousarray(w, np.float64)
        buf = None if buffer is None else np.ascontiguousarray(buffer, np.int32)
        tab = normal_table(self.nmu, normal_variant)
        c2 = np.ascontiguousarray(np.asarray(cot2, np.float64).T.ravel())
        c3 = None if cot3 is None else np.ascontiguousarray(np.asarray(cot3, np.float64).T.ravel())
        g = np.zeros(self.n)
        lib().orc_adjoint_3pcf(self._h, _p(w, _d), _p(buf, _i32), int(n_data),
                               _p(np.ascontiguousarray(tab.T.ravel()), _i32), _p(c2, _d),
                               _p(c3, _d), _p(g, _d))
        return g

    def adjoint4(self, w, n_data, cot2, cot3=None, cotN=None, cotR=None, buffer=None):
        """Gradient of sum(cot2 N2 + cot3 N3 + cotN discN + cotR discR) of
        pcf4 with respect to w; cotangents in the shapes pcf4 returns."""
        w = np.ascontiguousarray(w, np.float64)
        buf = None if buffer is None else np.ascontiguousarray(buffer, np.int32)
        f = lambda a: None if a is None else np.ascontiguousarray(np.asarray(a, np.float64).T.ravel())
        g = np.zeros(self.n)
        lib().orc_adjoint_4pcf(self._h, _p(w, _d), _p(buf, _i32), int(n_data), _p(f(cot2), _d),
                               _p(f(cot3), _d), _p(f(cotN), _d), _p(f(cotR), _d), _p(g, _d))
        return g


def edge_eval(pi, pj, rmin, rmax, nbins, nmu=1, logbins=False):
    """Reference predicate for one pair: (is_edge, bin, mu_fwd, mu_rev)."""
    a = np.ascontiguousarray(pi, np.float64)
    b = np.ascontiguousarray(pj, np.float64)
    out = np.zeros(3, np.int32)
    e = lib().orc_edge_eval(_p(a, _d), _p(b, _d), float(rmin), float(rmax), int(nbins), int(nmu),
                            int(bool(logbins)), _p(out, _i32))
    return bool(e), int(out[0]), int(out[1]), int(out[2])


def normal_table(nmu, variant=0):
    """find_normal for all (mu1, mu2): array [mu1-1, mu2-1] (variant 0 plain, 1 FMA)."""
    out = np.zeros(nmu * nmu, np.int32)
    lib().orc_normal_table(int(nmu), int(variant), _p(out, _i32))
    return out.reshape(nmu, nmu).T.copy()  # stored [mu1-1 + nmu*(mu2-1)]


def bintable3(a, b, c, nbins):
    return int(lib().orc_bintable3(a, b, c, nbins))


def bintable4(a, b, c, d, nbins):
    return int(lib().orc_bintable4(a, b, c, d, nbins))


def normalise(w, n_data, n_rand):
    w = np.array(w, np.float64, copy=True)
    lib().orc_normalise(_p(w, _d), int(n_data), int(n_rand))
    return w


def max_threads():
    return int(lib().orc_max_threads())
