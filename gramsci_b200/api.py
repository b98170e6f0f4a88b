"""Python front end of the B200 N-point correlation library.

Mirrors the reference program's flow (src/gramsci.F90:55-224): a catalogue of
galaxies then randoms with signed normalised weights, a binning (rmin, rmax,
nbins, nmu, log), then one query (2PCF, 3PCF or 4PCF) whose results have the
reference's array shapes:

    2PCF  N2, N3 (nbins, nmu)                       query_graph_2pcf
    3PCF  N2, N3 (ncfg3, nmu)                       query_graph_3pcf_all
    4PCF  N2, N3 (ncfg4, nbins, nbins),
          discN, discR (ncfg4, nbins, nbins, 6)     query_4pcf_all2

plus integer counts by galaxy/random category.  Inputs may be numpy arrays
(host) or CUDA torch tensors (device-resident; no host copy is made).
"""
import ctypes

import numpy as np

from . import _native
from ._native import GramsciError  # noqa: F401


def ncfg3(nbins):
    return nbins * (nbins + 1) * (nbins + 2) // 6


def ncfg4(nbins):
    return nbins * (nbins + 1) * (nbins + 2) * (nbins + 3) // 24


def _fortran(a, *shape):
    """View a flat Fortran-ordered buffer with the given shape."""
    return np.asarray(a).reshape(shape[::-1]).transpose()


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def _is_torch_cuda(x):
    return hasattr(x, "is_cuda") and hasattr(x, "data_ptr") and x.is_cuda


class Context:
    """One library context (device state, catalogue, binning)."""

    def __init__(self, device=0):
        self._lib = _native.load()
        h = ctypes.c_void_p()
        rc = self._lib.gr_create(ctypes.byref(h), int(device))
        if rc != 0:
            raise GramsciError(rc, "gr_create failed (no CUDA device?)")
        self._h = h
        self.device = device
        self.nbins = self.nmu = None
        self.n = None
        self._nsplit = 0
        self.nregions = 0
        self._keep = None

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.gr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc):
        return _native.check(self._lib, self._h, rc)

    # -- state -----------------------------------------------------------
    def set_stream(self, stream):
        """Run on a caller-owned CUDA stream (torch.cuda.Stream or raw handle)."""
        handle = getattr(stream, "cuda_stream", stream)
        self._check(self._lib.gr_set_stream(self._h, ctypes.c_void_p(handle or 0)))

    def set_catalog(self, xyz, w, n_data, buffer=None):
        """xyz (N,3) FP64, w (N,) signed normalised FP64 weights, galaxies
        first (n_data of them), buffer (N,) 0/1 or None.  Clears region ids
        and mocks (they describe the points of a catalogue)."""
        self.nregions = self._nsplit ** 3
        if _is_torch_cuda(xyz):
            import torch

            xyz = xyz.detach().to(torch.float64).contiguous()
            w = w.detach().to(torch.float64).contiguous()
            buf = None if buffer is None else buffer.detach().to(torch.int32).contiguous()
            n = xyz.shape[0]
            self._keep = (xyz, w, buf)
            self.n = int(n)
            self._check(self._lib.gr_set_catalog_dev(
                self._h, ctypes.c_void_p(xyz.data_ptr()), ctypes.c_void_p(w.data_ptr()),
                ctypes.c_void_p(buf.data_ptr()) if buf is not None else None,
                int(n_data), int(n - n_data)))
            return
        xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
        w = np.ascontiguousarray(w, np.float64)
        n = xyz.shape[0]
        if w.shape[0] != n:
            raise ValueError("w must have one entry per point")
        buf = None if buffer is None else np.ascontiguousarray(buffer, np.int32)
        self.n = int(n)
        self._check(self._lib.gr_set_catalog(self._h, _ptr(xyz), _ptr(w), _ptr(buf),
                                             int(n_data), int(n - n_data)))

    def set_bins(self, rmin, rmax, nbins, nmu=1, logbins=False):
        self._check(self._lib.gr_set_bins(self._h, float(rmin), float(rmax), int(nbins),
                                          int(nmu), int(bool(logbins))))
        self.nbins, self.nmu = int(nbins), int(nmu)

    def set_precision(self, mode):
        """'f32' (FP32 separations + FP64 guard band, default) or 'f64'."""
        v = {"f32": 0, "f64": 1}[mode]
        self._check(self._lib.gr_set_option(self._h, _native.GR_OPT_PRECISION, v))

    def set_autotune(self, mode):
        """'on' (time kernel variants once per workload class, cached; dense
        catalogues take cells of rmax/2 and the tile sweep), 'off', or an
        int variant to force (0 warp per cell, 1/2 block per cell of 128/256
        threads, 3 warp per cell with queued binning, 4/5 block per cell of
        128/256 with queued binning, 6 the tile sweep, 7 the tile sweep on
        cells of rmax/2)."""
        v = {"off": 0, "on": 1}.get(mode, None)
        if v is None:
            v = 2 + int(mode)
        self._check(self._lib.gr_set_option(self._h, _native.GR_OPT_AUTOTUNE, v))

    def stats(self):
        s = _native.GrStats()
        self._check(self._lib.gr_get_stats(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in s._fields_}

    # -- queries ---------------------------------------------------------
    def count_2pcf(self):
        nb, nm = self.nbins, self.nmu
        N2, N3 = np.zeros(nb * nm), np.zeros(nb * nm)
        counts = np.zeros(nb * nm * 4, np.int64)
        catsum = np.zeros(nb * nm * 4)
        self._check(self._lib.gr_count_2pcf(self._h, _ptr(N2), _ptr(N3), _ptr(counts), _ptr(catsum)))
        return dict(N2=_fortran(N2, nb, nm), N3=_fortran(N3, nb, nm),
                    counts=_fortran(counts, nb, nm, 4), catsum=_fortran(catsum, nb, nm, 4))

    def count_3pcf(self, counts=True):
        """N2, N3 (ncfg, nmu) and the category sums; with counts=False the
        integer counts (not part of the reference's output) are not kept,
        which spares the kernel one atomic per rooted triangle when the
        weights are not uniform."""
        nb, nm = self.nbins, self.nmu
        nc = ncfg3(nb)
        N2, N3 = np.zeros(nc * nm), np.zeros(nc * nm)
        cnt = np.zeros(nc * nm * 4, np.int64) if counts else None
        catsum = np.zeros(nc * nm * 4)
        self._check(self._lib.gr_count_3pcf(self._h, _ptr(N2), _ptr(N3),
                                            _ptr(cnt) if counts else None, _ptr(catsum)))
        out = dict(N2=_fortran(N2, nc, nm), N3=_fortran(N3, nc, nm),
                   catsum=_fortran(catsum, nc, nm, 4))
        if counts:
            out["counts"] = _fortran(cnt, nc, nm, 4)
        return out

    def count_4pcf(self, counts=True):
        """N2, N3 (ncfg, nbins, nbins), discN, discR (ncfg, nbins, nbins, 6)
        and the category sums; with counts=False the integer counts (not
        part of the reference's output) are not kept, which spares the
        weighted kernel one reduction per update."""
        nb = self.nbins
        nc = ncfg4(nb)
        nbin = nc * nb * nb
        N2, N3 = np.zeros(nbin), np.zeros(nbin)
        dN, dR = np.zeros(nbin * 6), np.zeros(nbin * 6)
        cnt = np.zeros(nbin * 5, np.int64) if counts else None
        catsum = np.zeros(nbin * 5)
        dcount = np.zeros(nbin * 24, np.int64) if counts else None
        dsum = np.zeros(nbin * 24)
        self._check(self._lib.gr_count_4pcf(self._h, _ptr(N2), _ptr(N3), _ptr(dN), _ptr(dR),
                                            _ptr(cnt), _ptr(catsum), _ptr(dcount), _ptr(dsum)))
        out = dict(N2=_fortran(N2, nc, nb, nb), N3=_fortran(N3, nc, nb, nb),
                   discN=_fortran(dN, nc, nb, nb, 6), discR=_fortran(dR, nc, nb, nb, 6),
                   catsum=_fortran(catsum, nc, nb, nb, 5), dsum=_fortran(dsum, nc, nb, nb, 6, 4))
        if counts:
            out["counts"] = _fortran(cnt, nc, nb, nb, 5)
            out["dcount"] = _fortran(dcount, nc, nb, nb, 6, 4)
        return out

    # -- batched regions -------------------------------------------------
    def set_regions(self, nsplit):
        """Split the catalogue box into nsplit^3 regions with Rmax halos."""
        self._check(self._lib.gr_set_regions(self._h, int(nsplit)))
        self._nsplit = int(nsplit)
        self.nregions = self._nsplit ** 3

    def count_2pcf_batched(self):
        """2PCF of all regions in one launch (CUDA-graph replay after the
        first call); equals count_2pcf on the whole catalogue."""
        nb, nm = self.nbins, self.nmu
        N2, N3 = np.zeros(nb * nm), np.zeros(nb * nm)
        counts = np.zeros(nb * nm * 4, np.int64)
        catsum = np.zeros(nb * nm * 4)
        self._check(self._lib.gr_count_2pcf_batched(self._h, _ptr(N2), _ptr(N3), _ptr(counts),
                                                    _ptr(catsum)))
        return dict(N2=_fortran(N2, nb, nm), N3=_fortran(N3, nb, nm),
                    counts=_fortran(counts, nb, nm, 4), catsum=_fortran(catsum, nb, nm, 4))

    def set_region_ids(self, region_of_point, nregions):
        """Regions from a region id per point (e.g. jackknife regions): each
        region's halo is the bounding box of its points grown by rmax."""
        ids = np.ascontiguousarray(region_of_point, np.int32)
        if ids.shape != (self.n,):
            raise ValueError("one region id per catalogue point")
        self._check(self._lib.gr_set_region_ids(self._h, _ptr(ids), int(nregions)))
        self.nregions = int(nregions)

    def set_mocks(self, n_data, n_rand):
        """The catalogue is several independent mocks one after another (each
        galaxies first, weights normalised within the mock); batched calls
        count them all in one launch, never pairing two mocks."""
        nd = np.ascontiguousarray(n_data, np.int64)
        nr = np.ascontiguousarray(n_rand, np.int64)
        if nd.shape != nr.shape or nd.ndim != 1:
            raise ValueError("n_data and n_rand: one entry per mock")
        self._check(self._lib.gr_set_mocks(self._h, int(nd.size), _ptr(nd), _ptr(nr)))
        self.nregions = int(nd.size)

    def count_2pcf_regions(self):
        """2PCF of every region (or mock) separately, in one launch: N2, N3
        (nbins, nmu, nregions), counts and catsum (nbins, nmu, 4, nregions)."""
        nb, nm = self.nbins, self.nmu
        R = self.nregions
        N2, N3 = np.zeros(nb * nm * R), np.zeros(nb * nm * R)
        counts = np.zeros(nb * nm * 4 * R, np.int64)
        catsum = np.zeros(nb * nm * 4 * R)
        self._check(self._lib.gr_count_2pcf_regions(self._h, _ptr(N2), _ptr(N3), _ptr(counts),
                                                    _ptr(catsum)))
        return dict(N2=_fortran(N2, nb, nm, R), N3=_fortran(N3, nb, nm, R),
                    counts=_fortran(counts, nb, nm, 4, R), catsum=_fortran(catsum, nb, nm, 4, R))

    def count_3pcf_batched(self):
        """3PCF of all regions (or mocks) in one pass, summed; shapes as
        count_3pcf."""
        nb, nm = self.nbins, self.nmu
        nc = ncfg3(nb)
        N2, N3 = np.zeros(nc * nm), np.zeros(nc * nm)
        cnt = np.zeros(nc * nm * 4, np.int64)
        catsum = np.zeros(nc * nm * 4)
        self._check(self._lib.gr_count_3pcf_batched(self._h, _ptr(N2), _ptr(N3), _ptr(cnt),
                                                    _ptr(catsum)))
        return dict(N2=_fortran(N2, nc, nm), N3=_fortran(N3, nc, nm),
                    counts=_fortran(cnt, nc, nm, 4), catsum=_fortran(catsum, nc, nm, 4))

    def regions(self):
        """Region layout of the last batched call: list of (member catalogue
        indices, buffer flags) per region."""
        nr = ctypes.c_int32()
        nm = ctypes.c_int64()
        self._check(self._lib.gr_regions_info(self._h, ctypes.byref(nr), ctypes.byref(nm)))
        off = np.zeros(nr.value + 1, np.int64)
        orig = np.zeros(max(nm.value, 1), np.int32)
        buf = np.zeros(max(nm.value, 1), np.int32)
        self._check(self._lib.gr_regions_export(self._h, _ptr(off), _ptr(orig), _ptr(buf)))
        return [(orig[off[r]:off[r + 1]], buf[off[r]:off[r + 1]]) for r in range(nr.value)]

    def _adjoint(self, fn, cot2, cot3, shape):
        c2 = np.ascontiguousarray(np.asarray(cot2, np.float64).reshape(shape).T.ravel())
        c3 = None if cot3 is None else np.ascontiguousarray(
            np.asarray(cot3, np.float64).reshape(shape).T.ravel())
        g = np.zeros(self.n)
        self._check(fn(self._h, _ptr(c2), _ptr(c3), _ptr(g)))
        return g

    def adjoint_2pcf(self, cot2, cot3=None):
        """Gradient of sum(cot2*N2) + sum(cot3*N3) of the 2PCF with respect to
        the weights (catalogue order)."""
        return self._adjoint(self._lib.gr_adjoint_2pcf, cot2, cot3, (self.nbins, self.nmu))

    def adjoint_3pcf(self, cot2, cot3=None):
        """Gradient of sum(cot2*N2) + sum(cot3*N3) of the 3PCF with respect to
        the weights (catalogue order)."""
        return self._adjoint(self._lib.gr_adjoint_3pcf, cot2, cot3, (ncfg3(self.nbins), self.nmu))

    def adjoint_4pcf(self, cot2, cot3=None, cotN=None, cotR=None):
        """Gradient of sum(cot2*N2) + sum(cot3*N3) + sum(cotN*discN) +
        sum(cotR*discR) of the 4PCF with respect to the weights (catalogue
        order); cotangents in the shapes count_4pcf returns."""
        nb = self.nbins
        nc = ncfg4(nb)

        def f(a, *shape):
            if a is None:
                return None
            return np.ascontiguousarray(np.asarray(a, np.float64).reshape(shape).T.ravel())

        c2, c3 = f(cot2, nc, nb, nb), f(cot3, nc, nb, nb)
        cN, cR = f(cotN, nc, nb, nb, 6), f(cotR, nc, nb, nb, 6)
        g = np.zeros(self.n)
        self._check(self._lib.gr_adjoint_4pcf(self._h, _ptr(c2), _ptr(c3), _ptr(cN), _ptr(cR),
                                              _ptr(g)))
        return g

    def set_clique_mode(self, mode):
        """How the 3PCF / 4PCF kernels find the edges among a root's
        larger-label neighbours: "auto", "hash" (probes of the neighbours'
        rows) or "geometric" (the graph's membership test on the pairs).
        Results are identical."""
        v = {"auto": 0, "hash": 1, "geometric": 2}[mode]
        self._check(self._lib.gr_set_option(self._h, _native.GR_OPT_CLIQUE_MODE, v))

    def set_keep_graph(self, on):
        """Reuse the last call's graph until the catalogue, bins or precision change."""
        self._check(self._lib.gr_set_option(self._h, _native.GR_OPT_KEEP_GRAPH,
                                            int(bool(on))))

    def graph_save(self, path):
        """Write the neighbour graph of the current catalogue and bins to `path`."""
        self._check(self._lib.gr_graph_save(self._h, str(path).encode()))

    def graph_load(self, path):
        """Load a graph written by graph_save for the same catalogue and bins;
        later count calls reuse it."""
        self._check(self._lib.gr_graph_load(self._h, str(path).encode()))

    def count_equi(self):
        """-equi: equilateral triangles per radial bin (and mu bin)."""
        nb, nm = self.nbins, self.nmu
        N2, N3 = np.zeros(nb * nm), np.zeros(nb * nm)
        counts = np.zeros(nb * nm * 4, np.int64)
        catsum = np.zeros(nb * nm * 4)
        self._check(self._lib.gr_count_equi(self._h, _ptr(N2), _ptr(N3), _ptr(counts), _ptr(catsum)))
        return dict(N2=_fortran(N2, nb, nm), N3=_fortran(N3, nb, nm),
                    counts=_fortran(counts, nb, nm, 4), catsum=_fortran(catsum, nb, nm, 4))

    def count_tetra(self):
        """-tetra: regular tetrahedra per radial bin, with the six gated terms."""
        nb = self.nbins
        N2, N3 = np.zeros(nb), np.zeros(nb)
        dN, dR = np.zeros(nb * 6), np.zeros(nb * 6)
        counts = np.zeros(nb * 5, np.int64)
        catsum = np.zeros(nb * 5)
        dcount = np.zeros(nb * 30, np.int64)
        dsum = np.zeros(nb * 30)
        self._check(self._lib.gr_count_tetra(self._h, _ptr(N2), _ptr(N3), _ptr(dN), _ptr(dR),
                                             _ptr(counts), _ptr(catsum), _ptr(dcount), _ptr(dsum)))
        return dict(N2=N2, N3=N3, discN=_fortran(dN, nb, 6), discR=_fortran(dR, nb, 6),
                    counts=_fortran(counts, nb, 5), catsum=_fortran(catsum, nb, 5),
                    dcount=_fortran(dcount, nb, 6, 5), dsum=_fortran(dsum, nb, 6, 5))

    def graph(self):
        """The (rmin, rmax) neighbour graph in the reference's layout: rows in
        catalogue order, ids sorted, radial bin and mu bin per edge."""
        self._check(self._lib.gr_graph_build(self._h))
        E = ctypes.c_int64()
        self._check(self._lib.gr_graph_nedges(self._h, ctypes.byref(E)))
        n = self.n
        row_ptr = np.zeros(n + 1, np.int64)
        col = np.zeros(E.value, np.int32)
        b = np.zeros(E.value, np.uint8)
        mu = np.zeros(E.value, np.uint8)
        self._check(self._lib.gr_graph_export(self._h, _ptr(row_ptr), _ptr(col), _ptr(b), _ptr(mu)))
        return row_ptr, col, b, mu


def version():
    return _native.load().gr_version().decode()
