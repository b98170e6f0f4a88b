"""Differentiable weighted 2PCF / 3PCF / 4PCF counts (torch.autograd.Function).

The forward pass runs the counting kernels; the backward pass runs the
hand-written adjoint kernels (gr_adjoint_2pcf / _3pcf / _4pcf): for
L = sum(gN2 * N2) + sum(gN3 * N3) (+ sum(gdN * discN) + sum(gdR * discR)
for the 4PCF), dL/dw_k is the sum over the rooted pairs, triangles or
4-cliques containing k of the cotangent of their bin times the product of
the other weights (the partner's weight for the 4PCF pair terms).  Positions and bin membership are exact and not
differentiated.  The weights here are the signed normalised weights the
reference forms after reading (src/gramsci.F90:1390-1391); normalise raw
weights with `normalise` to differentiate through that step too.
"""
import itertools

import numpy as np
import torch

from . import api

_contexts = {}
# the forward call whose catalogue and bins each context holds (by device)
_holder = {}
_tokens = itertools.count(1)


def _context(device):
    idx = device.index if device.type == "cuda" and device.index is not None else 0
    if idx not in _contexts:
        _contexts[idx] = api.Context(idx)
    return _contexts[idx]


def _load(c, w, xyz, n_data, bins):
    """Hand the catalogue to the library: CUDA tensors by device pointer
    (gr_set_catalog_dev, no host round trip), host tensors through NumPy."""
    if xyz.is_cuda and w.is_cuda:
        c.set_catalog(xyz.detach(), w.detach(), n_data)
    else:
        c.set_catalog(xyz.detach().cpu().numpy(), w.detach().cpu().numpy(), n_data)
    c.set_bins(*bins)


def normalise(w_raw, n_data):
    """Galaxy weights over their sum, random weights negated over theirs, as
    torch operations (differentiable)."""
    g = w_raw[:n_data] / w_raw[:n_data].sum()
    r = -w_raw[n_data:] / w_raw[n_data:].sum()
    return torch.cat([g, r])


class _PCF(torch.autograd.Function):
    @staticmethod
    def forward(ctx, w, xyz, n_data, bins, order):
        c = _context(w.device)
        _load(c, w, xyz, n_data, bins)
        count = {2: c.count_2pcf, 3: c.count_3pcf, 4: c.count_4pcf}[order]
        out = count()
        ctx.save_for_backward(w, xyz)
        ctx.n_data, ctx.bins, ctx.order = n_data, bins, order
        # the context keeps this catalogue (and its graph) until another
        # forward pass replaces it; the backward pass then skips the upload
        ctx.token = next(_tokens)
        _holder[id(c)] = ctx.token
        to = dict(dtype=torch.float64, device=w.device)
        names = ("N2", "N3", "discN", "discR") if order == 4 else ("N2", "N3")
        ctx.shapes = [out[k].shape for k in names]
        return tuple(torch.as_tensor(out[k], **to) for k in names)

    @staticmethod
    def backward(ctx, *grads):
        w, xyz = ctx.saved_tensors
        c = _context(w.device)
        if _holder.get(id(c)) != ctx.token:
            # another forward pass ran in between: upload this one's inputs
            # again (the graph is then rebuilt by the adjoint call)
            _load(c, w, xyz, ctx.n_data, ctx.bins)
            _holder[id(c)] = ctx.token
        cots = [None if g is None else g.detach().cpu().numpy() for g in grads]
        if cots[0] is None:
            cots[0] = np.zeros(ctx.shapes[0])
        fn = {2: c.adjoint_2pcf, 3: c.adjoint_3pcf, 4: c.adjoint_4pcf}[ctx.order]
        g = fn(*cots)
        return torch.as_tensor(g, dtype=w.dtype, device=w.device), None, None, None, None


def pcf2(w, xyz, n_data, rmin, rmax, nbins, nmu=1):
    """Weighted 2PCF sums (N2, N3), each (nbins, nmu), differentiable in w."""
    return _PCF.apply(w, xyz, int(n_data), (float(rmin), float(rmax), int(nbins), int(nmu)), 2)


def pcf3(w, xyz, n_data, rmin, rmax, nbins, nmu=1):
    """Weighted 3PCF sums (N2, N3), each (ncfg, nmu), differentiable in w."""
    return _PCF.apply(w, xyz, int(n_data), (float(rmin), float(rmax), int(nbins), int(nmu)), 3)


def pcf4(w, xyz, n_data, rmin, rmax, nbins):
    """Weighted 4PCF sums (N2, N3, discN, discR): N2 and N3 (ncfg, nbins,
    nbins), discN and discR (ncfg, nbins, nbins, 6), differentiable in w."""
    return _PCF.apply(w, xyz, int(n_data), (float(rmin), float(rmax), int(nbins), 1), 4)
