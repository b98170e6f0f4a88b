"""Differentiable weighted 2PCF / 3PCF counts (torch.autograd.Function).

The forward pass runs the counting kernels; the backward pass runs the
hand-written adjoint kernels (gr_adjoint_2pcf / gr_adjoint_3pcf): for
L = sum(gN2 * N2) + sum(gN3 * N3), dL/dw_k is the sum over the rooted pairs
or triangles containing k of the cotangent of their bin times the product of
the other weights.  Positions and bin membership are exact and not
differentiated.  The weights here are the signed normalised weights the
reference forms after reading (src/gramsci.F90:1390-1391); normalise raw
weights with `normalise` to differentiate through that step too.
"""
import numpy as np
import torch

from . import api

_contexts = {}


def _context(device):
    idx = device.index if device.type == "cuda" and device.index is not None else 0
    if idx not in _contexts:
        _contexts[idx] = api.Context(idx)
    return _contexts[idx]


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
        c.set_catalog(xyz.detach().cpu().numpy(), w.detach().cpu().numpy(), n_data)
        c.set_bins(*bins)
        out = c.count_2pcf() if order == 2 else c.count_3pcf()
        ctx.save_for_backward(w, xyz)
        ctx.n_data, ctx.bins, ctx.order = n_data, bins, order
        to = dict(dtype=torch.float64, device=w.device)
        return torch.as_tensor(out["N2"], **to), torch.as_tensor(out["N3"], **to)

    @staticmethod
    def backward(ctx, gN2, gN3):
        w, xyz = ctx.saved_tensors
        c = _context(w.device)
        c.set_catalog(xyz.detach().cpu().numpy(), w.detach().cpu().numpy(), ctx.n_data)
        c.set_bins(*ctx.bins)
        g2 = np.zeros(1) if gN2 is None else gN2.detach().cpu().numpy()
        g3 = None if gN3 is None else gN3.detach().cpu().numpy()
        if gN2 is None:
            g2 = np.zeros_like(g3)
        fn = c.adjoint_2pcf if ctx.order == 2 else c.adjoint_3pcf
        g = fn(g2, g3)
        return torch.as_tensor(g, dtype=w.dtype, device=w.device), None, None, None, None


def pcf2(w, xyz, n_data, rmin, rmax, nbins, nmu=1):
    """Weighted 2PCF sums (N2, N3), each (nbins, nmu), differentiable in w."""
    return _PCF.apply(w, xyz, int(n_data), (float(rmin), float(rmax), int(nbins), int(nmu)), 2)


def pcf3(w, xyz, n_data, rmin, rmax, nbins, nmu=1):
    """Weighted 3PCF sums (N2, N3), each (ncfg, nmu), differentiable in w."""
    return _PCF.apply(w, xyz, int(n_data), (float(rmin), float(rmax), int(nbins), int(nmu)), 3)
