"""One catalogue over several GPUs: slabs of roots with Rmax halos.

The reference splits a survey into regions; the points within Rmax of a
region but outside it are its buffer points (src/domain_decomposition.f90:
39-80), and only a region's own points are roots (src/gramsci.F90:363, 476,
672).  Every tuple is counted once per non-buffer vertex, so the rooted
histograms of the regions add up to those of the whole catalogue.  Here the
regions are slabs along the longest axis of the bounding box, one per rank,
cut at quantiles of that coordinate so that every rank holds about as many
roots.  A rank counts its slab (roots) with its halo (buffer points) on its
own GPU, and one all-reduce (sum) of the histograms gives every rank the
counts of the whole catalogue: integer counts exactly, weighted sums to a
few units in the last place (each rank's sums are exact fixed point rounded
once to FP64; the ranks' doubles are then added).

Every point within Rmax of a root lies in the root's slab or its halo: a
neighbour is closer than Rmax in every coordinate, and the halo reaches a
little beyond Rmax on both sides.  Extra halo points change nothing (they
are no roots, and a tuple counts only through its roots).  The shards keep
the catalogue order (galaxies first), which the mu-bin convention of the
3PCF and 4PCF (neighbours taken in catalogue-id order) depends on.
"""
import numpy as np

# the halo reaches this much beyond Rmax, relative to the coordinates'
# magnitude, so that rounding in the comparisons never drops a neighbour
_HALO_SLACK = 1e-9


def slab_axis(xyz):
    """Axis of the largest extent of the catalogue's bounding box."""
    xyz = np.asarray(xyz, np.float64).reshape(-1, 3)
    if xyz.shape[0] == 0:
        return 0
    return int(np.argmax(xyz.max(axis=0) - xyz.min(axis=0)))


def slab_edges(coord, world):
    """world + 1 slab edges along one coordinate: -inf, the interior cuts at
    the k/world quantiles, +inf.  Slab r holds the points with
    edges[r] <= coord < edges[r + 1]."""
    coord = np.asarray(coord, np.float64)
    world = int(world)
    if world < 1:
        raise ValueError("world must be at least 1")
    edges = np.empty(world + 1)
    edges[0], edges[-1] = -np.inf, np.inf
    if world > 1:
        if coord.size == 0:
            edges[1:-1] = 0.0
        else:
            edges[1:-1] = np.quantile(coord, np.arange(1, world) / world)
    return edges


def shard(xyz, w, n_data, rank, world, rmax, buffer=None, axis=None):
    """The points rank `rank` of `world` counts: its slab's points as roots
    and the halo within Rmax of the slab as buffer points, in catalogue
    order.  A point that is a buffer point of the whole catalogue (buffer
    given) stays one.  Returns (xyz, w, n_data, buffer, index): the shard's
    coordinates (M, 3), weights (M,), galaxies among them, 0/1 buffer flags
    (int32) and the catalogue index of every shard point."""
    xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
    w = np.ascontiguousarray(w, np.float64)
    n = xyz.shape[0]
    if w.shape[0] != n:
        raise ValueError("w must have one entry per point")
    if not 0 <= int(n_data) <= n:
        raise ValueError("n_data out of range")
    if not 0 <= int(rank) < int(world):
        raise ValueError("rank out of range")
    if not rmax > 0:
        raise ValueError("rmax must be positive")
    ax = slab_axis(xyz) if axis is None else int(axis)
    c = xyz[:, ax]
    edges = slab_edges(c, world)
    lo, hi = edges[rank], edges[rank + 1]
    own = (c >= lo) & (c < hi)
    scale = float(np.abs(c).max()) if n else 0.0
    reach = float(rmax) * (1.0 + _HALO_SLACK) + _HALO_SLACK * scale
    keep = (c > lo - reach) & (c < hi + reach)
    if buffer is not None:
        own &= np.asarray(buffer).reshape(-1) == 0
    index = np.nonzero(keep)[0]
    buf = (~own[index]).astype(np.int32)
    return xyz[index], w[index], int(np.count_nonzero(index < n_data)), buf, index


def allreduce_counts(out, group=None, device="cpu"):
    """Sum every histogram of a count over the ranks of the process group
    (torch.distributed, which must be initialised), in place; returns out.
    Integer arrays are summed as int64, the rest as FP64."""
    import torch
    import torch.distributed as dist

    for k in sorted(out):
        v = np.asarray(out[k])
        dt = torch.int64 if np.issubdtype(v.dtype, np.integer) else torch.float64
        flat = np.ascontiguousarray(v.ravel(order="F"))
        t = torch.from_numpy(flat).to(device=device, dtype=dt)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        out[k] = t.cpu().numpy().astype(v.dtype, copy=False).reshape(v.shape, order="F")
    return out


def count(ctx, kind, xyz, w, n_data, rank, world, rmax, group=None, device="cpu",
          buffer=None, **kwargs):
    """The histograms of the whole catalogue from rank `rank`'s slab:
    ctx.set_catalog with the shard, ctx.count_<kind>(**kwargs), then the
    all-reduce over the group (none when world is 1).  kind: "2pcf",
    "3pcf" or "4pcf"."""
    if kind not in ("2pcf", "3pcf", "4pcf"):
        raise ValueError("kind must be 2pcf, 3pcf or 4pcf")
    sx, sw, snd, sb, _ = shard(xyz, w, n_data, rank, world, rmax, buffer=buffer)
    ctx.set_catalog(sx, sw, snd, buffer=sb)
    out = getattr(ctx, "count_" + kind)(**kwargs)
    if int(world) > 1:
        allreduce_counts(out, group=group, device=device)
    return out
