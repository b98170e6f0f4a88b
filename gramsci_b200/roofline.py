"""Roofline figures for the bench line: measured peaks and the algorithmic
work of the counting kernels."""
import json
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FALLBACK_HBM_GBS = 6650.0


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    except Exception:
        return {"hbm_gbs": FALLBACK_HBM_GBS, "source": "fallback"}


def tri3_bytes(stats):
    """Algorithmic bytes of one triangle-kernel launch.

    Per upper edge (p, a): the root row entry (col + meta, 8 B) and the two
    row offsets of a (16 B).  Per probe (an entry c of the row of a looked up
    in the row of p): its column index (4 B).  Per rooted triangle
    contribution the (a, c) edge metadata and the two far vertices' flags,
    ids and weights are gathered: counted as 4 + 2 * 13 B per triangle.
    """
    e = stats["upper_edges"]
    return 24 * e + 4 * stats["probes"] + 30 * stats["tuples"]


def tri3_roofline(ctx, q_ms, pk):
    st = ctx.stats()
    ms = sum(q_ms) / len(q_ms)
    b = tri3_bytes(st)
    achieved = b / (ms * 1e-3) / 1e9
    return {"bound": "hbm", "kernel": "tri3_kernel", "achieved": achieved, "peak": pk["hbm_gbs"],
            "unit": "GB/s", "frac": achieved / pk["hbm_gbs"], "traffic": None,
            "bytes_per_launch": b, "ms_per_launch": ms, "peak_source": pk["source"]}


def quad4_bytes(stats, geometric):
    """Algorithmic bytes of one 4-clique-kernel launch.

    Hash mode (quad4_kernel): per upper edge (p, a) the root row entry (8 B)
    and the two row offsets of a (16 B); per probe (a record of the row of a,
    or of the row of an X entry b, read and looked up in the row of p) the
    record (8 B); per rooted contribution the (b, d) edge metadata and the
    far vertex's flags, id and weight (4 + 13 B).
    Geometric mode (quad4g_kernel): it reads only the roots' rows and the
    members' data: per upper edge the record (8 B), the FP32 position
    (16 B), flags, catalogue id and full degree (9 B); per point its row
    start, length, flags, id and full degree (21 B).  Its pair tests run on
    shared memory.
    """
    if geometric:
        return 33 * stats["upper_edges"] + 21 * stats["n_points"]
    return 24 * stats["upper_edges"] + 8 * stats["probes"] + 17 * stats["rooted"]


def quad4_roofline(ctx, q_ms, pk, geometric):
    st = ctx.stats()
    ms = sum(q_ms) / len(q_ms)
    b = quad4_bytes(st, geometric)
    achieved = b / (ms * 1e-3) / 1e9
    kernel = "quad4g_kernel" if geometric else "quad4_kernel"
    return {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": pk["hbm_gbs"],
            "unit": "GB/s", "frac": achieved / pk["hbm_gbs"], "traffic": None,
            "bytes_per_launch": b, "ms_per_launch": ms, "peak_source": pk["source"]}


def profiled_traffic(kernel, scale, workload="c2"):
    """DRAM bytes (read + write) per launch of `kernel` from the committed ncu
    summary profiles/<kernel>_<workload>.json, for the full-size workload
    only."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.json")
    if scale != 1.0 or not os.path.exists(p):
        return None
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["dram_bytes_read"]) + float(d["dram_bytes_write"])
    except Exception:
        return None
