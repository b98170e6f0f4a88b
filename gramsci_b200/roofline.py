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


def profile(kernel, workload):
    """The committed ncu summary profiles/<kernel>_<workload>.json, or None."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.json")
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return None


def issue_roofline(prof, units, ms, sm_mhz, n_sm):
    """Instruction-issue ceiling of a kernel: warp instructions per work unit
    from its committed ncu summary (warp_instructions / units of the profiled
    launch) times the units of this launch, over the issue slots of the
    launch (n_sm SMs x 4 schedulers x SM clock x duration).  None without a
    profile or a clock reading."""
    if not prof or not sm_mhz or not ms or "warp_instructions" not in prof or not prof.get("units"):
        return None
    per_unit = float(prof["warp_instructions"]) / float(prof["units"])
    achieved = per_unit * units / (ms * 1e-3) / 1e9
    peak = n_sm * 4 * sm_mhz * 1e6 / 1e9
    return {"unit": "G warp instructions/s", "achieved": achieved, "peak": peak,
            "frac": achieved / peak, "warp_inst_per_unit": per_unit,
            "work_unit": prof.get("unit_name", "tuple"), "source": prof.get("file")}


def atomic_roofline(prof, units, ms, sm_mhz, n_sm):
    """Shared-memory atomic rate of a binning kernel: shared atomic
    wavefronts per work unit from its ncu summary times this launch's units,
    per second, against one shared-memory wavefront per SM per cycle (the
    shared-memory pipe's peak)."""
    if not prof or not sm_mhz or not ms or "shared_atomic_wavefronts" not in prof or not prof.get("units"):
        return None
    per_unit = float(prof["shared_atomic_wavefronts"]) / float(prof["units"])
    rate = per_unit * units / (ms * 1e-3) / 1e9
    peak = n_sm * sm_mhz * 1e6 / 1e9
    return {"unit": "G shared atomic wavefronts/s", "achieved": rate, "peak": peak,
            "frac": rate / peak, "wavefronts_per_unit": per_unit, "source": prof.get("file")}


def graph_bytes(stats):
    """Algorithmic bytes of the one-pass graph build (csr_fill_kernel): each
    point's FP32 position read once (16 B) and its row start, length and
    full degree written (16 B), and one 8-byte record written per upper
    edge."""
    return 32 * stats["n_points"] + 8 * stats["upper_edges"]


def graph_roofline(stats, ms, pk, traffic):
    b = graph_bytes(stats)
    achieved = b / (ms * 1e-3) / 1e9
    return {"bound": "hbm", "kernel": "csr_fill_kernel", "achieved": achieved,
            "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": achieved / pk["hbm_gbs"],
            "traffic": traffic, "bytes_per_launch": b, "ms_per_launch": ms,
            "peak_source": pk["source"]}


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


def fp32_binning_roofline(binned_directed_pairs, nmu, ms, sm_mhz, n_sm):
    """FP32 arithmetic of 2PCF binning against the chip's nominal FP32 rate:
    per binned directed pair 11 operations without mu bins (3 subtractions,
    5 for the squared separation, a square root, 2 for the bin) and 27 with
    them (16 more for the midpoint, dot product, norms and reciprocal square
    root), an FMA counted as 2; the peak is 128 FP32 lanes x 2 per SM per
    cycle at the sampled SM clock.  Candidate pairs outside the range are
    not credited.  None without a clock reading."""
    if not sm_mhz or not ms:
        return None
    f = 11 if nmu <= 1 else 27
    achieved = binned_directed_pairs * f / (ms * 1e-3) / 1e12
    peak = n_sm * 128 * 2 * sm_mhz * 1e6 / 1e12
    return {"unit": "TFLOP/s", "achieved": achieved, "peak": peak, "frac": achieved / peak,
            "flop_per_binned_pair": f, "peak_kind": "nominal FP32 FMA rate at the sampled clock"}


def mark_binding(rf):
    """Name the ceiling that binds a kernel: of its fractions (the top-level
    one, against HBM, and those of its `issue`, `atomics` and `fp32`
    entries) the largest, as rf["binding"] with rf["binding_frac"].  A
    kernel far below its HBM ceiling but near its issue ceiling is
    issue-bound, and the line says so.  Returns rf."""
    fr = {}
    if isinstance(rf.get("frac"), (int, float)):
        fr[rf.get("bound", "hbm")] = float(rf["frac"])
    for k in ("issue", "atomics", "fp32"):
        v = rf.get(k)
        if isinstance(v, dict) and isinstance(v.get("frac"), (int, float)):
            fr[k] = float(v["frac"])
    if fr:
        b = max(fr, key=fr.get)
        rf["binding"] = b
        rf["binding_frac"] = fr[b]
    return rf
