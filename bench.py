"""Benchmark: 2/3/4PCF tuples binned per second on one B200.

Headline workload (one "step" = the whole hot path over one catalogue, from
the device-resident catalogue to the binned histograms): 100,000 Neyman-Scott
galaxies (10,000 parents, Poisson(10) children, Gaussian sigma 4 Mpc/h) and
300,000 uniform randoms in [0,1000]^3, lognormal(0, 0.3) weights, rmin 5,
rmax 25, 8 radial bins, 5 mu bins (line-of-sight binning on).  Each step
builds the cell index, the CSR neighbour graph and counts every triangle.

value      distinct triangles binned / second of device time (inputs in HBM)
e2e        the same through the public API with host inputs: pinned host ->
           device copy of the catalogue, the count, and the histogram read back
roofline   the triangle kernel: algorithmic bytes / its CUDA-event time, with
           its instruction-issue and shared-atomic rates (`issue`, `atomics`)
           from the committed ncu summary; `graph_roofline` the graph build
cpu_baseline  the CPU restatement of the reference algorithm (kd-tree range
           search, id-sorted rows, the reference's 3PCF loop) on the host cores
parity     the GPU result on the full catalogue against that CPU result
fp64_path  the same steps with every pair in FP64 (GR_OPT_PRECISION=1), and
           whether its counts and sums are identical to the FP32 path's

With one GPU the line also carries the other workloads as sub-records, each
with its device-time value, end-to-end value (host inputs), parity against
the oracle and CPU baseline:
pcf2       plain 2PCF: 20,000 + 50,000 uniform points in [0,1000]^3, rmin 10,
           rmax 50, 10 bins
quad       4PCF: 30,000 Neyman-Scott galaxies + 90,000 randoms in [0,300]^3,
           rmin 2, rmax 12, 4 bins (unit weights; lognormal weights beside it)
batched    2PCF over 125 regions with 60 Mpc/h buffers of 4M density-ramped
           Neyman-Scott galaxies + 8M randoms in [0,2000]^3 (rmin 10, rmax 60,
           12 bins, nmu 10): all regions in one graph-replayed launch against
           one launch per region, FP32 + guard band and plain FP64
adjoint    weighted 2PCF (rmin 10, rmax 40, 10 bins, nmu 4) and 3PCF (rmin 10,
           rmax 30, 6 bins) of 1M lognormal-weighted galaxies + 2M randoms and
           their weight adjoints, through the C ABI and through
           torch.autograd

--impl reference times the CPU restatement of the reference algorithm on
the headline workload (the Fortran reference itself cannot be built here).
Multi-GPU (torchrun): each rank runs its own independently seeded mock of the
same size (weak scaling, no collective on the data path); the sub-records
run with one GPU only.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
import types

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "2/3/4PCF tuples binned/s on 1 B200 (exact counts), batched+adjoint vs plain GPU"
WORKLOAD = "c2_3pcf"
L2_NOTE = "flushed between steps (256 MB write)"


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="workload scale (1.0 = full size)")
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sub-records", action="store_true",
                    help="headline line only (no pcf2 / quad / batched / adjoint sub-records)")
    ap.add_argument("--shard", action="store_true",
                    help="one catalogue over the ranks: slabs with Rmax halos and one all-reduce "
                         "of the histograms per step (strong scaling); default: one independent "
                         "mock per rank (weak scaling)")
    ap.add_argument("--workload", default="c2_3pcf",
                    choices=["c2_3pcf", "c1_2pcf", "c3_4pcf", "c4_batched", "c5_adjoint"],
                    help="c2_3pcf is the headline line; the others print one sub-record alone")
    return ap.parse_args(argv)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def rank_seed(rank):
    """Seed of rank `rank`'s mock: rank 0 uses the workload's own seed, the
    others independent ones (weak scaling over independent mocks)."""
    return None if rank == 0 else 1000 + rank


def reduce_over_ranks(value, op, device):
    """All-reduce one number over the ranks ('max' or 'sum')."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def make_catalogue(name, scale, seed=None):
    from gramsci_b200 import catalogs

    cat = catalogs.make(name, scale=scale, seed=seed)
    w = catalogs.normalise(cat.w, cat.n_data, cat.n_rand)
    return cat, w, catalogs.WORKLOADS[name]


def c2_config(cat, sp, scale, world, triangles, rooted, edges, parallelism=None):
    """The headline line's config: the same keys and values in both arms."""
    if parallelism is None:
        parallelism = f"replicas{world}" if world > 1 else "single"
    return {
        "workload": f"{WORKLOAD}: Neyman-Scott 3PCF, {cat.n_data} galaxies + {cat.n_rand} randoms, "
                    f"box {cat.meta['box']:.0f}, rmin {sp['rmin']}, rmax {sp['rmax']}, "
                    f"nbins {sp['nbins']}, nmu {sp['nmu']}, lognormal weights",
        "n_points": int(cat.n),
        "scale": scale,
        "l2": L2_NOTE,
        "parallelism": parallelism,
        "triangles_per_step": int(triangles),
        "rooted_per_step": int(rooted),
        "edges": int(edges),
    }


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region
    (every 20 ms; samples are time-stamped and only those inside the region
    passed to stop() are summarised)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # wait (bounded) for the first sample so that the region is covered
            t_end = time.monotonic() + 5.0
            while not self.lines and time.monotonic() < t_end:
                time.sleep(0.01)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def stop(self, t0=None, t1=None):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        inside = [ln for t, ln in self.lines if (t0 is None or t >= t0) and (t1 is None or t <= t1)]
        window = "timed region"
        if not inside:  # region shorter than the sampling period: nearest samples
            inside = [ln for _, ln in self.lines]
            window = "whole run (timed region shorter than the sampling period)"
        for ln in inside:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() in ("active", "0x1", "1"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "window": window}


class Clocked:
    """Clock samples around one timed region: `with Clocked(dev) as c: ...`,
    then c.clocks."""

    def __init__(self, device):
        self.s = ClockSampler(device)

    def __enter__(self):
        self.s.start()
        self.t0 = time.monotonic()
        return self

    def __exit__(self, *a):
        self.clocks = self.s.stop(self.t0, time.monotonic())


# ------------------------------------------------------------- CPU side ----
def cpu_flush(mb=256):
    """Write a buffer larger than the host's last-level cache (the CPU arm's
    counterpart of the GPU's L2 flush)."""
    buf = np.empty(mb * 1024 * 1024 // 8)
    buf.fill(1.0)
    return float(buf[-1])


def cpu_reference_run(cat, w, sp, threads, order=3, buffer=None, xyz=None, n_data=None):
    """The reference algorithm restated on the CPU (kd-tree graph build with
    id-sorted rows, then the 2PCF, 3PCF or 4PCF loop), timed on the host
    cores.  Returns the phase times and the oracle's result."""
    from oracle import oracle

    xyz = cat.xyz if xyz is None else xyz
    n_data = cat.n_data if n_data is None else n_data
    t0 = time.perf_counter()
    G = oracle.Graph(xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"], method="kdtree",
                     threads=threads)
    t1 = time.perf_counter()
    fn = {2: G.pcf2, 3: G.pcf3, 4: G.pcf4}[order]
    r = fn(w, n_data, buffer=buffer)
    t2 = time.perf_counter()
    rooted = int(r["counts"].sum())
    return dict(graph_s=t1 - t0, query_s=t2 - t1, total_s=t2 - t0, rooted=rooted,
                edges=int(G.nedges), result=r)


def subcube(cat, w, rmax, side, seed):
    """A seeded sub-cube of the catalogue for a bounded CPU sample: the points
    within `side`/2 + rmax of a random centre, those outside the inner cube
    of edge `side` marked as buffer points (neighbours only), so the roots
    keep their full neighbourhoods."""
    rng = np.random.default_rng(seed)
    lo, hi = cat.xyz.min(0), cat.xyz.max(0)
    c = rng.uniform(lo + side / 2 + rmax, hi - side / 2 - rmax)
    d = np.abs(cat.xyz - c).max(axis=1)
    sel = np.nonzero(d < side / 2 + rmax)[0]
    buf = (d[sel] >= side / 2).astype(np.int32)
    nd = int(np.sum(sel < cat.n_data))
    return cat.xyz[sel], w[sel], buf, nd, c.tolist()


def parity_record(got, ref, keys=("catsum",)):
    """GPU result against the oracle's on the same inputs: integer counts
    identical, and the relative error of the weighted sums per bin (each
    category sum has one sign, so its relative error is well defined; N2 is
    compared relative to the sum of the absolute category sums of its bin)."""
    rec = {"counts_exact": bool(np.array_equal(got["counts"], ref["counts"]))}
    for k in keys:
        den = np.abs(ref[k])
        err = np.abs(got[k] - ref[k])
        rel = np.where(den > 0, err / np.maximum(den, 1e-300), np.where(err > 0, np.inf, 0.0))
        rec[f"max_rel_{k}"] = float(rel.max()) if rel.size else 0.0
        if k == "catsum":
            # per bin: the largest relative error over the categories (last axis)
            per_bin = rel.reshape(-1, rel.shape[-1], order="F") if rel.ndim > 1 else rel
            per_bin = per_bin.max(axis=1) if per_bin.ndim > 1 else per_bin
            rec["per_bin_max_rel"] = [float(f"{x:.2g}") for x in per_bin]
            scale = np.abs(ref["catsum"]).sum(axis=-1)
            e2 = np.abs(got["N2"] - ref["N2"])
            rec["max_rel_N2"] = float(np.max(np.where(scale > 0, e2 / np.maximum(scale, 1e-300),
                                                      0.0)))
    return rec


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    cat, w, sp = make_catalogue(WORKLOAD, args.scale)
    for _ in range(max(0, args.warmup)):
        cpu_flush()
        r = cpu_reference_run(cat, w, sp, threads)
    times = []
    for _ in range(max(1, args.steps)):
        cpu_flush()
        r = cpu_reference_run(cat, w, sp, threads)
        times.append(r["total_s"])
    t = float(np.mean(times))
    rooted = r["rooted"]
    tri = rooted // 3  # no buffer points: every triangle is rooted at its three vertices
    value = tri / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "tuples/s",
        "n_gpus": world, "steps": max(1, args.steps), "warmup": max(0, args.warmup),
        "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded Neyman-Scott galaxies + uniform randoms)",
        "config": c2_config(cat, sp, args.scale, world, tri, rooted, r["edges"]),
        "cpu_baseline": {"value": value, "unit": "tuples/s", "cores": threads, "kind": "port",
                         "sample": f"the full {WORKLOAD} catalogue per step, kd-tree graph build "
                                   "+ 3PCF query (C++ OpenMP restatement of the reference "
                                   "algorithm; no Fortran compiler here), host caches flushed "
                                   "between steps"},
        "e2e": {"value": value, "unit": "tuples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "phases_s": {"graph": r["graph_s"], "query": r["query_s"]},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------- GPU side ----
def _ev():
    import torch

    return torch.cuda.Event(enable_timing=True)


def timed(fn, steps, stream, flush=None):
    """Device time (ms) of `fn` per call, CUDA events on `stream`, L2 flushed
    before each call when `flush` is given."""
    import torch

    ms = []
    for _ in range(steps):
        if flush is not None:
            flush.zero_()
        a, b = _ev(), _ev()
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    return ms


def e2e_loop(ctx, cat, w, count, stream, flush, steps, buffer=None):
    """End to end through the C ABI: pinned host catalogue (and buffer
    flags, when given) -> device, the count, results read back; the first
    two calls are warm-up."""
    import torch

    xyz_h = torch.from_numpy(cat.xyz).pin_memory()
    w_h = torch.from_numpy(w).pin_memory()
    b_h = None if buffer is None else torch.from_numpy(np.ascontiguousarray(buffer, np.int32)).pin_memory()
    out = {}

    def call():
        ctx._check(ctx._lib.gr_set_catalog(ctx._h, xyz_h.data_ptr(), w_h.data_ptr(),
                                           None if b_h is None else b_h.data_ptr(),
                                           cat.n_data, cat.n_rand))
        out["r"] = count()

    timed(call, 2, stream, flush)
    ms = timed(call, steps, stream, flush)
    e2e_loop.spread = [float(np.min(ms)), float(np.median(ms)), float(np.max(ms))]
    return float(np.mean(ms)), out["r"]


def device_info():
    import torch

    p = torch.cuda.get_device_properties(0)
    return {"name": p.name, "sms": p.multi_processor_count}


def run_ours(args):
    import torch

    rank, world, local = dist_env()
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    device = local if world > 1 else 0
    torch.cuda.set_device(device)
    from gramsci_b200 import api, roofline

    cat, w, sp = make_catalogue(WORKLOAD, args.scale, rank_seed(rank))
    stream = torch.cuda.current_stream()
    ctx = api.Context(device)
    ctx.set_stream(stream)
    ctx.set_precision(args.precision)
    xyz_d = torch.from_numpy(cat.xyz).to(f"cuda:{device}")
    w_d = torch.from_numpy(w).to(f"cuda:{device}")
    ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    ctx.set_catalog(xyz_d, w_d, cat.n_data)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{device}")

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    sampler = ClockSampler(device)
    sampler.start()
    # N2 / N3 as the reference computes them (no integer counts)
    for _ in range(args.warmup):
        ctx.count_3pcf(counts=False)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    t_region0 = time.monotonic()
    ev = [(_ev(), _ev()) for _ in range(args.steps)]
    q_ms, g_ms, tri, launches = [], [], 0, 0
    st = None
    for k in range(args.steps):
        flush.zero_()
        ev[k][0].record(stream)
        ctx.count_3pcf(counts=False)
        ev[k][1].record(stream)
        st = ctx.stats()
        q_ms.append(st["ms_query"])
        g_ms.append(st["ms_graph"])
        tri += st["tuples"]
        launches += st["kernel_launches"]
    torch.cuda.synchronize()
    t_region1 = time.monotonic()
    barrier()
    clocks = sampler.stop(t_region0, t_region1)
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = float(sum(step_ms))
    t_max = total_ms
    tri_all = tri
    if world > 1:
        t_max = reduce_over_ranks(total_ms, "max", f"cuda:{device}")
        tri_all = reduce_over_ranks(tri, "sum", f"cuda:{device}")
    value = tri_all / (t_max / 1e3)

    # end to end through the public API: pinned host catalogue -> device,
    # count, histograms back to the host, every step
    e2e_t, out = e2e_loop(ctx, cat, w, lambda: ctx.count_3pcf(counts=False), stream, flush,
                          max(3, min(args.steps, 20)))
    e2e_tri = ctx.stats()["tuples"]
    if world > 1:
        e2e_t = reduce_over_ranks(e2e_t, "max", f"cuda:{device}")
    e2e_value = e2e_tri * world / (e2e_t / 1e3)
    nh = out["catsum"].size
    h2d = int(cat.xyz.nbytes + w.nbytes)
    d2h = int(nh * 8 * 2 + 8 * 8)

    # roofline of the triangle kernel (algorithmic bytes over its event time)
    # with its issue and shared-atomic rates, and of the graph build
    pk = roofline.peaks()
    rf = roofline.tri3_roofline(ctx, q_ms, pk)
    rf["traffic"] = roofline.profiled_traffic("tri3_kernel", args.scale)
    dev = device_info()
    sm_mhz = clocks.get("sm_mhz")
    prof = roofline.profile("tri3_kernel", "c2") if args.scale == 1.0 else None
    rf["issue"] = roofline.issue_roofline(prof, st["tuples"], rf["ms_per_launch"], sm_mhz, dev["sms"])
    rf["atomics"] = roofline.atomic_roofline(prof, st["tuples"], rf["ms_per_launch"], sm_mhz,
                                             dev["sms"])
    gprof = roofline.profile("csr_fill_kernel", "c2") if args.scale == 1.0 else None
    gtraffic = (float(gprof["dram_bytes_read"]) + float(gprof["dram_bytes_write"])) if gprof else None
    grf = roofline.graph_roofline(st, float(np.mean(g_ms)), pk, gtraffic)
    grf["issue"] = roofline.issue_roofline(gprof, st["upper_edges"], grf["ms_per_launch"], sm_mhz,
                                           dev["sms"])

    line = {
        "metric": METRIC, "value": value, "unit": "tuples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded Neyman-Scott galaxies + uniform randoms)",
        "config": c2_config(cat, sp, args.scale, world, st["tuples"], st["rooted"], st["n_edges"]),
        "stats": {"precision": args.precision, "fp64_rechecks": st["fp64_rechecks"],
                  "fp64_recheck_fraction": st["fp64_rechecks"] / max(1, st["candidates"]),
                  "upper_edges": st["upper_edges"], "probes": st["probes"],
                  "phase_ms": {"index": st["ms_index"], "graph": st["ms_graph"],
                               "query": st["ms_query"]}},
        "e2e": {"value": e2e_value, "unit": "tuples/s", "h2d_bytes_per_step": h2d,
                "ms_per_step": e2e_t, "ms_min_median_max": e2e_loop.spread,
                "d2h_bytes_per_step": d2h},
        "roofline": roofline.mark_binding(rf),
        "graph_roofline": roofline.mark_binding(grf),
        "clocks": clocks,
        "gpu_launches": launches,
        "device": dev,
    }
    ref32 = None
    if world == 1 and args.precision == "f32":
        # the 3PCF workload's precision comparison: the same steps through
        # the plain FP64 path (every pair in FP64 arithmetic); results must
        # be identical
        ref32 = ctx.count_3pcf()
        ctx.set_catalog(xyz_d, w_d, cat.n_data)
        ctx.set_precision("f64")
        for _ in range(args.warmup):
            ctx.count_3pcf(counts=False)
        n64 = max(1, min(args.steps, 50))
        ms64 = float(np.mean(timed(lambda: ctx.count_3pcf(counts=False), n64, stream, flush)))
        ref64 = ctx.count_3pcf()
        st64 = ctx.stats()
        same = all(np.array_equal(ref32[k], ref64[k]) for k in ("counts", "catsum", "N2", "N3"))
        line["fp64_path"] = {"ms_per_step": ms64, "value": st64["tuples"] / (ms64 / 1e3),
                             "steps": n64, "identical_to_fp32_path": bool(same),
                             "phase_ms": {"index": st64["ms_index"], "graph": st64["ms_graph"],
                                          "query": st64["ms_query"]}}
        ctx.set_precision("f32")
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        r = cpu_reference_run(cat, w, sp, threads)
        line["cpu_baseline"] = {
            "value": (r["rooted"] // 3) / r["total_s"], "unit": "tuples/s", "cores": threads,
            "kind": "port",
            "sample": f"the full {WORKLOAD} catalogue once: kd-tree graph build "
                      f"{r['graph_s']:.2f} s + 3PCF query {r['query_s']:.2f} s "
                      "(C++ OpenMP restatement of the reference algorithm)"}
        if ref32 is not None:
            line["parity"] = parity_record(ref32, r["result"])
            line["parity"]["against"] = "oracle (FP64 CPU restatement) on the same full catalogue"
    ctx.close()
    del xyz_d, w_d
    if rank == 0 and world == 1 and not args.no_sub_records:
        for key, fn in (("pcf2", sub_pcf2), ("quad", sub_quad), ("batched", sub_batched),
                        ("adjoint", sub_adjoint)):
            torch.cuda.empty_cache()
            try:
                line[key] = fn(args, stream, flush)
            except Exception as e:  # recorded, not hidden: the line says what failed
                line[key] = {"error": f"{type(e).__name__}: {e}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


# --------------------------------------------------------- sub-records ----
def sub_pcf2(args, stream, flush):
    """Plain 2PCF (20,000 + 50,000 uniform points, rmin 10, rmax 50, 10
    bins): pairs binned per second of device time, end to end, parity and
    the CPU restatement."""
    import torch

    from gramsci_b200 import api, roofline

    name = "c1_2pcf"
    cat, w, sp = make_catalogue(name, args.scale)
    ctx = api.Context(0)
    ctx.set_stream(stream)
    ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    ctx.set_catalog(torch.from_numpy(cat.xyz).cuda(), torch.from_numpy(w).cuda(), cat.n_data)
    steps = max(3, min(args.steps, 50))
    for _ in range(max(3, args.warmup)):
        ctx.count_2pcf()
    with Clocked(0) as ck:
        ms = timed(ctx.count_2pcf, steps, stream, flush)
    st = ctx.stats()
    got = ctx.count_2pcf()
    e2e_ms, _ = e2e_loop(ctx, cat, w, ctx.count_2pcf, stream, flush, steps)
    pairs = st["tuples"]
    rec = {"workload": f"{name}: {cat.n_data} uniform galaxies + {cat.n_rand} uniform randoms, box "
                       f"{cat.meta['box']:.0f}, rmin {sp['rmin']}, rmax {sp['rmax']}, "
                       f"nbins {sp['nbins']}, unit weights",
           "unit": "pairs/s", "value": pairs / (np.mean(ms) / 1e3), "ms_per_step": float(np.mean(ms)),
           "steps": steps, "pairs_per_step": pairs, "l2": L2_NOTE,
           "e2e": {"value": pairs / (e2e_ms / 1e3), "unit": "pairs/s",
                   "h2d_bytes_per_step": int(cat.xyz.nbytes + w.nbytes),
                   "d2h_bytes_per_step": int(sum(v.nbytes for v in got.values()))},
           "clocks": ck.clocks, "phase_ms": {"index": st["ms_index"], "query": st["ms_query"]},
           "fp64_recheck_fraction": st["fp64_rechecks"] / max(1, st["candidates"])}
    # the pair sweep's FP32 arithmetic over its own device time
    rec["roofline"] = roofline.mark_binding(
        {"kernel": "pair sweep", "ms": st["ms_query"],
         "fp32": roofline.fp32_binning_roofline(
             int(got["counts"].sum()), sp["nmu"], st["ms_query"], ck.clocks.get("sm_mhz"),
             torch.cuda.get_device_properties(0).multi_processor_count)})
    ctx.close()
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        r = cpu_reference_run(cat, w, sp, threads, order=2)
        rec["cpu_baseline"] = {"value": (r["rooted"] // 2) / r["total_s"], "unit": "pairs/s",
                               "cores": threads, "kind": "port",
                               "sample": f"the full {name} catalogue once: kd-tree graph build "
                                         f"{r['graph_s']:.2f} s + 2PCF query {r['query_s']:.2f} s"}
        rec["parity"] = parity_record(got, r["result"])
    return rec


def sub_quad(args, stream, flush):
    """4PCF on the small dense clustered set (30k galaxies + 90k randoms in a
    300 Mpc/h box, unit weights): rooted 4-clique contributions binned per
    second of device time (index + graph + 4-clique kernel per step), end to
    end, the geometric 4-clique kernel's roofline, parity and the CPU
    restatement; beside it the same catalogue with lognormal weights
    (weighted forward pass, adjoint and their parity)."""
    import torch

    from gramsci_b200 import api, catalogs, roofline

    name = "c3_4pcf"
    cat, w, sp = make_catalogue(name, args.scale)
    ctx = api.Context(0)
    ctx.set_stream(stream)
    ctx.set_precision(args.precision)
    xyz_d = torch.from_numpy(cat.xyz).cuda()
    ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    ctx.set_catalog(xyz_d, torch.from_numpy(w).cuda(), cat.n_data)
    # the geometric 4-clique kernel: what the automatic choice takes for
    # unit weights with rows of at most 256 neighbours, set explicitly so
    # that the roofline below names the kernel that ran
    ctx.set_clique_mode("geometric")
    steps = max(3, min(args.steps, 50))
    for _ in range(max(3, args.warmup)):
        ctx.count_4pcf()
    q_ms, rooted, launches = [], 0, 0
    with Clocked(0) as ck:
        ev = []
        for _ in range(steps):
            flush.zero_()
            a, b = _ev(), _ev()
            a.record(stream)
            ctx.count_4pcf()
            b.record(stream)
            ev.append((a, b))
            s = ctx.stats()
            q_ms.append(s["ms_query"])
            rooted += s["rooted"]
            launches += s["kernel_launches"]
        torch.cuda.synchronize()
    st = ctx.stats()
    total_ms = float(sum(a.elapsed_time(b) for a, b in ev))
    got = ctx.count_4pcf()
    e2e_ms, out = e2e_loop(ctx, cat, w, ctx.count_4pcf, stream, flush, max(3, min(args.steps, 10)))
    pk = roofline.peaks()
    rf = roofline.quad4_roofline(ctx, q_ms, pk, geometric=True)
    rf["traffic"] = roofline.profiled_traffic("quad4g_kernel", args.scale, "c3")
    # issue ceiling: warp instructions per 4-clique from the committed ncu summary
    prof = roofline.profile("quad4g_kernel", "c3") if args.scale == 1.0 else None
    n_sm = torch.cuda.get_device_properties(0).multi_processor_count
    rf["issue"] = roofline.issue_roofline(prof, st["tuples"], rf["ms_per_launch"],
                                          ck.clocks.get("sm_mhz"), n_sm)
    # lognormal weights (automatic kernel choice): weighted sums and adjoint
    ctx.set_clique_mode("auto")
    rng = np.random.default_rng(5)
    wl = catalogs.normalise(rng.lognormal(0.0, 0.3, cat.n), cat.n_data, cat.n_rand)
    ctx.set_catalog(xyz_d, torch.from_numpy(wl).cuda(), cat.n_data)
    fwd, adj = [], []
    for k in range(4):
        # N2, N3, discN, discR as the reference computes them (no counts)
        r = ctx.count_4pcf(counts=False)
        fwd.append(ctx.stats()["ms_query"])
        cot = [rng.normal(size=r[x].shape) for x in ("N2", "N3", "discN", "discR")]
        ctx.adjoint_4pcf(*cot)
        adj.append(ctx.stats()["ms_query"])
    gotw = ctx.count_4pcf()  # with the counts, for the parity record
    ctx.close()
    rec = {"workload": f"{name}: Neyman-Scott 4PCF, {cat.n_data} galaxies + {cat.n_rand} randoms, "
                       f"box {cat.meta['box']:.0f}, rmin {sp['rmin']}, rmax {sp['rmax']}, "
                       f"nbins {sp['nbins']}, unit weights",
           "unit": "tuples/s", "tuples": "rooted 4-clique contributions (one per reference root)",
           "value": rooted / (total_ms / 1e3), "ms_per_step": total_ms / steps, "steps": steps,
           "cliques_per_step": st["tuples"], "rooted_per_step": st["rooted"], "l2": L2_NOTE,
           "phase_ms": {"index": st["ms_index"], "graph": st["ms_graph"], "query": st["ms_query"]},
           "e2e": {"value": st["rooted"] / (e2e_ms / 1e3), "unit": "tuples/s",
                   "h2d_bytes_per_step": int(cat.xyz.nbytes + w.nbytes),
                   "d2h_bytes_per_step": int(sum(v.nbytes for v in out.values()) + 64)},
           "roofline": roofline.mark_binding(rf), "clocks": ck.clocks, "gpu_launches": launches,
           "lognormal_weights": {"forward_query_ms": float(np.median(fwd[1:])),
                                 "adjoint_ms": float(np.median(adj[1:])),
                                 "adjoint_over_forward": float(np.median(adj[1:]) / np.median(fwd[1:])),
                                 "unit_weight_query_ms": float(np.median(q_ms))}}
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        r = cpu_reference_run(cat, w, sp, threads, order=4)
        rec["cpu_baseline"] = {"value": r["rooted"] / r["total_s"], "unit": "tuples/s",
                               "cores": threads, "kind": "port",
                               "sample": f"the full {name} catalogue once: kd-tree graph build "
                                         f"{r['graph_s']:.2f} s + 4PCF query {r['query_s']:.2f} s"}
        rec["parity"] = parity_record(got, r["result"], keys=("catsum", "dsum"))
        rw = cpu_reference_run(cat, wl, sp, threads, order=4)["result"]
        rec["lognormal_weights"]["parity"] = parity_record(gotw, rw, keys=("catsum", "dsum"))
    return rec


def sub_batched(args, stream, flush):
    """Batched regions: 2PCF of 4M density-ramped galaxies + 8M randoms over
    5^3 regions with Rmax buffers, all regions in one graph-replayed launch,
    against one launch per region on the same regions -- with the same FP32
    + guard-band kernels, and in the plain FP64 form."""
    import torch

    from gramsci_b200 import api, roofline

    name = "c4_batched"
    cat, w, sp = make_catalogue(name, args.scale)
    dev = torch.device("cuda:0")
    ctx = api.Context(0)
    ctx.set_stream(stream)
    ctx.set_precision(args.precision)
    xyz_d = torch.from_numpy(cat.xyz).to(dev)
    w_d = torch.from_numpy(w).to(dev)
    ctx.set_catalog(xyz_d, w_d, cat.n_data)
    ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    ctx.set_regions(sp["nsplit"])
    ref = ctx.count_2pcf_batched()
    regions = ctx.regions()
    sizes = [len(o) for o, _ in regions]
    reg_dev = []
    for o, bf in regions:
        if len(o) == 0:
            continue
        oi = torch.from_numpy(o.astype(np.int64)).to(dev)
        reg_dev.append((xyz_d[oi].contiguous(), w_d[oi].contiguous(),
                        torch.from_numpy(bf).to(dev), int(np.sum(o < cat.n_data))))

    def per_region(c):
        def run():
            tot = 0
            for x, ww, b, nd in reg_dev:
                c.set_catalog(x, ww, nd, buffer=b)
                tot = tot + c.count_2pcf()["counts"]
            per_region.tot = tot
        return run

    steps = max(1, min(args.steps, 10))
    for _ in range(max(1, args.warmup)):
        ctx.count_2pcf_batched()
    out = {}

    def batched():
        out["r"] = ctx.count_2pcf_batched()

    with Clocked(0) as ck:
        t_batch = timed(batched, steps, stream, flush)
    st = ctx.stats()
    res = {}
    for prec in ("f32", "f64"):
        c = api.Context(0)
        c.set_stream(stream)
        c.set_precision(prec)
        c.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
        run = per_region(c)
        run()  # warm-up: tunes the sweep per region class
        t = timed(run, max(1, min(steps, 3)), stream, flush)
        res[prec] = (float(np.median(t)), bool(np.array_equal(per_region.tot, out["r"]["counts"])))
        c.close()
    counts_equal = bool(np.array_equal(out["r"]["counts"], ref["counts"]))
    tb = float(np.median(t_batch))
    pairs = int(out["r"]["counts"].sum()) // 2
    rec = {"workload": f"{name}: {cat.n_data} galaxies + {cat.n_rand} randoms, box "
                       f"{cat.meta['box']:.0f}, rmin {sp['rmin']}, rmax {sp['rmax']}, "
                       f"{sp['nbins']} bins, nmu {sp['nmu']}, {len(regions)} regions with "
                       f"{sp['rmax']:.0f} Mpc/h buffers",
           "unit": "pairs/s", "value": pairs / (tb / 1e3), "batched_ms": tb, "steps": steps,
           "l2": "inputs larger than L2 (22.9M region members, 2.8 GB of layout) and flushed",
           "members": int(sum(sizes)), "region_members_min_max": [int(min(sizes)), int(max(sizes))],
           "pairs": pairs, "rooted": int(out["r"]["counts"].sum()),
           "candidates": st["candidates"], "fp64_rechecks": st["fp64_rechecks"],
           "per_region_ms": res["f32"][0], "per_region_plain_fp64_ms": res["f64"][0],
           "batched_over_per_region": res["f32"][0] / tb,
           "batched_over_per_region_plain_fp64": res["f64"][0] / tb,
           "per_region_form": "one gr_set_catalog + gr_count_2pcf call per region (its members and "
                              "buffer flags), same FP32 + guard-band kernels; the plain form runs "
                              "them in FP64",
           "identical_counts": {"batched_vs_first_call": counts_equal,
                                "per_region_sum_f32": res["f32"][1],
                                "per_region_sum_f64": res["f64"][1]},
           "clocks": ck.clocks}
    # issue and shared-atomic ceilings of the tile sweep, from its ncu summary
    # (10%-scale catalogue: the same density, so the same instructions per
    # pair test), over the whole batched call's device time (layout kernels
    # included: a lower bound for the sweep kernel alone)
    prof = roofline.profile("pair2_tile_kernel", "c4")
    n_sm = torch.cuda.get_device_properties(0).multi_processor_count
    rf = {"kernel": "pair2_tile_kernel", "ms": tb, "ms_is": "whole batched call"}
    rf["issue"] = roofline.issue_roofline(prof, st["candidates"], tb, ck.clocks.get("sm_mhz"), n_sm)
    rf["atomics"] = roofline.atomic_roofline(prof, st["candidates"], tb, ck.clocks.get("sm_mhz"), n_sm)
    rf["fp32"] = roofline.fp32_binning_roofline(rec["rooted"], sp["nmu"], tb, ck.clocks.get("sm_mhz"),
                                                n_sm)
    rec["roofline"] = roofline.mark_binding(rf)
    rec["fp64_recheck_fraction"] = st["fp64_rechecks"] / max(1, st["candidates"])
    ctx.close()
    del reg_dev, xyz_d, w_d
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        xs, ws, bs, nd, centre = subcube(cat, w, sp["rmax"], 240.0, seed=4)
        r = cpu_reference_run(cat, ws, sp, threads, order=2, buffer=bs, xyz=xs, n_data=nd)
        rate = (r["rooted"] / 2) / r["total_s"]
        rec["cpu_baseline"] = {
            "value": rate, "unit": "pairs/s", "cores": threads, "kind": "port",
            "sample": f"a seeded sub-cube of the catalogue (edge 240 Mpc/h around {np.round(centre, 1).tolist()}"
                      f", {len(xs)} points with a {sp['rmax']:.0f} Mpc/h buffer shell, "
                      f"{r['rooted']} rooted pairs): kd-tree graph build {r['graph_s']:.2f} s + 2PCF "
                      f"{r['query_s']:.2f} s; the whole job at this rate: {pairs / rate:.0f} s"}
    return rec


def sub_adjoint(args, stream, flush):
    """Adjoints: weighted 2PCF and 3PCF forward passes over 1M lognormal-
    weighted galaxies + 2M randoms and their weight adjoints, timed on the
    C ABI (count, then adjoint on the same graph) and through
    torch.autograd (forward pass, then loss.backward())."""
    import torch

    from gramsci_b200 import api, autograd

    rec = {}
    for name, order in (("c5_adjoint_2pcf", 2), ("c5_adjoint_3pcf", 3)):
        cat, w, sp = make_catalogue(name, args.scale)
        xyz_d = torch.from_numpy(cat.xyz).cuda()
        w_d = torch.from_numpy(w).cuda()
        ctx = api.Context(0)
        ctx.set_stream(stream)
        ctx.set_catalog(xyz_d, w_d, cat.n_data)
        ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
        rng = np.random.default_rng(5)
        count = ctx.count_2pcf if order == 2 else ctx.count_3pcf
        adjoint = ctx.adjoint_2pcf if order == 2 else ctx.adjoint_3pcf
        fwd, adj = [], []
        with Clocked(0) as ck:
            for k in range(4):
                r = count()
                s = ctx.stats()
                c2 = rng.normal(size=r["N2"].shape)
                c3 = rng.normal(size=r["N3"].shape)
                adjoint(c2, c3)
                a = ctx.stats()
                if k > 0:
                    fwd.append(s["ms_total"])
                    adj.append(a["ms_total"])
        ctx.close()
        # through torch.autograd: the same weights as a CUDA tensor
        wt = w_d.clone().requires_grad_(True)
        fn = autograd.pcf2 if order == 2 else autograd.pcf3
        bins = (sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
        af, ab = [], []
        for k in range(3):
            wt.grad = None
            a0, a1, a2 = _ev(), _ev(), _ev()
            a0.record(stream)
            N2, N3 = fn(wt, xyz_d, cat.n_data, *bins)
            a1.record(stream)
            loss = (torch.from_numpy(c2).cuda() * N2).sum() + (torch.from_numpy(c3).cuda() * N3).sum()
            loss.backward()
            a2.record(stream)
            torch.cuda.synchronize()
            if k > 0:
                af.append(a0.elapsed_time(a1))
                ab.append(a1.elapsed_time(a2))
        rec[name] = {"n_points": int(cat.n), "tuples": int(s["tuples"]),
                     "forward_ms": float(np.median(fwd)), "adjoint_ms": float(np.median(adj)),
                     "adjoint_over_forward": float(np.median(adj) / np.median(fwd)),
                     "autograd_forward_ms": float(np.median(af)),
                     "autograd_backward_ms": float(np.median(ab)),
                     "autograd_backward_over_forward": float(np.median(ab) / np.median(af)),
                     "timing": "C ABI: device time of the whole call (index, graph, kernels) as "
                               "gr_get_stats reports it; autograd: CUDA events around the forward "
                               "call and around loss.backward()",
                     "clocks": ck.clocks}
        if not args.no_cpu_baseline:
            from oracle import oracle

            threads = os.cpu_count() or 1
            side = 160.0 if order == 2 else 120.0
            xs, ws, bs, nd, centre = subcube(cat, w, sp["rmax"], side, seed=5)
            t0 = time.perf_counter()
            G = oracle.Graph(xs, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"], method="kdtree",
                             threads=threads)
            t1 = time.perf_counter()
            rr = (G.pcf2 if order == 2 else G.pcf3)(ws, nd, buffer=bs)
            t2 = time.perf_counter()
            cs = np.random.default_rng(6).normal(size=rr["N2"].shape)
            (G.adjoint2 if order == 2 else G.adjoint3)(ws, nd, cs, buffer=bs)
            t3 = time.perf_counter()
            k = order
            units = int(rr["counts"].sum())
            rec[name]["cpu_baseline"] = {
                "value": units / (t2 - t0), "unit": "rooted tuples/s", "cores": threads,
                "kind": "port", "adjoint_s": t3 - t2, "forward_s": t2 - t0,
                "sample": f"a seeded sub-cube (edge {side:.0f} Mpc/h, {len(xs)} points with a "
                          f"{sp['rmax']:.0f} Mpc/h buffer shell, {units} rooted {k}-tuples): "
                          f"kd-tree graph {t1 - t0:.2f} s + query {t2 - t1:.2f} s, adjoint "
                          f"{t3 - t2:.2f} s (oracle restatement)"}
        del xyz_d, w_d, wt
        torch.cuda.empty_cache()
    return rec


def run_sub(args, fn):
    import torch

    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda:0")
    rec = fn(args, stream, flush)
    print(json.dumps({"metric": METRIC, "workload": args.workload, "scale": args.scale, **rec}),
          flush=True)
    return 0


def run_shard(args):
    """The headline workload as ONE catalogue over the ranks
    (gramsci_b200/shard.py): every rank holds the whole catalogue, counts the
    slab of roots it owns with the slab's Rmax halo as buffer points, and one
    all-reduce (NCCL, sum) of the histograms per step gives every rank the
    whole catalogue's counts.  A step is the rank's count plus the
    all-reduce; the tuples are the whole catalogue's distinct triangles
    (counted once on rank 0 before the timed region), so the work is fixed as
    the ranks grow (strong scaling)."""
    import torch

    rank, world, local = dist_env()
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    device = local if world > 1 else 0
    torch.cuda.set_device(device)
    dv = f"cuda:{device}"
    from gramsci_b200 import api, roofline, shard

    cat, w, sp = make_catalogue(WORKLOAD, args.scale)  # the same catalogue on every rank
    stream = torch.cuda.current_stream()
    ctx = api.Context(device)
    ctx.set_stream(stream)
    ctx.set_precision(args.precision)
    ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dv)
    full, full_st = None, None
    if rank == 0:
        ctx.set_catalog(torch.from_numpy(cat.xyz).to(dv), torch.from_numpy(w).to(dv), cat.n_data)
        full = ctx.count_3pcf()
        full_st = ctx.stats()
    sx, sw, snd, sb, idx = shard.shard(cat.xyz, w, cat.n_data, rank, world, sp["rmax"])
    xyz_d = torch.from_numpy(sx).to(dv)
    w_d = torch.from_numpy(sw).to(dv)
    b_d = torch.from_numpy(sb).to(dv)
    ctx.set_catalog(xyz_d, w_d, snd, buffer=b_d)

    def step(counts=False):
        out = ctx.count_3pcf(counts=counts)
        if world > 1:
            shard.allreduce_counts(out, device=dv)
        return out

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    sampler = ClockSampler(device)
    sampler.start()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    t_region0 = time.monotonic()
    ev = [(_ev(), _ev()) for _ in range(args.steps)]
    q_ms, launches, out = [], 0, None
    for k in range(args.steps):
        flush.zero_()
        ev[k][0].record(stream)
        out = step()
        ev[k][1].record(stream)
        st = ctx.stats()
        q_ms.append(st["ms_query"])
        launches += st["kernel_launches"]
    torch.cuda.synchronize()
    t_region1 = time.monotonic()
    barrier()
    clocks = sampler.stop(t_region0, t_region1)
    total_ms = float(sum(a.elapsed_time(b) for a, b in ev))
    t_max = reduce_over_ranks(total_ms, "max", dv) if world > 1 else total_ms
    # end to end: the rank's shard (coordinates, weights, buffer flags) from
    # pinned host memory, the count, the all-reduce, the histograms back
    shard_cat = types.SimpleNamespace(xyz=sx, n_data=snd, n_rand=int(sx.shape[0]) - snd)
    e2e_t, _ = e2e_loop(ctx, shard_cat, sw, step, stream, flush, max(3, min(args.steps, 20)),
                        buffer=sb)
    if world > 1:
        e2e_t = reduce_over_ranks(e2e_t, "max", dv)
    # parity: the sharded counts (with the integer counts) against rank 0's
    # call on the whole catalogue; every rank takes this step
    chk = step(counts=True)
    pk = roofline.peaks()
    rf = roofline.tri3_roofline(ctx, q_ms, pk)
    rf["of"] = "rank 0's slab"
    line = None
    if rank == 0:
        tri = int(full_st["tuples"])
        value = tri * args.steps / (t_max / 1e3)
        nh = out["catsum"].size
        line = {
            "metric": METRIC, "value": value, "unit": "tuples/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32+f64", "data": "synthetic (seeded Neyman-Scott galaxies + uniform randoms)",
            "config": c2_config(cat, sp, args.scale, world, tri, full_st["rooted"],
                                full_st["n_edges"], parallelism=f"slabs{world}"),
            "e2e": {"value": tri / (e2e_t / 1e3), "unit": "tuples/s", "ms_per_step": e2e_t,
                    "h2d_bytes_per_step": int(sx.nbytes + sw.nbytes + sb.nbytes),
                    "d2h_bytes_per_step": int(nh * 8 * 2 + 8 * 8),
                    "ms_min_median_max": e2e_loop.spread},
            "roofline": rf,
            "clocks": clocks,
            "gpu_launches": launches,
            "device": device_info(),
            "shard": {"points": int(sx.shape[0]), "roots": int(np.count_nonzero(sb == 0)),
                      "catalogue_points": int(cat.n), "collective": "all_reduce(sum) per step"
                      if world > 1 else "none"},
            "parity": {"against": "one call on the whole catalogue on rank 0",
                       "counts_exact": bool(np.array_equal(chk["counts"], full["counts"])),
                       "max_rel_catsum": float(np.max(np.abs(chk["catsum"] - full["catsum"]) /
                                                      np.maximum(np.abs(full["catsum"]), 1e-300)))},
        }
    ctx.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.shard and args.workload == "c2_3pcf":
        return run_shard(args)
    subs = {"c1_2pcf": sub_pcf2, "c3_4pcf": sub_quad, "c4_batched": sub_batched,
            "c5_adjoint": sub_adjoint}
    if args.workload in subs:
        return run_sub(args, subs[args.workload])
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
