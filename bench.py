"""Benchmark: 3PCF triangles binned per second on one B200 (clustered catalogue).

Workload (one "step" = the whole hot path over one catalogue, from the
device-resident catalogue to the binned histograms): 100,000 Neyman-Scott
galaxies (10,000 parents, Poisson(10) children, Gaussian sigma 4 Mpc/h) and
300,000 uniform randoms in [0,1000]^3, lognormal(0, 0.3) weights, rmin 5,
rmax 25, 8 radial bins, 5 mu bins (line-of-sight binning on).  Each step
builds the cell index, the CSR neighbour graph and counts every triangle.

value      distinct triangles binned / second of device time (inputs in HBM)
e2e        the same through the public API with host inputs: pinned host ->
           device copy of the catalogue, the count, and the histogram read back
roofline   the triangle kernel: algorithmic bytes / its CUDA-event time
cpu_baseline  the CPU restatement of the reference algorithm (kd-tree range
           search, id-sorted rows, the reference's 3PCF loop) on the host cores
fp64_path  the same steps with every pair in FP64 (GR_OPT_PRECISION=1), and
           whether its counts and sums are identical to the FP32 path's

--impl reference times that CPU restatement on the same workload (it is the
reference's algorithm; the Fortran reference itself cannot be built here).
Multi-GPU (torchrun): each rank runs its own independently seeded mock of the
same size (weak scaling, no collective on the data path).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "2/3/4PCF tuples binned/s on 1 B200 (exact counts), batched+adjoint vs plain GPU"
WORKLOAD = "c2_3pcf"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="workload scale (1.0 = full size)")
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="c2_3pcf",
                    choices=["c2_3pcf", "c3_4pcf", "c4_batched", "c5_adjoint"],
                    help="c2_3pcf is the headline line; c4_batched and c5_adjoint print the "
                         "batched-vs-per-region and adjoint-vs-forward comparisons")
    return ap.parse_args()


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


def make_catalogue(scale, seed):
    from gramsci_b200 import catalogs

    cat = catalogs.make(WORKLOAD, scale=scale, seed=seed)
    w = catalogs.normalise(cat.w, cat.n_data, cat.n_rand)
    return cat, w, catalogs.WORKLOADS[WORKLOAD]


def workload_config(cat, sp, scale, extra=None):
    cfg = {
        "workload": f"{WORKLOAD}: Neyman-Scott 3PCF, {cat.n_data} galaxies + {cat.n_rand} randoms, "
                    f"box {cat.meta['box']:.0f}, rmin {sp['rmin']}, rmax {sp['rmax']}, "
                    f"nbins {sp['nbins']}, nmu {sp['nmu']}, lognormal weights",
        "n_points": int(cat.n),
        "scale": scale,
        "l2": "flushed between steps (256 MB write)",
    }
    if extra:
        cfg.update(extra)
    return cfg


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


def cpu_reference_run(cat, w, sp, threads):
    """The reference algorithm restated on the CPU (kd-tree graph build with
    id-sorted rows, then the 3PCF loop), timed on the host cores."""
    from oracle import oracle

    t0 = time.perf_counter()
    G = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"], method="kdtree",
                     threads=threads)
    t1 = time.perf_counter()
    r = G.pcf3(w, cat.n_data)
    t2 = time.perf_counter()
    rooted = int(r["counts"].sum())
    return dict(graph_s=t1 - t0, query_s=t2 - t1, total_s=t2 - t0, rooted=rooted,
                triangles=rooted // 3)


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import oracle

    threads = os.cpu_count() or 1
    cat, w, sp = make_catalogue(args.scale, None)
    cfg = workload_config(cat, sp, args.scale)
    times, tri = [], 0
    nsteps = max(1, min(args.steps, 3))
    r = cpu_reference_run(cat, w, sp, threads)  # warm-up (page-in, thread pool)
    for _ in range(nsteps):
        r = cpu_reference_run(cat, w, sp, threads)
        times.append(r["total_s"])
        tri = r["triangles"]
    t = float(np.mean(times))
    value = tri / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "tuples/s",
        "n_gpus": world, "steps": nsteps, "warmup": 1, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Neyman-Scott + uniform randoms)", "config": cfg,
        "cpu_baseline": {"value": value, "unit": "tuples/s", "cores": threads, "kind": "port",
                         "sample": f"full {WORKLOAD} catalogue, {nsteps} timed runs, "
                                   "kd-tree graph build + 3PCF query (C++ OpenMP restatement "
                                   "of the reference algorithm; no Fortran compiler here)"},
        "e2e": {"value": value, "unit": "tuples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "phases_s": {"graph": r["graph_s"], "query": r["query_s"]},
    }
    print(json.dumps(line), flush=True)
    return 0


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
    from gramsci_b200 import api

    cat, w, sp = make_catalogue(args.scale, rank_seed(rank))
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
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    q_ms, tri, launches = [], 0, 0
    st = None
    for k in range(args.steps):
        flush.zero_()
        ev[k][0].record(stream)
        ctx.count_3pcf(counts=False)
        ev[k][1].record(stream)
        st = ctx.stats()
        q_ms.append(st["ms_query"])
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
    xyz_h = torch.from_numpy(cat.xyz).pin_memory()
    w_h = torch.from_numpy(w).pin_memory()
    e2e_ms = []
    n_e2e = max(3, min(args.steps, 20))
    for k in range(n_e2e + 2):  # the first two calls are warm-up
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ctx._check(ctx._lib.gr_set_catalog(ctx._h, xyz_h.data_ptr(), w_h.data_ptr(), None,
                                           cat.n_data, cat.n_rand))
        out = ctx.count_3pcf(counts=False)
        b.record(stream)
        torch.cuda.synchronize()
        if k >= 2:
            e2e_ms.append(a.elapsed_time(b))
    e2e_tri = ctx.stats()["tuples"]
    e2e_t = float(np.mean(e2e_ms))
    if world > 1:
        e2e_t = reduce_over_ranks(e2e_t, "max", f"cuda:{device}")
    e2e_value = e2e_tri * world / (e2e_t / 1e3)
    nh = out["catsum"].size
    h2d = int(cat.xyz.nbytes + w.nbytes)
    d2h = int(nh * 8 * 2 + 8 * 8)

    # roofline of the triangle kernel: algorithmic CSR bytes it must stream
    # (8 B per upper-row entry read: the root's row and, per neighbour a, the
    # row of a; 16 B of row offsets per neighbour) over its event time
    from gramsci_b200 import roofline

    peaks = roofline.peaks()
    rf = roofline.tri3_roofline(ctx, q_ms, peaks)
    rf["traffic"] = roofline.profiled_traffic("tri3_kernel", args.scale)

    line = {
        "metric": METRIC, "value": value, "unit": "tuples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded Neyman-Scott galaxies + uniform randoms)",
        "config": workload_config(cat, sp, args.scale, {
            "parallelism": f"replicas{world}" if world > 1 else "single",
            "precision": args.precision,
            "triangles_per_step": st["tuples"], "rooted_per_step": st["rooted"],
            "edges": st["n_edges"], "fp64_rechecks": st["fp64_rechecks"],
            "phase_ms": {"index": st["ms_index"], "graph": st["ms_graph"], "query": st["ms_query"]},
        }),
        "e2e": {"value": e2e_value, "unit": "tuples/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "roofline": rf,
        "clocks": clocks,
        "gpu_launches": launches,
    }
    if world == 1 and args.precision == "f32":
        # the 3PCF workload's precision comparison: the same steps through
        # the plain FP64 path
        # (every pair in FP64 arithmetic); results must be identical
        ref32 = ctx.count_3pcf()
        ctx.set_catalog(xyz_d, w_d, cat.n_data)
        ctx.set_precision("f64")
        for _ in range(args.warmup):
            ctx.count_3pcf(counts=False)
        n64 = max(1, min(args.steps, 50))
        ev64 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                for _ in range(n64)]
        for k in range(n64):
            flush.zero_()
            ev64[k][0].record(stream)
            ctx.count_3pcf(counts=False)
            ev64[k][1].record(stream)
        torch.cuda.synchronize()
        ms64 = float(sum(a.elapsed_time(b) for a, b in ev64)) / n64
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
            "value": r["triangles"] / r["total_s"], "unit": "tuples/s", "cores": threads,
            "kind": "port",
            "sample": f"the full {WORKLOAD} catalogue once: kd-tree graph build "
                      f"{r['graph_s']:.2f} s + 3PCF query {r['query_s']:.2f} s "
                      "(C++ OpenMP restatement of the reference algorithm)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def run_batched(args):
    """Batched regions: 2PCF of 4M density-ramped galaxies + 8M randoms over
    5^3 regions with Rmax buffers, all regions in one
    graph-replayed launch, against one launch per region on the same regions."""
    import torch

    from gramsci_b200 import api, catalogs

    cat = catalogs.make("c4_batched", scale=args.scale)
    sp = catalogs.WORKLOADS["c4_batched"]
    w = catalogs.normalise(cat.w, cat.n_data, cat.n_rand)
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream()
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
    loop_ctx = api.Context(0)
    loop_ctx.set_stream(stream)
    loop_ctx.set_precision(args.precision)
    loop_ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])

    def per_region():
        tot = 0
        for x, ww, b, nd in reg_dev:
            loop_ctx.set_catalog(x, ww, nd, buffer=b)
            r = loop_ctx.count_2pcf()
            tot = tot + r["counts"]
        return tot

    def timed(fn, steps):
        ms = []
        for _ in range(steps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            out = fn()
            b.record(stream)
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        return float(np.median(ms)), out

    for _ in range(max(1, args.warmup)):
        ctx.count_2pcf_batched()
    t_batch, out = timed(ctx.count_2pcf_batched, max(1, args.steps))
    st = ctx.stats()
    per_region()
    t_loop, tot = timed(per_region, max(1, min(args.steps, 3)))
    assert np.array_equal(tot, out["counts"]) and np.array_equal(out["counts"], ref["counts"])
    pairs = int(out["counts"].sum()) // 2
    line = {
        "metric": METRIC + " [batched regions]", "value": pairs / (t_batch / 1e3),
        "unit": "pairs/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_batch, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic (seeded ramped Neyman-Scott + uniform randoms)",
        "config": {"workload": f"c4_batched: {cat.n_data} galaxies + {cat.n_rand} randoms, box "
                               f"{cat.meta['box']:.0f}, rmin 10, rmax 60, 12 bins, nmu 10, "
                               f"{len(regions)} regions with 60 Mpc/h buffers",
                   "scale": args.scale, "members": int(sum(sizes)),
                   "region_members_min_max": [int(min(sizes)), int(max(sizes))],
                   "pairs": pairs, "rooted": int(out["counts"].sum())},
        "per_region_ms": t_loop, "per_region_pairs_per_s": pairs / (t_loop / 1e3),
        "batched_over_per_region": t_loop / t_batch,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_adjoint(args):
    """Adjoints: weighted 2PCF and 3PCF forward passes over 1M lognormal-
    weighted galaxies + 2M randoms and their weight
    adjoints (device time of the counting vs the adjoint kernels)."""
    from gramsci_b200 import api, catalogs

    out = {}
    for name, order in (("c5_adjoint_2pcf", 2), ("c5_adjoint_3pcf", 3)):
        cat = catalogs.make(name, scale=args.scale)
        sp = catalogs.WORKLOADS[name]
        w = catalogs.normalise(cat.w, cat.n_data, cat.n_rand)
        ctx = api.Context(0)
        ctx.set_catalog(cat.xyz, w, cat.n_data)
        ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
        rng = np.random.default_rng(5)
        fwd, adj = [], []
        for k in range(max(2, args.steps)):
            r = ctx.count_2pcf() if order == 2 else ctx.count_3pcf()
            s = ctx.stats()
            c2 = rng.normal(size=r["N2"].shape)
            c3 = rng.normal(size=r["N3"].shape)
            g = ctx.adjoint_2pcf(c2, c3) if order == 2 else ctx.adjoint_3pcf(c2, c3)
            a = ctx.stats()
            if k > 0:
                fwd.append(s["ms_query"])
                adj.append(a["ms_query"])
        out[name] = {"n_points": cat.n, "forward_query_ms": float(np.median(fwd)),
                     "adjoint_ms": float(np.median(adj)),
                     "adjoint_over_forward": float(np.median(adj) / np.median(fwd)),
                     "tuples": s["tuples"]}
        ctx.close()
    print(json.dumps({"metric": METRIC + " [weight adjoint]", "scale": args.scale, **out}), flush=True)
    return 0


def run_quad(args):
    """4PCF on the small dense clustered set (30k galaxies + 90k randoms in a
    300 Mpc/h box, unit weights).
    value: rooted 4-clique contributions binned per second of device time
    (index + graph + 4-clique kernel per step); e2e through the public API
    with host inputs; beside it the same catalogue with lognormal weights
    (weighted forward pass and weight adjoint, device time)."""
    import torch

    from gramsci_b200 import api, catalogs, roofline

    name = "c3_4pcf"
    cat = catalogs.make(name, scale=args.scale)
    sp = catalogs.WORKLOADS[name]
    w = catalogs.normalise(cat.w, cat.n_data, cat.n_rand)
    stream = torch.cuda.current_stream()
    ctx = api.Context(0)
    ctx.set_stream(stream)
    ctx.set_precision(args.precision)
    xyz_d = torch.from_numpy(cat.xyz).to("cuda:0")
    w_d = torch.from_numpy(w).to("cuda:0")
    ctx.set_bins(sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"])
    ctx.set_catalog(xyz_d, w_d, cat.n_data)
    # the geometric 4-clique kernel: what the automatic choice takes for
    # unit weights with rows of at most 256 neighbours (this catalogue's
    # longest upper row has 96), set explicitly so that the roofline below
    # names the kernel that ran
    ctx.set_clique_mode("geometric")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda:0")
    sampler = ClockSampler(0)
    sampler.start()
    for _ in range(args.warmup):
        ctx.count_4pcf()
    torch.cuda.synchronize()
    t_region0 = time.monotonic()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    q_ms, rooted, launches, st = [], 0, 0, None
    for k in range(args.steps):
        flush.zero_()
        ev[k][0].record(stream)
        ctx.count_4pcf()
        ev[k][1].record(stream)
        st = ctx.stats()
        q_ms.append(st["ms_query"])
        rooted += st["rooted"]
        launches += st["kernel_launches"]
    torch.cuda.synchronize()
    t_region1 = time.monotonic()
    clocks = sampler.stop(t_region0, t_region1)
    total_ms = float(sum(a.elapsed_time(b) for a, b in ev))
    value = rooted / (total_ms / 1e3)

    xyz_h = torch.from_numpy(cat.xyz).pin_memory()
    w_h = torch.from_numpy(w).pin_memory()
    e2e_ms = []
    for k in range(max(3, min(args.steps, 10)) + 2):  # the first two calls are warm-up
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ctx._check(ctx._lib.gr_set_catalog(ctx._h, xyz_h.data_ptr(), w_h.data_ptr(), None,
                                           cat.n_data, cat.n_rand))
        out = ctx.count_4pcf()
        b.record(stream)
        torch.cuda.synchronize()
        if k >= 2:
            e2e_ms.append(a.elapsed_time(b))
    e2e_value = ctx.stats()["rooted"] / (float(np.mean(e2e_ms)) / 1e3)
    d2h = int(sum(v.nbytes for v in out.values()) + 8 * 8)

    pk = roofline.peaks()
    rf = roofline.quad4_roofline(ctx, q_ms, pk, geometric=True)
    rf["traffic"] = roofline.profiled_traffic("quad4g_kernel", args.scale, "c3")

    # the same catalogue with lognormal weights (automatic kernel choice):
    # weighted sums and adjoint
    ctx.set_clique_mode("auto")
    rng = np.random.default_rng(5)
    wl = catalogs.normalise(rng.lognormal(0.0, 0.3, cat.n), cat.n_data, cat.n_rand)
    ctx.set_catalog(torch.from_numpy(cat.xyz).to("cuda:0"), torch.from_numpy(wl).to("cuda:0"),
                    cat.n_data)
    fwd, adj = [], []
    for k in range(4):
        r = ctx.count_4pcf()
        fwd.append(ctx.stats()["ms_query"])
        cot = [rng.normal(size=r[x].shape) for x in ("N2", "N3", "discN", "discR")]
        ctx.adjoint_4pcf(*cot)
        adj.append(ctx.stats()["ms_query"])
    line = {
        "metric": METRIC + " [4PCF]", "value": value, "unit": "tuples/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded Neyman-Scott galaxies + uniform randoms)",
        "config": {"workload": f"{name}: Neyman-Scott 4PCF, {cat.n_data} galaxies + {cat.n_rand} "
                               f"randoms, box {cat.meta['box']:.0f}, rmin {sp['rmin']}, "
                               f"rmax {sp['rmax']}, nbins {sp['nbins']}, unit weights",
                   "n_points": int(cat.n), "scale": args.scale, "tuples": "rooted 4-clique "
                   "contributions (one per reference root)", "l2": "flushed between steps (256 MB write)",
                   "precision": args.precision, "cliques_per_step": st["tuples"],
                   "rooted_per_step": st["rooted"], "edges": st["n_edges"],
                   "phase_ms": {"index": st["ms_index"], "graph": st["ms_graph"],
                                "query": st["ms_query"]}},
        "e2e": {"value": e2e_value, "unit": "tuples/s",
                "h2d_bytes_per_step": int(cat.xyz.nbytes + w.nbytes), "d2h_bytes_per_step": d2h},
        "roofline": rf,
        "clocks": clocks,
        "gpu_launches": launches,
        "lognormal_weights": {"forward_query_ms": float(np.median(fwd[1:])),
                              "adjoint_ms": float(np.median(adj[1:])),
                              "adjoint_over_forward": float(np.median(adj[1:]) / np.median(fwd[1:]))},
    }
    if not args.no_cpu_baseline:
        from oracle import oracle

        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        G = oracle.Graph(cat.xyz, sp["rmin"], sp["rmax"], sp["nbins"], sp["nmu"], method="kdtree",
                         threads=threads)
        t1 = time.perf_counter()
        r = G.pcf4(w, cat.n_data)
        t2 = time.perf_counter()
        line["cpu_baseline"] = {
            "value": int(r["counts"].sum()) / (t2 - t0), "unit": "tuples/s", "cores": threads,
            "kind": "port",
            "sample": f"the full {name} catalogue once: kd-tree graph build {t1 - t0:.2f} s + "
                      f"4PCF query {t2 - t1:.2f} s (C++ OpenMP restatement of the reference "
                      "algorithm)"}
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "c4_batched":
        return run_batched(args)
    if args.workload == "c5_adjoint":
        return run_adjoint(args)
    if args.workload == "c3_4pcf":
        return run_quad(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
