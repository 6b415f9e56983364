#!/usr/bin/env python
"""W-towers gridding throughput on B200 (visibilities per second).

One step = one rg_grid_wtowers call over one observation resident in HBM:
w-range reduction, per-visibility tower/floor binning, coordinates and
column-strip marks, Romein gridding of every active (tower, w-floor)
sub-grid, backward column transforms of the marked strips, the fused
row-transform / Fresnel-step / w=0-transfer stage with the forward row
transform, forward column transforms and the FP64 add-back into the master
grid — the
loop of the reference's grid_wtowers (src/reference/grid.c:295-555) and
wtowers_CUDA_flat (src/grid/grid_cuda.cu:522-744) up to the final FFT.

Workload (N = 1): the W-towers configuration — 2048 x 2048 grid (theta 0.1,
lambda 20480), 512-cell sub-grids with 16-cell margins, w-increment 10,
SKA-Low-like 256 stations (32,640 baselines x 16 dumps x 4 channels =
2,088,960 visibilities), 16 x 16 taps at 32x oversampling (11 w-planes,
|dw| <= 5), which keeps the image within 1e-4 RMS of the FP64 DFT.  Synthetic, seeded.
With --gpus N the towers of the one observation are split over the ranks
(rg_wtowers_tower_loads + rg_wtowers_partition: balanced by visibilities and
active w-floors), each rank grids its share into its own FP64 master grid
(rg_grid_wtowers_part) and one NCCL reduce sums the master grids onto rank 0:
total work fixed (strong scaling).

``--impl reference`` times the reference's own CPU grid_wtowers
(src/reference/grid.c, compiled from its sources into oracle/_ref with its
makefile flags and -DOMP_TOWERS) on the host cores, same workload.
"""
from __future__ import annotations

import argparse
import importlib
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "W-towers vis/s on 1 B200 at <=1e-4 RMS vs FP64 DFT; learned vs table kernel"
GRID, THETA, LAM, SUBGRID, MARGIN, WINC = 2048, 0.1, 20480.0, 512, 16, 10.0
KSIZE, OVER = 16, 32
FALLBACK_HBM_GBS = 6650.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-image-check", action="store_true")
    p.add_argument("--no-learned", action="store_true",
                   help="skip the learned-kernel W-towers measurement (training takes ~40 s)")
    p.add_argument("--no-autotune", action="store_true",
                   help="keep the default schedule (Romein 8 points per thread, 8 row-stage items per SM: the "
                        "tuner's usual choice here) instead of timing candidates; for profiled runs, whose "
                        "serialised launches would skew the tuner")
    p.add_argument("--study", choices=STUDIES, default=None,
                   help="run one of the studies beside the headline line instead (one JSON object each)")
    p.add_argument("--stations", type=int, default=256,
                   help="array size of the workload (256: the benchmark; fewer: a smaller case for profiling)")
    return p.parse_args()


def workload(stations: int = 256):
    """The observation every rank grids a share of (seeded)."""
    sim = importlib.import_module("radio-gridders_b200.simulate")
    obs = sim.wtowers_plain(seed=1, n_st=stations)
    wk = sim.generate_wkernel(THETA, np.arange(-5, 6, 1.0), KSIZE, OVER)
    return obs, wk


def peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for n, val in zip(names, parts[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


STAGES = ("prepare", "romein", "fft_cols_backward", "tower_rows", "tower_finish", "fft_cols_forward",
          "add_back")


def stage_bytes(stage, stats, nvis):
    """Algorithmic HBM bytes of one launch of each stage (for the roofline).
    Sub-grids are touched only in their marked column strips (8 columns x S
    rows x 8 B each): gridding writes them once, the column transform reads
    and writes them, the row stage reads and clears them."""
    s2 = SUBGRID * SUBGRID
    strip = 8 * 8 * SUBGRID * stats["marked_strips"]
    nt, ng = stats["towers_with_data"], stats["floor_groups"]
    ntow = (GRID // (SUBGRID - MARGIN) + 1) ** 2
    return {
        "prepare": 40 * nvis + 24 * nvis,                   # f64 uvw + c128 in, record + c64 out
        "romein": 24 * nvis + strip,                        # records + vis in, marked strips out
        "fft_cols_backward": 2 * strip,                     # marked strips in place
        "tower_rows": 2 * strip + 8 * s2 * ng,              # strips in + cleared, partials out
        "tower_finish": 8 * s2 * ng + 8 * s2 * nt,          # partials in, sub-images out
        "fft_cols_forward": 16 * s2 * ntow,                 # every tower sub-image in place
        "add_back": 8 * s2 * nt + 16 * GRID * GRID,         # read sub-images, write master
    }.get(stage)


def algorithmic_bytes(stats, nvis):
    """Bytes per step of the sparse dataflow: the sum over its stages."""
    return sum(stage_bytes(k, stats, nvis) for k in STAGES)


def dense_dataflow_bytes(stats, nvis):
    """Bytes per step of the dense dataflow the reference's pipeline implies
    (every active sub-grid zeroed, gridded, row- and column-transformed in
    full, one HBM pass per stage): 20 B per visibility, 48 S^2 per active
    sub-grid, 24 S^2 per tower with data, 32 N^2 for the master grid."""
    s2 = SUBGRID * SUBGRID
    return (20 * nvis + 48 * s2 * stats["active_subgrids"] + 24 * s2 * stats["towers_with_data"]
            + 32 * GRID * GRID)


def cpu_baseline(obs, wk, reps=1):
    """The reference's own grid_wtowers (OMP_TOWERS build) on the host cores;
    falls back to the single-threaded C restatement if the reference build is
    absent.  Baselines whose footprint would fall before the reference's
    sub-grid buffer are left out (grid.c:177-182 has no bounds check)."""
    import oracle
    cores = len(os.sched_getaffinity(0))
    mask = oracle.reference_safe_baselines(obs, GRID, THETA, SUBGRID, MARGIN, KSIZE, OVER)
    sub = oracle.subset_baselines(obs, mask)
    if oracle.reference_available(omp=True):
        times = []
        for _ in range(reps):
            t = time.perf_counter()
            oracle.ref_grid_wtowers(GRID, THETA, sub, wk, SUBGRID, MARGIN, WINC, omp=True)
            times.append(time.perf_counter() - t)
        dt = min(times)
        return {"value": sub.nvis / dt, "unit": "vis/s", "cores": cores, "kind": "reference",
                "sample": (f"full workload less {int((~mask).sum())} of {len(mask)} baselines "
                           f"whose footprints would leave the reference's sub-grid buffer; "
                           f"{sub.nvis} vis, {dt:.2f} s, best of {reps}"),
                "seconds": dt}
    u, v, w, vis = sub.flat()
    t = time.perf_counter()
    oracle.grid_wtowers(GRID, THETA, u, v, w, vis, wk, SUBGRID, MARGIN, WINC)
    dt = time.perf_counter() - t
    return {"value": sub.nvis / dt, "unit": "vis/s", "cores": 1, "kind": "port",
            "sample": f"full workload, {sub.nvis} vis, C restatement single-threaded, {dt:.2f} s",
            "seconds": dt}


def workload_config(nvis, stations):
    """The workload both arms time (identical in their lines)."""
    return {"workload": "wtowers_plain: 2048x2048 grid (theta 0.1, lambda 20480), subgrid 512, "
                        f"margin 16, winc 10, {nvis:,} vis ({stations} stations, 16 dumps x 4 ch), "
                        "16x16 taps x32 oversampled, 11 w-planes",
            "grid_size": GRID, "theta": THETA, "subgrid": SUBGRID, "margin": MARGIN, "winc": WINC,
            "vis_per_step": nvis}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    import oracle
    obs, wk = workload()
    cores = len(os.sched_getaffinity(0))
    if not oracle.reference_available(omp=True):
        kind = "port"
    else:
        kind = "reference"
    res = None
    times = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(obs, wk)
        if i >= args.warmup:
            times.append(r["seconds"])
        res = r
    per = statistics.mean(times) if times else res["seconds"]
    nvis = int(round(res["value"] * res["seconds"]))
    value = nvis / per
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "vis/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": per * 1e3, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": workload_config(len(obs.flat()[0]), 256),
            "run": {"parallelism": f"{cores} host threads (OpenMP over towers)" if kind == "reference"
                    else "1 host thread"},
            "cpu_baseline": {"value": value, "unit": "vis/s", "cores": res["cores"] if kind == "reference" else 1,
                             "kind": kind, "sample": res["sample"]},
            "e2e": {"value": value, "unit": "vis/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def learned_towers(args, ctx, V, grid, stream, flush, nvis, table_ms, wk, ref):
    """The metric's other half: the same workload gridded by the learned-kernel
    W-towers gridder (rg_grid_wtowers_learned).  The network is trained on the
    GPU by the library's own kernels (120,000 Adam steps of 32,768 taps drawn
    from 16,384 x 256 generator taps over |w - w_mid| <= winc/2 + 1, about
    40 s), then timed like the table path (warm-up, K steps
    with L2 flushed between them, CUDA events), and its image compared with the
    same FP64 DFT."""
    import torch
    rg = importlib.import_module("radio-gridders_b200")
    learned = importlib.import_module("radio-gridders_b200.learned")
    sim = importlib.import_module("radio-gridders_b200.simulate")
    half = WINC / 2
    t0 = time.time()
    mlp, losses = learned.train(ctx, wmax=half + 1.0, theta=THETA, ksize=KSIZE, n_triples=16384, steps=120000,
                                batch=32768, lr_max=2e-3)
    train_s = time.time() - t0
    tap_err, _ = learned.tap_error(mlp, wmax=half + 1.0, theta=THETA)

    def lstep():
        rg.grid_wtowers_learned(ctx, mlp, grid, GRID, THETA, V, SUBGRID, MARGIN, WINC, flags=rg.RG_GRID_OVERWRITE)

    for _ in range(max(args.warmup, 3)):
        lstep()
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        flush.fill_(1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        lstep()
        b.record(stream)
        b.synchronize()
        times.append(a.elapsed_time(b))
    ms = sum(times) / len(times)
    out = {"value": nvis / (ms * 1e-3), "unit": "vis/s", "ms_per_step": ms,
           "over_table": table_ms / ms, "target_over_table": 1.5,
           "network": "21 Fourier features -> 3 x 128 SiLU -> complex tap; FP16 tcgen05 inference",
           "train_steps": 120000, "train_triples": 16384, "train_s": train_s, "final_loss": losses[-1], "tap_error": tap_err}
    if ref is not None:
        img = ctx.image_from_grid(grid.cpu().numpy(), taper_1d=sim.taper_1d(THETA, GRID, wk.c))
        rms, pk = learned.image_errors(img, ref)
        out["image_error_vs_dft"] = {"rms": rms, "peak": pk}
    return out


def run_b200(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    rg = importlib.import_module("radio-gridders_b200")
    sharding = importlib.import_module("radio-gridders_b200.sharding")
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    obs, wk = workload(args.stations)
    u, v, w, vis = obs.flat()
    nvis = len(u)

    ctx = rg.Context(local_rank)
    stream = torch.cuda.current_stream(dev)
    ctx.set_stream(stream.cuda_stream)
    if args.no_autotune:
        ctx.set_autotune(False)

    # inputs resident in HBM
    du = torch.from_numpy(u).to(dev)
    dv = torch.from_numpy(v).to(dev)
    dw = torch.from_numpy(w).to(dev)
    dvis = torch.from_numpy(vis).to(dev)
    dwk = torch.from_numpy(np.ascontiguousarray(wk.data)).to(dev)
    grid = torch.zeros((GRID, GRID), dtype=torch.complex128, device=dev)
    V = rg.Visibilities(du, dv, dw, dvis)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    parts = None
    if world > 1:  # this rank's towers (planning, outside the timed steps)
        nv, nf = ctx.tower_loads(GRID, THETA, V, SUBGRID, MARGIN, WINC)
        parts = sharding.tower_parts(nv, nf, world)

    def step():
        if parts is None:
            ctx.grid_wtowers(grid, GRID, THETA, V, wk, SUBGRID, MARGIN, WINC,
                             flags=rg.RG_GRID_OVERWRITE, wkern_data=dwk)
        else:
            ctx.grid_wtowers_part(grid, GRID, THETA, V, wk, SUBGRID, MARGIN, WINC, parts, rank,
                                  flags=rg.RG_GRID_OVERWRITE, wkern_data=dwk)
        sharding.reduce_grid(grid, world)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    stats = ctx.last_stats()  # the first call sized the plan and tuned the schedule; later ones replay a graph

    # timed region (no per-stage events inside it)
    clocks = Clocks(local_rank)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms, stage_ms, launches = [], {}, 0
    for _ in range(args.steps):
        flush.fill_(1)  # evict L2 between steps (outside the step's events)
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        step()
        s1.record(stream)
        s1.synchronize()
        step_ms.append(s0.elapsed_time(s1))
        launches += ctx.last_stats()["launches"]
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()

    # per-stage breakdown: the same steps again with CUDA events around each stage
    ctx.set_profiling(True)
    for _ in range(args.steps):
        flush.fill_(1)
        step()
        torch.cuda.synchronize()
        for name, ms in ctx.last_timings():
            stage_ms.setdefault(name, []).append(ms)
    ctx.set_profiling(False)

    total = torch.tensor([sum(step_ms)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(total, op=dist.ReduceOp.MAX)
    ms_per_step = total.item() / args.steps
    value = nvis / (ms_per_step * 1e-3)  # one observation per step, over all ranks

    # end to end through the C ABI with pinned host buffers
    hu = torch.from_numpy(u).pin_memory()
    hv = torch.from_numpy(v).pin_memory()
    hw = torch.from_numpy(w).pin_memory()
    hvis = torch.from_numpy(vis).pin_memory()
    hwk = torch.from_numpy(np.ascontiguousarray(wk.data)).pin_memory().numpy()
    hgrid_t = torch.zeros((GRID, GRID), dtype=torch.complex128).pin_memory()
    hgrid = hgrid_t.numpy()
    if world == 1:
        HV = rg.Visibilities(hu.numpy(), hv.numpy(), hw.numpy(), hvis.numpy())
        for _ in range(2):
            ctx.grid_wtowers(hgrid, GRID, THETA, HV, wk, SUBGRID, MARGIN, WINC,
                             flags=rg.RG_GRID_OVERWRITE, wkern_data=hwk)
        torch.cuda.synchronize()
        # (a) one call per step
        e2e_single = []
        for _ in range(args.steps):
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            ctx.grid_wtowers(hgrid, GRID, THETA, HV, wk, SUBGRID, MARGIN, WINC,
                             flags=rg.RG_GRID_OVERWRITE, wkern_data=hwk)
            t1.record(stream)
            t1.synchronize()
            e2e_single.append(t0.elapsed_time(t1))
        # (b) the steps as one batch call: each step's inputs copied in and grid
        # copied out, overlapping the neighbouring steps' passes
        hgrids = [hgrid] * args.steps
        HVs = [HV] * args.steps
        ctx.grid_wtowers_batch(hgrids[:2], GRID, THETA, HVs[:2], wk, SUBGRID, MARGIN, WINC,
                               flags=rg.RG_GRID_OVERWRITE, wkern_data=hwk)
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        ctx.grid_wtowers_batch(hgrids, GRID, THETA, HVs, wk, SUBGRID, MARGIN, WINC,
                               flags=rg.RG_GRID_OVERWRITE, wkern_data=hwk)
        t1.record(stream)
        t1.synchronize()
        e2e_ms = [t0.elapsed_time(t1) / args.steps]
        e2e_call = f"rg_grid_wtowers_batch over {args.steps} steps (pinned host buffers)"
        h2d = 8 * 3 * nvis + 16 * nvis + 16 * wk.data.size / args.steps
    else:
        # per step: every rank copies the observation in from pinned host
        # memory, grids its towers, the master grids are reduced onto rank 0,
        # which copies the grid out
        def e2e_step():
            for dst, src in ((du, hu), (dv, hv), (dw, hw), (dvis, hvis)):
                dst.copy_(src, non_blocking=True)
            step()
            if rank == 0:
                hgrid_t.copy_(grid, non_blocking=True)

        for _ in range(2):
            e2e_step()
        torch.cuda.synchronize()
        dist.barrier()
        e2e_ms = []
        for _ in range(args.steps):
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            e2e_step()
            t1.record(stream)
            t1.synchronize()
            e2e_ms.append(t0.elapsed_time(t1))
        e2e_single = e2e_ms
        e2e_call = "per step: H2D of the observation on every rank, rg_grid_wtowers_part, NCCL reduce, D2H on rank 0"
        h2d = world * (8 * 3 * nvis + 16 * nvis)
    e2e_t = torch.tensor([sum(e2e_ms) / len(e2e_ms)], dtype=torch.float64, device=dev)
    single_t = torch.tensor([sum(e2e_single) / len(e2e_single)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
        dist.all_reduce(single_t, op=dist.ReduceOp.MAX)
    e2e_value = nvis / (e2e_t.item() * 1e-3)
    d2h = 16 * GRID * GRID

    if rank != 0:
        return 0
    # roofline of the dominant stage (HBM-bound)
    peak, peak_kind = peaks()
    kernel_stages = {k: statistics.mean(v) for k, v in stage_ms.items()
                     if k not in ("stage_in", "stage_out", "w_range", "compact")}
    dom = max(kernel_stages, key=kernel_stages.get)
    dom_ms = kernel_stages[dom]
    dom_bytes = stage_bytes(dom, stats, nvis)
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    # DRAM traffic of the dominant kernel: not measured in this run (a run
    # under ncu gives no bench number); the per-launch figure of the committed
    # one-pass ncu capture of this workload, labelled as such
    traffic, traffic_src = None, None
    tpath = os.path.join(REPO, "profiles", "wtowers_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tdoc = json.load(f)
        entry = tdoc.get(dom)
        traffic = entry["dram_bytes"] if isinstance(entry, dict) else entry  # None for a kernel not captured
        traffic_src = ("profiles/wtowers_traffic.json: ncu dram__bytes_read.sum + dram__bytes_write.sum per launch "
                       "on the 128-station case, scaled to this workload by the kernel's algorithmic bytes; "
                       "captured separately (not this run)") if entry else None
    path_bytes = algorithmic_bytes(stats, nvis)
    # the bytes no implementation avoids: 20 B per visibility in (f32 u, v, w
    # and complex64) and the FP64 master grid out
    compulsory = 20 * nvis + 16 * GRID * GRID
    dense_bytes = dense_dataflow_bytes(stats, nvis)
    # The row stage is bound by instruction issue, not HBM: its FP32 work
    # against the FP32 pipe (the 5 N log2 N convention per transform, as the
    # reference's complexity analysis counts FFTs, plus 8 flops per Fresnel
    # multiply-add), for context beside the HBM roofline.
    rows_ms = kernel_stages.get("tower_rows")
    compute_roofline = None
    if rows_ms:
        s2 = SUBGRID * SUBGRID
        flops = stats["active_subgrids"] * (SUBGRID * 5 * SUBGRID * math.log2(SUBGRID) + 8 * s2)
        fp32_peak = 148 * 128 * 2 * 1.965e9 / 1e12
        compute_roofline = {"kernel": "tower_rows", "flops_per_launch": flops,
                            "achieved": flops / (rows_ms * 1e-3) / 1e12, "peak": fp32_peak, "unit": "TFLOP/s",
                            "frac": flops / (rows_ms * 1e-3) / 1e12 / fp32_peak,
                            "peak_source": "nominal FP32 (148 SMs x 128 lanes x 2 x 1.965 GHz); "
                                           "no measured FP32 peak on this pool"}
    # The heavy kernels are bound by instruction issue: their warp instructions
    # per launch (one-kernel ncu captures of the 128-station case, scaled to
    # this workload by each kernel's work unit; not measured in this run) over
    # the launch time, against 4 issues per SM per clock at the clock sampled
    # during the timed steps.
    issue_roofline = None
    ipath = os.path.join(REPO, "profiles", "wtowers_instructions.json")
    if os.path.exists(ipath) and args.stations == 256:
        with open(ipath) as f:
            idoc = json.load(f)
        sm_hz = ((clk or {}).get("sm_mhz") or 1965.0) * 1e6
        issue_peak = 148 * 4 * sm_hz / 1e12
        issue_roofline = {"unit": "T warp instructions/s", "peak": issue_peak,
                          "peak_source": "148 SMs x 4 schedulers x one issue per clock at the sampled SM clock",
                          "instructions_source": "profiles/wtowers_instructions.json (ncu smsp__inst_executed.sum, "
                                                 "128-station case scaled by work units; not this run)",
                          "kernels": {}}
        for k in ("tower_rows", "romein", "fft_cols_backward", "prepare"):
            if k in idoc and k in kernel_stages:
                rate = idoc[k]["warp_instructions"] / (kernel_stages[k] * 1e-3) / 1e12
                issue_roofline["kernels"][k] = {"achieved": rate, "frac": rate / issue_peak,
                                                "warp_instructions_per_launch": idoc[k]["warp_instructions"],
                                                "launch_ms": kernel_stages[k]}
    line = {
        "impl": "b200", "metric": METRIC, "value": value, "unit": "vis/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Earth-rotation synthesis, power-law point sources)",
        "config": workload_config(nvis, args.stations),
        "run": {"parallelism": (f"{world} ranks, the observation's towers split by load, FP64 master grids "
                                "reduced over NCCL") if world > 1 else "1 GPU",
                "vis_per_gpu": nvis, "active_subgrids": stats["active_subgrids"],
                "towers_with_data": stats["towers_with_data"], "floors": stats["floors"],
                "l2": "256 MiB buffer written between steps, outside each step's event pair",
                "precision": "FP32 sub-grids and transforms; FP64 coordinates, Fresnel phase and master grid",
                "schedule": {"romein_points_per_thread": stats["romein_points"],
                             "row_stage_items_per_sm": stats["group_items_per_sm"],
                             "graph_replay": bool(stats["graph"]), "autotuned": not args.no_autotune},
                "marked_strips": stats["marked_strips"], "floor_groups": stats["floor_groups"]},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": dom_bytes, "launch_ms": dom_ms,
                     "traffic": traffic, "traffic_source": traffic_src},
        "path_roofline": {"algorithmic_bytes_per_step": path_bytes,
                          "achieved_gbs": path_bytes / (ms_per_step * 1e-3) / 1e9,
                          "frac": path_bytes / (ms_per_step * 1e-3) / 1e9 / peak,
                          "compulsory_bytes_per_step": compulsory,
                          "compulsory_gbs": compulsory / (ms_per_step * 1e-3) / 1e9,
                          "compulsory_frac": compulsory / (ms_per_step * 1e-3) / 1e9 / peak,
                          "dense_dataflow_bytes_per_step": dense_bytes,
                          "dense_equivalent_gbs": dense_bytes / (ms_per_step * 1e-3) / 1e9,
                          "dense_equivalent_frac": dense_bytes / (ms_per_step * 1e-3) / 1e9 / peak},
        "compute_roofline": compute_roofline,
        "issue_roofline": issue_roofline,
        "step_ms_min_median_max": [round(min(step_ms), 4), round(statistics.median(step_ms), 4),
                                   round(max(step_ms), 4)],
        "stage_ms": {k: round(statistics.mean(v), 4) for k, v in stage_ms.items()},
        "e2e": {"value": e2e_value, "unit": "vis/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_t.item(),
                "call": e2e_call,
                "single_call_ms_per_step": single_t.item(),
                "single_call_vis_per_s": nvis / (single_t.item() * 1e-3)},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    ref = None
    if rank == 0 and not args.no_image_check:
        # the metric's accuracy condition: image of this step's grid against the
        # FP64-reduced direct DFT (computed once, outside the timed region)
        sim = importlib.import_module("radio-gridders_b200.simulate")
        learned = importlib.import_module("radio-gridders_b200.learned")
        g_host = grid.cpu().numpy()
        if world == 1:
            img = ctx.image_from_grid(g_host, taper_1d=sim.taper_1d(THETA, GRID, wk.c))
            ref = ctx.dft_image(GRID, THETA, V, rg.RG_DFT_FP64_REDUCED, 2.0)
            rms, pk = learned.image_errors(img, ref)
            line["image_error_vs_dft"] = {"rms": rms, "peak": pk, "region": "central half of each axis",
                                          "normalisation": "DFT image peak"}
    if rank == 0 and world == 1 and not args.no_learned:
        line["learned"] = learned_towers(args, ctx, V, grid, stream, flush, nvis, ms_per_step, wk, ref)
    if world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(obs, wk, reps=2)
        cb.pop("seconds", None)
        line["cpu_baseline"] = cb
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# Studies beside the headline line (python bench.py --study NAME, one JSON
# object each): the DFT precision study, the table W-towers image error over
# oversampling, the learned kernel against the table (W-projection C3,
# W-towers C1 and C4), the other workloads against the reference's CPU code
# (baselines: C0, C2, C3, C4, the CPU side being the cpu_baseline leg of each)
# and a short learned run for profiling.
# ---------------------------------------------------------------------------
def _RG():
    return importlib.import_module("radio-gridders_b200")


def _SIM():
    return importlib.import_module("radio-gridders_b200.simulate")


def _LEARNED():
    return importlib.import_module("radio-gridders_b200.learned")


def _events_ms(fn, repeats=3):
    import torch
    best = None
    for _ in range(repeats):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        fn()
        b.record()
        b.synchronize()
        t = a.elapsed_time(b)
        best = t if best is None else min(best, t)
    return best


def dft_precision(ctx, n_vis=200_000, grid_size=1024):
    """Direct-DFT precision study: 1024^2 image at theta 0.05, 200,000
    visibilities (|u|,|v| <= 10,240 lambda, |w| <= 2,000 lambda).  RMS and peak
    error of the FP32 modes against the all-FP64 mode (itself checked against
    the CPU FP64 oracle in the tests), and throughput in pixel-visibility
    pairs per second."""
    import torch
    obs = _SIM().dft_study(n_vis=n_vis)
    u, v, w, vis = (a[:n_vis] for a in obs.flat())
    th = obs.meta["theta"]
    dev = torch.device("cuda", 0)
    ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
    T = [torch.from_numpy(x).to(dev) for x in (u, v, w, vis)]
    V = _RG().Visibilities(*T)
    out = {"grid_size": grid_size, "n_vis": len(u), "theta": th}
    imgs = {}
    for name, mode in (("fp64", _RG().RG_DFT_FP64), ("fp64_reduced", _RG().RG_DFT_FP64_REDUCED),
                       ("fp32_naive", _RG().RG_DFT_FP32_NAIVE)):
        img = torch.empty((grid_size, grid_size), dtype=torch.float64, device=dev)
        ms = _events_ms(lambda: ctx.dft_image(grid_size, th, V, mode, 2.0, image=img),
                        repeats=1 if mode == _RG().RG_DFT_FP64 else 3)
        imgs[name] = img.cpu().numpy()
        out[name + "_ms"] = ms
        out[name + "_pairs_per_s"] = grid_size * grid_size * len(u) / (ms * 1e-3)
    ref = imgs["fp64"]
    peak = np.abs(ref).max()
    for name in ("fp64_reduced", "fp32_naive"):
        d = imgs[name] - ref
        out[name + "_rms"] = float(np.sqrt(np.mean(d * d)) / peak)
        out[name + "_peak"] = float(np.abs(d).max() / peak)
    ctx.set_stream(None)
    return out


def towers_image_error(ctx, oversampling=8, w_step=1.0):
    """Image error of the table W-towers gridder on the benchmark workload
    (2048^2, S 512, margin 16, winc 10, 2.09M visibilities): grid, image
    (hermitian, shift, FFT, shift), grid correction by the PSWF taper, against
    the FP64-reduced direct DFT, over the central half of the field."""
    obs = _SIM().wtowers_plain()
    u, v, w, vis = obs.flat()
    n, th = 2048, 0.1
    V = _RG().Visibilities(u, v, w, vis)
    wk = _SIM().generate_wkernel(th, np.arange(-5 - w_step, 5 + 1.5 * w_step, w_step), 16, oversampling)
    g = np.zeros((n, n), np.complex128)
    ctx.set_profiling(True)
    ctx.grid_wtowers(g, n, th, V, wk, 512, 16, 10.0, flags=1)
    ctx.grid_wtowers(g, n, th, V, wk, 512, 16, 10.0, flags=1)
    stages = dict(ctx.last_timings())
    ctx.set_profiling(False)
    img = ctx.image_from_grid(g, taper_1d=_SIM().taper_1d(th, n, wk.c))
    t0 = time.time()
    ref = ctx.dft_image(n, th, V, _RG().RG_DFT_FP64_REDUCED, 2.0)
    rms, pk = _LEARNED().image_errors(img, ref)
    return {"workload": "wtowers_plain", "oversampling": oversampling, "w_step": w_step,
            "image_rms_vs_dft": rms, "image_peak_vs_dft": pk, "romein_ms": stages.get("romein"),
            "region": "central half of each axis", "dft_s": time.time() - t0}


def study_learned_towers(ctx, config="C1", steps=120000, n_triples=16384):
    """Learned-kernel W-towers against the table W-towers on the same
    workload: a network trained on the GPU (own forward/backward kernels) on
    generator kernels over the residual w range |w - w_mid| <= winc/2, then
    both gridders timed (CUDA events around the call, inputs in HBM) and both
    images compared with the FP64-reduced DFT.  C1: 2048^2, S 512, margin 16,
    winc 10, 2.09M vis; C4: 4096^2, S 512, margin 32, winc 20, 8.4M vis."""
    import torch
    if config == "C4":
        obs, n, S, M, winc = _SIM().wtowers_full(), 4096, 512, 32, 20.0
    else:
        obs, n, S, M, winc = _SIM().wtowers_plain(), 2048, 512, 16, 10.0
    th = 0.1
    half = winc / 2
    u, v, w, vis = obs.flat()
    t0 = time.time()
    mlp, losses = _LEARNED().train(ctx, wmax=half + 1.0, theta=th, ksize=16, n_triples=n_triples, steps=steps,
                                 batch=32768, lr_max=2e-3)
    train_s = time.time() - t0
    err, held = _LEARNED().tap_error(mlp, wmax=half + 1.0, theta=th)
    wk = _SIM().generate_wkernel(th, np.arange(-half - 1.0, half + 1.5, 1.0), 16, 32)
    table_err = _LEARNED().table_tap_error(wk, held)
    dev = torch.device("cuda", 0)
    ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
    V = _RG().Visibilities(*(torch.from_numpy(a).to(dev) for a in (u, v, w)), torch.from_numpy(vis).to(dev))
    dwk = torch.from_numpy(np.ascontiguousarray(wk.data)).to(dev)
    g = torch.zeros((n, n), dtype=torch.complex128, device=dev)
    table_ms = _events_ms(lambda: ctx.grid_wtowers(g, n, th, V, wk, S, M, winc, flags=1, wkern_data=dwk))
    img_t = ctx.image_from_grid(g.cpu().numpy(), taper_1d=_SIM().taper_1d(th, n, wk.c))
    learned_ms = _events_ms(lambda: _RG().grid_wtowers_learned(ctx, mlp, g, n, th, V, S, M, winc, flags=1),
                            repeats=2)
    img_l = ctx.image_from_grid(g.cpu().numpy(), taper_1d=_SIM().taper_1d(th, n, wk.c))
    t1 = time.time()
    ref = ctx.dft_image(n, th, _RG().Visibilities(u, v, w, vis), _RG().RG_DFT_FP64_REDUCED, 2.0)
    dft_s = time.time() - t1
    t_rms, t_pk = _LEARNED().image_errors(img_t, ref)
    l_rms, l_pk = _LEARNED().image_errors(img_l, ref)
    ctx.set_stream(None)
    return {"config": config, "n_vis": len(u), "grid_size": n, "subgrid": S, "margin": M, "winc": winc,
            "train_s": train_s, "train_steps": steps, "final_loss": losses[-1],
            "tap_err": err, "table_tap_err_ov32": table_err,
            "table_ms": table_ms, "table_vis_per_s": len(u) / (table_ms * 1e-3),
            "learned_ms": learned_ms, "learned_vis_per_s": len(u) / (learned_ms * 1e-3),
            "learned_over_table_speed": table_ms / learned_ms,
            "table_image_rms": t_rms, "table_image_peak": t_pk,
            "learned_image_rms": l_rms, "learned_image_peak": l_pk, "dft_s": dft_s,
            "region": "central half of each axis"}


def baselines(ctx):
    """GPU against the reference's CPU code on the configurations C0, C2, C3,
    C4 (C1 is bench.py's line).  GPU: CUDA events around whole calls, inputs
    in HBM.  CPU: the reference's grid.c built from its sources (IEEE build,
    one core, for W-projection; OpenMP build on all cores for W-towers, on the
    baselines it can grid safely) and the OpenMP FP64 DFT oracle, each on a
    bounded sample scaled to the metric's unit."""
    import os
    import torch
    import oracle
    cores = len(os.sched_getaffinity(0))
    dev = torch.device("cuda", 0)
    ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)

    def dV(u, v, w, vis):
        return _RG().Visibilities(*(torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (u, v, w)),
                                torch.from_numpy(np.ascontiguousarray(vis)).to(dev))

    out = {"host_cores": cores}
    # C0: plain W-projection, 512^2, 22,464 vis
    obs = _SIM().wproj_plain()
    u, v, w, vis = obs.flat()
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    wk = _SIM().wkernel_for(w, th, 10.0, size=16, oversampling=8)
    g = torch.zeros((n, n), dtype=torch.complex128, device=dev)
    dwk = torch.from_numpy(np.ascontiguousarray(wk.data)).to(dev)
    V = dV(u, v, w, vis)
    ms = _events_ms(lambda: ctx.grid_wprojection(g, n, th, V, wk, flags=1, wkern_data=dwk), repeats=5)
    t0 = time.time()
    oracle.ref_grid_wprojection(n, th, obs, wk)
    cpu_s = time.time() - t0
    img = ctx.image_from_grid(g.cpu().numpy(), taper_1d=_SIM().taper_1d(th, n, wk.c))
    ref = ctx.dft_image(n, th, _RG().Visibilities(u, v, w, vis), _RG().RG_DFT_FP64_REDUCED, 2.0)
    rms, pk = _LEARNED().image_errors(img, ref)
    out["C0"] = {"n_vis": len(u), "gpu_ms": ms, "gpu_vis_per_s": len(u) / (ms * 1e-3), "cpu_s": cpu_s,
                 "cpu_vis_per_s": len(u) / cpu_s, "cpu_cores": 1, "image_rms": rms, "image_peak": pk}
    # C2: direct DFT, 1024^2 at theta 0.05, 200k vis; CPU on a 2,000-visibility sample
    obs = _SIM().dft_study(n_vis=200_000)
    u, v, w, vis = (a[:200_000] for a in obs.flat())
    th, n = obs.meta["theta"], 1024
    img = torch.zeros((n, n), dtype=torch.float64, device=dev)
    V = dV(u, v, w, vis)
    ms = _events_ms(lambda: ctx.dft_image(n, th, V, _RG().RG_DFT_FP64_REDUCED, 2.0, image=img), repeats=2)
    k = 2000
    t0 = time.time()
    oracle.dft_image(n, th, u[:k], v[:k], w[:k], vis[:k])
    cpu_s = time.time() - t0
    out["C2"] = {"n_vis": len(u), "grid_size": n, "gpu_ms": ms, "gpu_pairs_per_s": n * n * len(u) / (ms * 1e-3),
                 "cpu_sample_vis": k, "cpu_s": cpu_s, "cpu_pairs_per_s": n * n * k / cpu_s, "cpu_cores": cores}
    # C3: table W-projection on the learned-kernel workload (2048^2, 1M vis); CPU on a 100k sample
    obs = _SIM().learned_wproj(n_vis=1_000_000)
    u, v, w, vis = (a[:1_000_000] for a in obs.flat())
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    wk = _SIM().generate_wkernel(th, np.arange(-2010.0, 2011.0, 10.0), 16, 8)
    g = torch.zeros((n, n), dtype=torch.complex128, device=dev)
    dwk = torch.from_numpy(np.ascontiguousarray(wk.data)).to(dev)
    V = dV(u, v, w, vis)
    ms = _events_ms(lambda: ctx.grid_wprojection(g, n, th, V, wk, flags=1, wkern_data=dwk), repeats=3)
    k = 100_000
    t0 = time.time()
    oracle.grid_wprojection(n, th, u[:k], v[:k], w[:k], vis[:k], wk)
    cpu_s = time.time() - t0
    out["C3_table"] = {"n_vis": len(u), "gpu_ms": ms, "gpu_vis_per_s": len(u) / (ms * 1e-3),
                       "cpu_sample_vis": k, "cpu_s": cpu_s, "cpu_vis_per_s": k / cpu_s, "cpu_cores": 1,
                       "cpu_kind": "restatement of grid.c (bit-identical to it)"}
    # C4: table W-towers, 4096^2, S 512, margin 32, winc 20, 8.37M vis
    obs = _SIM().wtowers_full()
    u, v, w, vis = obs.flat()
    n, th, S, M, winc = 4096, 0.1, 512, 32, 20.0
    wk = _SIM().generate_wkernel(th, np.arange(-11.0, 11.5, 1.0), 16, 32)
    g = torch.zeros((n, n), dtype=torch.complex128, device=dev)
    dwk = torch.from_numpy(np.ascontiguousarray(wk.data)).to(dev)
    V = dV(u, v, w, vis)
    ms = _events_ms(lambda: ctx.grid_wtowers(g, n, th, V, wk, S, M, winc, flags=1, wkern_data=dwk))
    mask = oracle.reference_safe_baselines(obs, n, th, S, M, 16, 32)
    sub = oracle.subset_baselines(obs, mask)
    t0 = time.time()
    oracle.ref_grid_wtowers(n, th, sub, wk, S, M, winc, omp=True)
    cpu_s = time.time() - t0
    out["C4_table"] = {"n_vis": len(u), "gpu_ms": ms, "gpu_vis_per_s": len(u) / (ms * 1e-3),
                       "cpu_vis": sub.nvis, "cpu_s": cpu_s, "cpu_vis_per_s": sub.nvis / cpu_s, "cpu_cores": cores,
                       "cpu_kind": "reference grid.c, -DOMP_TOWERS, its makefile flags"}
    ctx.set_stream(None)
    return out


def learned_small(ctx, stations=64, steps=2000):
    """A short learned W-towers run (a briefly trained network, 2048^2, S 512,
    margin 16, winc 10, `stations` stations, inputs and grid in HBM) for
    profiling the learned gridding kernel: the whole call and its gridding
    stage (CUDA events of the library's stage timers)."""
    import torch
    obs = _SIM().wtowers_plain(n_st=stations)
    u, v, w, vis = obs.flat()
    mlp, _ = _LEARNED().train(ctx, wmax=6.0, theta=0.1, ksize=16, n_triples=512, steps=steps, batch=16384,
                            lr_max=4e-3)
    dev = torch.device("cuda", 0)
    ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
    V = _RG().Visibilities(*(torch.from_numpy(a).to(dev) for a in (u, v, w)), torch.from_numpy(vis).to(dev))
    g = torch.zeros((2048, 2048), dtype=torch.complex128, device=dev)
    call = lambda: _RG().grid_wtowers_learned(ctx, mlp, g, 2048, 0.1, V, 512, 16, 10.0, flags=1)
    ms = _events_ms(call, repeats=3)
    ctx.set_profiling(True)
    call()
    stage = dict(ctx.last_timings())["learned_gridding"]
    ctx.set_profiling(False)
    ctx.set_stream(None)
    return {"n_vis": len(u), "learned_ms": ms, "learned_vis_per_s": len(u) / (ms * 1e-3),
            "gridding_stage_ms": stage, "gridding_stage_vis_per_s": len(u) / (stage * 1e-3)}



def winc_sweep(ctx, wincs=(10.0, 20.0, 40.0, 80.0), steps=120000):
    """The learned kernel's algorithmic route: the same C1 observation
    (2048^2, S 512, margin 16, 2.09M vis) gridded by the table and the learned
    W-towers paths at several w increments.  A larger winc means fewer
    w-floors, hence fewer sub-grid transforms, but taps over a wider
    |w - w_mid| <= winc/2: the table needs one plane per lambda of w (32x
    oversampled 16-tap slices, 4.2 MB each stored twice), the network is
    retrained on the wider range.  Each path: CUDA events around the whole
    call (graph replay, L2 flushed between calls), image RMS / peak against the
    FP64-reduced DFT."""
    import torch
    obs = _SIM().wtowers_plain()
    u, v, w, vis = obs.flat()
    n, th, S, M = 2048, 0.1, 512, 16
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    ctx.set_stream(stream.cuda_stream)
    V = _RG().Visibilities(*(torch.from_numpy(a).to(dev) for a in (u, v, w)), torch.from_numpy(vis).to(dev))
    g = torch.zeros((n, n), dtype=torch.complex128, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    ref = ctx.dft_image(n, th, _RG().Visibilities(u, v, w, vis), _RG().RG_DFT_FP64_REDUCED, 2.0)

    def timed(fn, reps=5):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        out = []
        for _ in range(reps):
            flush.fill_(1)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            out.append(a.elapsed_time(b))
        return sorted(out)[len(out) // 2]

    rows = []
    for winc in wincs:
        half = winc / 2
        wk = _SIM().generate_wkernel(th, np.arange(-half - 1.0, half + 1.5, 1.0), 16, 32)
        dwk = torch.from_numpy(np.ascontiguousarray(wk.data)).to(dev)
        t_ms = timed(lambda: ctx.grid_wtowers(g, n, th, V, wk, S, M, winc, flags=1, wkern_data=dwk))
        st = ctx.last_stats()
        img_t = ctx.image_from_grid(g.cpu().numpy(), taper_1d=_SIM().taper_1d(th, n, wk.c))
        t_rms, t_pk = _LEARNED().image_errors(img_t, ref)
        del dwk
        t0 = time.time()
        mlp, losses = _LEARNED().train(ctx, wmax=half + 1.0, theta=th, ksize=16, n_triples=16384, steps=steps,
                                       batch=32768, lr_max=2e-3)
        train_s = time.time() - t0
        tap_err, _ = _LEARNED().tap_error(mlp, wmax=half + 1.0, theta=th)
        l_ms = timed(lambda: _RG().grid_wtowers_learned(ctx, mlp, g, n, th, V, S, M, winc, flags=1), reps=3)
        img_l = ctx.image_from_grid(g.cpu().numpy(), taper_1d=_SIM().taper_1d(th, n, wk.c))
        l_rms, l_pk = _LEARNED().image_errors(img_l, ref)
        mlp.close()
        rows.append({"winc": winc, "floors": st["floors"], "active_subgrids": st["active_subgrids"],
                     "table_planes": wk.plane_count, "table_mb_dup": 2 * wk.data.size * 8 / 1e6,
                     "table_ms": t_ms, "table_vis_per_s": len(u) / (t_ms * 1e-3),
                     "table_image_rms": t_rms, "table_image_peak": t_pk,
                     "learned_ms": l_ms, "learned_vis_per_s": len(u) / (l_ms * 1e-3),
                     "learned_image_rms": l_rms, "learned_image_peak": l_pk, "learned_tap_err": tap_err,
                     "train_s": train_s})
        print(json.dumps({"study": "winc_sweep_row", **rows[-1]}), flush=True)
    ok_t = [r for r in rows if r["table_image_rms"] <= 1e-4]
    ok_l = [r for r in rows if r["learned_image_rms"] <= 1e-4]
    best_t = min(ok_t, key=lambda r: r["table_ms"]) if ok_t else None
    best_l = min(ok_l, key=lambda r: r["learned_ms"]) if ok_l else None
    ctx.set_stream(None)
    return {"rows": rows, "best_table_winc": best_t and best_t["winc"], "best_learned_winc": best_l and best_l["winc"],
            "learned_over_table_at_best": (best_t["table_ms"] / best_l["learned_ms"]) if best_t and best_l else None}


STUDIES = ("dft", "towers", "towers_ov", "learned", "learned_small", "baselines", "learned_towers",
           "learned_towers_c4", "winc_sweep", "pcie")


def host_link(reps=10):
    """The host link's bound on the end-to-end figure: pinned copies of one
    benchmark step's bytes (its inputs in, 40 B per visibility, and its FP64
    master grid out) host to device, device to host, and both at once on two
    streams, timed with CUDA events."""
    import torch
    dev = torch.device("cuda", 0)
    n_in, n_out = (40 * 2_088_960) // 8, (16 * GRID * GRID) // 8
    hin = torch.empty(n_in, dtype=torch.float64).pin_memory()
    hout = torch.empty(n_out, dtype=torch.float64).pin_memory()
    din = torch.empty(n_in, dtype=torch.float64, device=dev)
    dout = torch.empty(n_out, dtype=torch.float64, device=dev)
    s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

    def h2d():
        din.copy_(hin, non_blocking=True)

    def d2h():
        hout.copy_(dout, non_blocking=True)

    def both():
        cur = torch.cuda.current_stream(dev)
        s_in.wait_stream(cur)
        s_out.wait_stream(cur)
        with torch.cuda.stream(s_in):
            din.copy_(hin, non_blocking=True)
        with torch.cuda.stream(s_out):
            hout.copy_(dout, non_blocking=True)
        cur.wait_stream(s_in)
        cur.wait_stream(s_out)

    out = {"in_bytes": n_in * 8, "out_bytes": n_out * 8}
    for name, fn in (("h2d", h2d), ("d2h", d2h), ("both", both)):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        b.synchronize()
        out[name + "_ms"] = a.elapsed_time(b) / reps
    out["h2d_gbs"] = out["in_bytes"] / out["h2d_ms"] / 1e6
    out["d2h_gbs"] = out["out_bytes"] / out["d2h_ms"] / 1e6
    out["e2e_bound_vis_per_s"] = 2_088_960 / (out["both_ms"] * 1e-3)
    return out


def run_study(which):
    if which == "pcie":
        print(json.dumps({"study": "host_link", **host_link()}), flush=True)
        return 0
    ctx = _RG().Context(0)
    if which == "dft":
        print(json.dumps({"study": "dft_precision", **dft_precision(ctx)}), flush=True)
    elif which == "towers":
        print(json.dumps({"study": "towers_image_error", **towers_image_error(ctx)}), flush=True)
    elif which == "towers_ov":
        for ov, ws in ((8, 1.0), (16, 1.0), (32, 1.0), (16, 0.5), (64, 1.0)):
            print(json.dumps({"study": "towers_image_error", **towers_image_error(ctx, ov, ws)}), flush=True)
    elif which == "learned":
        mlp, losses = _LEARNED().train(ctx, steps=40000, batch=16384, lr_max=4e-3)
        err, held = _LEARNED().tap_error(mlp)
        wk = _SIM().generate_wkernel(0.1, np.arange(-2010.0, 2011.0, 10.0), 16, 8)
        r = _LEARNED().study_wproj(ctx, mlp, n_vis=1_000_000, repeats=2)
        print(json.dumps({"study": "learned_wproj", "tap_err": err,
                          "table_tap_err": _LEARNED().table_tap_error(wk, held),
                          "final_loss": losses[-1], **r}), flush=True)
    elif which == "learned_small":
        print(json.dumps({"study": "learned_small", **learned_small(ctx)}), flush=True)
    elif which == "baselines":
        print(json.dumps({"study": "baselines", **baselines(ctx)}), flush=True)
    elif which == "winc_sweep":
        print(json.dumps({"study": "winc_sweep", **winc_sweep(ctx)}), flush=True)
    elif which in ("learned_towers", "learned_towers_c4"):
        cfg = "C4" if which.endswith("c4") else "C1"
        print(json.dumps({"study": "learned_towers", **study_learned_towers(ctx, cfg)}), flush=True)
    ctx.close()
    return 0


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.study:
        return run_study(args.study)
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        return run_b200(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
