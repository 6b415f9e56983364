"""Measurement studies beyond the headline benchmark: the DFT precision study
and the image error of the W-towers gridder against the direct DFT.

Run on a B200:  python radio-gridders_b200/studies.py [dft|towers|towers_ov|learned|learned_towers|learned_towers_c4|parity_c1|parity_c4|baselines|all]
Each study prints one JSON object."""
from __future__ import annotations

import importlib
import json
import os
import sys
import time

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

_rg = importlib.import_module("radio-gridders_b200")
_sim = importlib.import_module("radio-gridders_b200.simulate")
_learned = importlib.import_module("radio-gridders_b200.learned")


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
    obs = _sim.dft_study(n_vis=n_vis)
    u, v, w, vis = (a[:n_vis] for a in obs.flat())
    th = obs.meta["theta"]
    dev = torch.device("cuda", 0)
    ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
    T = [torch.from_numpy(x).to(dev) for x in (u, v, w, vis)]
    V = _rg.Visibilities(*T)
    out = {"grid_size": grid_size, "n_vis": len(u), "theta": th}
    imgs = {}
    for name, mode in (("fp64", _rg.RG_DFT_FP64), ("fp64_reduced", _rg.RG_DFT_FP64_REDUCED),
                       ("fp32_naive", _rg.RG_DFT_FP32_NAIVE)):
        img = torch.empty((grid_size, grid_size), dtype=torch.float64, device=dev)
        ms = _events_ms(lambda: ctx.dft_image(grid_size, th, V, mode, 2.0, image=img),
                        repeats=1 if mode == _rg.RG_DFT_FP64 else 3)
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
    obs = _sim.wtowers_plain()
    u, v, w, vis = obs.flat()
    n, th = 2048, 0.1
    V = _rg.Visibilities(u, v, w, vis)
    wk = _sim.generate_wkernel(th, np.arange(-5 - w_step, 5 + 1.5 * w_step, w_step), 16, oversampling)
    g = np.zeros((n, n), np.complex128)
    ctx.set_profiling(True)
    ctx.grid_wtowers(g, n, th, V, wk, 512, 16, 10.0, flags=1)
    ctx.grid_wtowers(g, n, th, V, wk, 512, 16, 10.0, flags=1)
    stages = dict(ctx.last_timings())
    ctx.set_profiling(False)
    img = ctx.image_from_grid(g, taper_1d=_sim.taper_1d(th, n, wk.c))
    t0 = time.time()
    ref = ctx.dft_image(n, th, V, _rg.RG_DFT_FP64_REDUCED, 2.0)
    rms, pk = _learned.image_errors(img, ref)
    return {"workload": "wtowers_plain", "oversampling": oversampling, "w_step": w_step,
            "image_rms_vs_dft": rms, "image_peak_vs_dft": pk, "romein_ms": stages.get("romein"),
            "region": "central half of each axis", "dft_s": time.time() - t0}


def learned_towers(ctx, config="C1", steps=120000, n_triples=16384):
    """Learned-kernel W-towers against the table W-towers on the same
    workload: a network trained on the GPU (own forward/backward kernels) on
    generator kernels over the residual w range |w - w_mid| <= winc/2, then
    both gridders timed (CUDA events around the call, inputs in HBM) and both
    images compared with the FP64-reduced DFT.  C1: 2048^2, S 512, margin 16,
    winc 10, 2.09M vis; C4: 4096^2, S 512, margin 32, winc 20, 8.4M vis."""
    import torch
    if config == "C4":
        obs, n, S, M, winc = _sim.wtowers_full(), 4096, 512, 32, 20.0
    else:
        obs, n, S, M, winc = _sim.wtowers_plain(), 2048, 512, 16, 10.0
    th = 0.1
    half = winc / 2
    u, v, w, vis = obs.flat()
    t0 = time.time()
    mlp, losses = _learned.train(ctx, wmax=half + 1.0, theta=th, ksize=16, n_triples=n_triples, steps=steps,
                                 batch=32768, lr_max=2e-3)
    train_s = time.time() - t0
    err, held = _learned.tap_error(mlp, wmax=half + 1.0, theta=th)
    wk = _sim.generate_wkernel(th, np.arange(-half - 1.0, half + 1.5, 1.0), 16, 32)
    table_err = _learned.table_tap_error(wk, held)
    dev = torch.device("cuda", 0)
    ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
    V = _rg.Visibilities(*(torch.from_numpy(a).to(dev) for a in (u, v, w)), torch.from_numpy(vis).to(dev))
    dwk = torch.from_numpy(np.ascontiguousarray(wk.data)).to(dev)
    g = torch.zeros((n, n), dtype=torch.complex128, device=dev)
    table_ms = _events_ms(lambda: ctx.grid_wtowers(g, n, th, V, wk, S, M, winc, flags=1, wkern_data=dwk))
    img_t = ctx.image_from_grid(g.cpu().numpy(), taper_1d=_sim.taper_1d(th, n, wk.c))
    learned_ms = _events_ms(lambda: _rg.grid_wtowers_learned(ctx, mlp, g, n, th, V, S, M, winc, flags=1),
                            repeats=2)
    img_l = ctx.image_from_grid(g.cpu().numpy(), taper_1d=_sim.taper_1d(th, n, wk.c))
    t1 = time.time()
    ref = ctx.dft_image(n, th, _rg.Visibilities(u, v, w, vis), _rg.RG_DFT_FP64_REDUCED, 2.0)
    dft_s = time.time() - t1
    t_rms, t_pk = _learned.image_errors(img_t, ref)
    l_rms, l_pk = _learned.image_errors(img_l, ref)
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


def parity_full(ctx, config="C4"):
    """Grid parity at full size against the CPU restatement of grid.c (which
    the tests pin bit-identical to the reference's own grid.c): relative RMS of
    the FP64 master grid.  C4: 4096^2, S 512, margin 32, winc 20, 8.37M vis."""
    import oracle
    if config == "C4":
        obs, n, S, M, winc = _sim.wtowers_full(), 4096, 512, 32, 20.0
    else:
        obs, n, S, M, winc = _sim.wtowers_plain(), 2048, 512, 16, 10.0
    th, half = 0.1, winc / 2
    u, v, w, vis = obs.flat()
    wk = _sim.generate_wkernel(th, np.arange(-half - 1.0, half + 1.5, 1.0), 16, 32)
    g = np.zeros((n, n), np.complex128)
    ctx.grid_wtowers(g, n, th, _rg.Visibilities(u, v, w, vis), wk, S, M, winc)
    st = ctx.last_stats()
    t0 = time.time()
    ref = oracle.grid_wtowers(n, th, u, v, w, vis, wk, S, M, winc)
    d = g - ref
    return {"config": config, "n_vis": len(u), "grid_size": n, "active_subgrids": st["active_subgrids"],
            "rel_rms": float(np.sqrt(np.mean(np.abs(d) ** 2) / np.mean(np.abs(ref) ** 2))),
            "oracle_s": time.time() - t0}


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
        return _rg.Visibilities(*(torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (u, v, w)),
                                torch.from_numpy(np.ascontiguousarray(vis)).to(dev))

    out = {"host_cores": cores}
    # C0: plain W-projection, 512^2, 22,464 vis
    obs = _sim.wproj_plain()
    u, v, w, vis = obs.flat()
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    wk = _sim.wkernel_for(w, th, 10.0, size=16, oversampling=8)
    g = torch.zeros((n, n), dtype=torch.complex128, device=dev)
    dwk = torch.from_numpy(np.ascontiguousarray(wk.data)).to(dev)
    V = dV(u, v, w, vis)
    ms = _events_ms(lambda: ctx.grid_wprojection(g, n, th, V, wk, flags=1, wkern_data=dwk), repeats=5)
    t0 = time.time()
    oracle.ref_grid_wprojection(n, th, obs, wk)
    cpu_s = time.time() - t0
    img = ctx.image_from_grid(g.cpu().numpy(), taper_1d=_sim.taper_1d(th, n, wk.c))
    ref = ctx.dft_image(n, th, _rg.Visibilities(u, v, w, vis), _rg.RG_DFT_FP64_REDUCED, 2.0)
    rms, pk = _learned.image_errors(img, ref)
    out["C0"] = {"n_vis": len(u), "gpu_ms": ms, "gpu_vis_per_s": len(u) / (ms * 1e-3), "cpu_s": cpu_s,
                 "cpu_vis_per_s": len(u) / cpu_s, "cpu_cores": 1, "image_rms": rms, "image_peak": pk}
    # C2: direct DFT, 1024^2 at theta 0.05, 200k vis; CPU on a 2,000-visibility sample
    obs = _sim.dft_study(n_vis=200_000)
    u, v, w, vis = (a[:200_000] for a in obs.flat())
    th, n = obs.meta["theta"], 1024
    img = torch.zeros((n, n), dtype=torch.float64, device=dev)
    V = dV(u, v, w, vis)
    ms = _events_ms(lambda: ctx.dft_image(n, th, V, _rg.RG_DFT_FP64_REDUCED, 2.0, image=img), repeats=2)
    k = 2000
    t0 = time.time()
    oracle.dft_image(n, th, u[:k], v[:k], w[:k], vis[:k])
    cpu_s = time.time() - t0
    out["C2"] = {"n_vis": len(u), "grid_size": n, "gpu_ms": ms, "gpu_pairs_per_s": n * n * len(u) / (ms * 1e-3),
                 "cpu_sample_vis": k, "cpu_s": cpu_s, "cpu_pairs_per_s": n * n * k / cpu_s, "cpu_cores": cores}
    # C3: table W-projection on the learned-kernel workload (2048^2, 1M vis); CPU on a 100k sample
    obs = _sim.learned_wproj(n_vis=1_000_000)
    u, v, w, vis = (a[:1_000_000] for a in obs.flat())
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    wk = _sim.generate_wkernel(th, np.arange(-2010.0, 2011.0, 10.0), 16, 8)
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
    obs = _sim.wtowers_full()
    u, v, w, vis = obs.flat()
    n, th, S, M, winc = 4096, 0.1, 512, 32, 20.0
    wk = _sim.generate_wkernel(th, np.arange(-11.0, 11.5, 1.0), 16, 32)
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
    obs = _sim.wtowers_plain(n_st=stations)
    u, v, w, vis = obs.flat()
    mlp, _ = _learned.train(ctx, wmax=6.0, theta=0.1, ksize=16, n_triples=512, steps=steps, batch=16384,
                            lr_max=4e-3)
    dev = torch.device("cuda", 0)
    ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
    V = _rg.Visibilities(*(torch.from_numpy(a).to(dev) for a in (u, v, w)), torch.from_numpy(vis).to(dev))
    g = torch.zeros((2048, 2048), dtype=torch.complex128, device=dev)
    call = lambda: _rg.grid_wtowers_learned(ctx, mlp, g, 2048, 0.1, V, 512, 16, 10.0, flags=1)
    ms = _events_ms(call, repeats=3)
    ctx.set_profiling(True)
    call()
    stage = dict(ctx.last_timings())["learned_gridding"]
    ctx.set_profiling(False)
    ctx.set_stream(None)
    return {"n_vis": len(u), "learned_ms": ms, "learned_vis_per_s": len(u) / (ms * 1e-3),
            "gridding_stage_ms": stage, "gridding_stage_vis_per_s": len(u) / (stage * 1e-3)}


def main(which):
    ctx = _rg.Context(0)
    if which in ("dft", "all"):
        print(json.dumps({"study": "dft_precision", **dft_precision(ctx)}), flush=True)
    if which in ("towers", "all"):
        print(json.dumps({"study": "towers_image_error", **towers_image_error(ctx)}), flush=True)
    if which == "towers_ov":
        for ov, ws in ((8, 1.0), (16, 1.0), (32, 1.0), (16, 0.5), (64, 1.0)):
            print(json.dumps({"study": "towers_image_error", **towers_image_error(ctx, ov, ws)}), flush=True)
    if which in ("learned", "all"):
        mlp, losses = _learned.train(ctx, steps=40000, batch=16384, lr_max=4e-3)
        err, held = _learned.tap_error(mlp)
        wk = _sim.generate_wkernel(0.1, np.arange(-2010.0, 2011.0, 10.0), 16, 8)
        r = _learned.study_wproj(ctx, mlp, n_vis=1_000_000, repeats=2)
        print(json.dumps({"study": "learned_wproj", "tap_err": err,
                          "table_tap_err": _learned.table_tap_error(wk, held),
                          "final_loss": losses[-1], **r}), flush=True)


    if which == "learned_small":
        print(json.dumps({"study": "learned_small", **learned_small(ctx)}), flush=True)
    if which == "baselines":
        print(json.dumps({"study": "baselines", **baselines(ctx)}), flush=True)
    if which in ("parity_c1", "parity_c4"):
        print(json.dumps({"study": "parity_full", **parity_full(ctx, which[-2:].upper())}), flush=True)
    if which in ("learned_towers", "learned_towers_c4"):
        cfg = "C4" if which.endswith("c4") else "C1"
        print(json.dumps({"study": "learned_towers", **learned_towers(ctx, cfg)}), flush=True)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "all")
