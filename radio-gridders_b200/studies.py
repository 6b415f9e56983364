"""Measurement studies beyond the headline benchmark: the DFT precision study
and the image error of the W-towers gridder against the direct DFT.

Run on a B200:  python radio-gridders_b200/studies.py [dft|towers|learned|all]
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


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "all")
