"""Training recipe and evaluation helpers for the learned w-kernel.

The network is trained on the GPU by the library's own kernels
(rg_mlp_train); this module builds the training set from the project's
w-kernel generator (simulate.learned_training_set) and runs a learning-rate
schedule.  Nothing here runs on the CPU beyond data generation."""
from __future__ import annotations

import importlib
import math

import numpy as np

_rg = importlib.import_module("radio-gridders_b200")
_sim = importlib.import_module("radio-gridders_b200.simulate")


def train(ctx, wmax=2000.0, theta=0.1, ksize=16, n_triples=8192, steps=20000, batch=16384,
          lr_max=2e-3, lr_min=1e-5, seed=0, out_scale=0.05, chunks=20, data=None):
    """Train a network on n_triples * ksize^2 generator taps (2M for the
    defaults).  Cosine learning-rate decay from lr_max to lr_min over `steps`,
    applied in `chunks` constant pieces.  Returns (network, losses)."""
    if data is None:
        data = _sim.learned_training_set(n_triples, wmax, theta, ksize, seed=seed)
    w, du, dv, tx, ty, tap = data
    # shuffle taps so every batch spans many (w, du, dv)
    perm = np.random.default_rng(seed + 1).permutation(len(w))
    S = _rg.LearnedKernel.samples(w[perm], du[perm], dv[perm], tx[perm], ty[perm])
    T = _rg.LearnedKernel.targets(tap[perm])
    mlp = _rg.LearnedKernel(ctx, ksize, wmax, out_scale, seed=seed)
    losses = []
    per = max(1, steps // chunks)
    done = 0
    while done < steps:
        k = min(per, steps - done)
        mid = done + k / 2
        lr = lr_min + 0.5 * (lr_max - lr_min) * (1 + math.cos(math.pi * mid / steps))
        losses.append(mlp.train(S, T, batch=batch, steps=k, lr=lr))
        done += k
    return mlp, losses


def tap_error(mlp, wmax=2000.0, theta=0.1, ksize=16, n_triples=256, seed=99):
    """Relative RMS error of the network's taps against the generator at
    random continuous (w, du, dv)."""
    w, du, dv, tx, ty, tap = _sim.learned_training_set(n_triples, wmax, theta, ksize, seed=seed)
    pred = mlp.eval(_rg.LearnedKernel.samples(w, du, dv, tx, ty))
    return float(np.linalg.norm(pred - tap) / np.linalg.norm(tap)), (w, du, dv, tx, ty, tap)


def table_tap_error(wk, held_out):
    """Relative RMS error of nearest-plane, nearest-sub-cell lookup in an
    oversampled table (the reference's w_project, src/reference/grid.c:37-57
    and :157-185) at the same continuous points."""
    w, du, dv, tx, ty, tap = held_out
    ov = wk.oversampling
    plane = np.floor((w - wk.w_min) / wk.w_step + 0.5).astype(int)
    ok = (plane >= 0) & (plane < wk.plane_count)
    # frac_coord: cell = floor(x + 1/(2 ov)), sub-cell = floor((x - cell) ov + 1/2)
    sx = (du + 0.5 / ov >= 1).astype(int)
    sy = (dv + 0.5 / ov >= 1).astype(int)
    xf = np.floor((du - sx) * ov + 0.5).astype(int)
    yf = np.floor((dv - sy) * ov + 0.5).astype(int)
    txi = tx.astype(int) - sx
    tyi = ty.astype(int) - sy
    ok &= (txi >= 0) & (tyi >= 0)
    tab = np.zeros_like(tap)
    tab[ok] = wk.data[plane[ok], yf[ok], xf[ok], tyi[ok], txi[ok]]
    return float(np.linalg.norm((tab - tap)[ok]) / np.linalg.norm(tap[ok]))


def image_errors(img, ref, region=0.5):
    """RMS and peak of (image - reference) over the central `region` fraction
    of each axis, normalised by the reference's peak there."""
    n = img.shape[0]
    a = int(n * (1 - region) / 2)
    b = n - a
    d = img[a:b, a:b] - ref[a:b, a:b]
    peak = np.abs(ref[a:b, a:b]).max()
    return float(np.sqrt(np.mean(d * d)) / peak), float(np.abs(d).max() / peak)


def study_wproj(ctx, mlp, n_vis=1_000_000, repeats=3):
    """Learned vs table W-projection on the learned-kernel workload (2048^2,
    theta 0.1, n_vis visibilities, |w| <= 2000): gridding time (CUDA events on
    the context stream, via the library's stage timers) and image RMS / peak
    error against the FP64-reduced DFT over the central half of the field."""
    import time

    obs = _sim.learned_wproj(n_vis=n_vis)
    u, v, w, vis = (a[:n_vis] for a in obs.flat())
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    V = _rg.Visibilities(u, v, w, vis)
    wk = _sim.generate_wkernel(th, np.arange(-2010.0, 2011.0, 10.0), 16, 8)
    taper = _sim.taper_1d(th, n, wk.c)
    ctx.set_profiling(True)
    out = {"n_vis": len(u), "grid_size": n}

    def timed(fn):
        best = None
        for _ in range(repeats):
            fn()
            t = dict(ctx.last_timings())
            k = t.get("romein", t.get("learned_gridding"))
            best = k if best is None else min(best, k)
        return best

    g_tab = np.zeros((n, n), np.complex128)
    out["table_grid_ms"] = timed(lambda: ctx.grid_wprojection(g_tab, n, th, V, wk, flags=1))
    g_lrn = np.zeros((n, n), np.complex128)
    out["learned_grid_ms"] = timed(lambda: grid_wprojection_learned_ctx(ctx, mlp, g_lrn, n, th, V))
    ctx.set_profiling(False)
    t0 = time.time()
    ref = ctx.dft_image(n, th, V, _rg.RG_DFT_FP64_REDUCED, 2.0)
    out["dft_s"] = time.time() - t0
    img_tab = ctx.image_from_grid(g_tab.copy(), taper_1d=taper)
    img_lrn = ctx.image_from_grid(g_lrn.copy(), taper_1d=taper)
    out["table_rms"], out["table_peak"] = image_errors(img_tab, ref)
    out["learned_rms"], out["learned_peak"] = image_errors(img_lrn, ref)
    out["table_vis_per_s"] = len(u) / (out["table_grid_ms"] * 1e-3)
    out["learned_vis_per_s"] = len(u) / (out["learned_grid_ms"] * 1e-3)
    return out


def grid_wprojection_learned_ctx(ctx, mlp, grid, n, theta, V, flags=1):
    return _rg.grid_wprojection_learned(ctx, mlp, grid, n, theta, V, flags)
