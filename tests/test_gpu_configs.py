"""Parity at the sizes of the other workloads, on the device, against the oracle.

* C4, the full W-towers configuration (4096^2 grid, sub-grids 512, margin 32,
  winc 20, 8,372,224 visibilities): the FP64 master grid against the CPU
  restatement of grid.c (src/reference/grid.c:295-555), and the N = 4096 dirty
  image (hermitian, shift, FFT, shift; src/reference/main.c:258-294) against
  the oracle's image of the same grid.
* C2, the DFT precision workload (1024^2 at theta 0.05, 200,000
  visibilities): the FP64-reduced and naive-FP32 modes against the FP64 DFT
  oracle on a seeded sample of pixels.
* C3, the learned-kernel W-projection workload (2048^2, |w| <= 2000): the
  tensor-core learned gridder on a 20,000-visibility sample against a CPU
  gridding with the FP64 oracle network.
* W-projection taps that leave the grid across an edge are dropped per axis,
  as the reference GPU gridder does (src/grid/grid_cuda.cu:25-41).
* grid.out -weight against weight() + grid_wprojection + the image pipeline
  (src/reference/main.c:153, :258-294).
"""
import importlib
import os
import subprocess

import numpy as np
import pytest

from conftest import rel_rms

pytestmark = pytest.mark.gpu
TOL = 1e-5


def test_c4_wtowers_full_size(rg, ctx, sim, oracle):
    obs = sim.wtowers_full()
    u, v, w, vis = obs.flat()
    assert len(u) == 8_372_224
    n, th, S, M, winc = 4096, 0.1, 512, 32, 20.0
    wk = sim.generate_wkernel(th, np.arange(-11.0, 11.5, 1.0), 16, 32)
    g = np.zeros((n, n), np.complex128)
    ctx.grid_wtowers(g, n, th, rg.Visibilities(u, v, w, vis), wk, S, M, winc)
    st = ctx.last_stats()
    ref = oracle.grid_wtowers(n, th, u, v, w, vis, wk, S, M, winc)
    assert rel_rms(g, ref) < TOL
    assert st["gridded"] + st["dropped"] == len(u) and st["active_subgrids"] > 3000
    # the dirty image at N = 4096 from the GPU grid, against the oracle's
    # image pipeline on the same grid (FP64 transforms on both sides)
    img = ctx.image_from_grid(g.copy())
    img_ref = oracle.image_from_grid(g.copy())
    assert rel_rms(img, img_ref) < 1e-12


def _pixel_sample(n, count, seed, extra=()):
    rng = np.random.default_rng(seed)
    px = rng.integers(0, n, count)
    py = rng.integers(0, n, count)
    for x, y in extra:
        px = np.append(px, x)
        py = np.append(py, y)
    return px, py


def test_c2_dft_precision_full_size(rg, ctx, sim, oracle):
    """RMS and peak error over 3,000 sampled pixels (plus the image's peak
    pixel), normalised by the oracle's largest value there.  The FP64-reduced
    phase stays within 1e-8 RMS; the naive FP32 phase is an order of magnitude
    worse on the same pixels."""
    obs = sim.dft_study(n_vis=200_000)
    u, v, w, vis = (a[:200_000] for a in obs.flat())
    n, th = 1024, obs.meta["theta"]
    V = rg.Visibilities(u, v, w, vis)
    red = ctx.dft_image(n, th, V, rg.RG_DFT_FP64_REDUCED, 2.0)
    naive = ctx.dft_image(n, th, V, rg.RG_DFT_FP32_NAIVE, 2.0)
    peak = np.unravel_index(np.argmax(np.abs(red)), red.shape)
    px, py = _pixel_sample(n, 3000, 21, extra=[(peak[1], peak[0]), (n // 2, n // 2)])
    ref = oracle.dft_pixels(n, th, u, v, w, vis, px, py, factor=2.0)
    scale = np.abs(ref).max()
    e_red = (red[py, px] - ref) / scale
    e_naive = (naive[py, px] - ref) / scale
    rms_red = float(np.sqrt(np.mean(e_red ** 2)))
    rms_naive = float(np.sqrt(np.mean(e_naive ** 2)))
    assert rms_red < 1e-8, rms_red
    assert np.abs(e_red).max() < 1e-6
    assert rms_naive > 10 * rms_red, (rms_naive, rms_red)


def test_c3_learned_wprojection_sample(rg, ctx, sim):
    """The learned-tap W-projection gridder on the C3 workload's grid
    (2048^2, theta 0.1, |w| <= 2000), first 20,000 visibilities, against CPU
    gridding with the FP64 oracle network at each visibility's exact offsets.
    Tolerance: the tensor-core inference rounds weights to BF16 and
    activations to FP16 (3e-2 relative, as the small-grid test)."""
    MO = importlib.import_module("oracle.mlp_oracle")
    obs = sim.learned_wproj(n_vis=1_000_000)
    u, v, w, vis = (np.ascontiguousarray(a[:20_000]) for a in obs.flat())
    n, th, K = obs.meta["grid_size"], obs.meta["theta"], 16
    mlp = rg.LearnedKernel(ctx, K, 2000.0, 0.05)
    mlp.set_params(MO.pack(MO.init_params(8)).astype(np.float32) * 0.5)
    P = MO.unpack(mlp.get_params().astype(np.float64))
    g = np.zeros((n, n), np.complex128)
    rg.grid_wprojection_learned(ctx, mlp, g, n, th, rg.Visibilities(u, v, w, vis))
    mlp.close()
    ref = np.zeros((n, n), np.complex128)
    tyy, txx = np.meshgrid(np.arange(K), np.arange(K), indexing="ij")
    tx, ty = txx.ravel(), tyy.ravel()
    x, y = th * u, th * v
    cx, cy = np.floor(x), np.floor(y)
    for b0 in range(0, len(u), 2000):
        sl = slice(b0, min(b0 + 2000, len(u)))
        m = sl.stop - sl.start
        f = MO.features(np.repeat(w[sl], K * K), np.repeat(x[sl] - cx[sl], K * K),
                        np.repeat(y[sl] - cy[sl], K * K), np.tile(tx, m), np.tile(ty, m), K, 2000.0)
        yv, _ = MO.forward(P, f)
        tap = ((yv[:, 0] + 1j * yv[:, 1]) * 0.05).reshape(m, K * K)
        col = (cx[sl].astype(np.int64) - K // 2 + n // 2)[:, None] + tx[None, :]
        row = (cy[sl].astype(np.int64) - K // 2 + n // 2)[:, None] + ty[None, :]
        np.add.at(ref, (row.ravel(), col.ravel()), (vis[sl, None] * np.conj(tap)).ravel())
    assert rel_rms(g, ref) < 3e-2


def _edge_expected(oracle, n, th, u, v, w, vis, wk):
    """The reference GPU gridder's rule for taps off the grid: each tap's
    column and row are checked on their own (src/grid/grid_cuda.cu:25-41), with
    grid.c's frac_coord cells and sub-cells (src/reference/grid.c:37-57)."""
    K, ov = wk.size, wk.oversampling
    g = np.zeros((n, n), np.complex128)
    base = (n // 2 - K // 2) * n
    for i in range(len(u)):
        col0 = oracle.frac_coord(n, K, ov, th, u[i], 0.0)[0] - base
        row0 = oracle.frac_coord(n, K, ov, th, v[i], 0.0)[0] - base
        so = oracle.frac_coord(n, K, ov, th, u[i], v[i])[1] // (K * K)
        plane = int(np.floor((w[i] - wk.w_min) / wk.w_step + 0.5))
        taps = wk.data[plane, so // ov, so % ov]
        for ty in range(K):
            for tx in range(K):
                c, r = col0 + tx, row0 + ty
                if 0 <= c < n and 0 <= r < n:
                    g[r, c] += vis[i] * np.conj(taps[ty, tx])
    return g


def test_wprojection_footprint_across_the_edge(rg, ctx, sim, oracle):
    """Visibilities whose 16-tap footprints cross the left, right, top and
    bottom edges of a 256-cell grid: the taps off the grid are dropped on
    each axis (none wraps into the neighbouring row)."""
    n, th = 256, 0.1
    u = np.array([-1252.3, 1294.6, 35.2, -60.4, 301.0, -1249.0, 1291.2])
    v = np.array([41.7, -88.1, -1251.6, 1293.3, -120.9, -1251.2, 1292.8])
    w = np.array([3.0, -7.5, 12.0, -1.0, 0.4, 8.8, -14.2])
    rng = np.random.default_rng(9)
    vis = rng.normal(size=len(u)) + 1j * rng.normal(size=len(u))
    wk = sim.generate_wkernel(th, np.arange(-20.0, 21.0, 5.0), 16, 8)
    expected = _edge_expected(oracle, n, th, u, v, w, vis, wk)
    g = np.zeros((n, n), np.complex128)
    ctx.grid_wprojection(g, n, th, rg.Visibilities(u, v, w, vis), wk)
    assert rel_rms(g, expected) < TOL
    # grid.c itself wraps such taps into the neighbouring row: the two differ
    assert rel_rms(oracle.grid_wprojection(n, th, u, v, w, vis, wk), expected) > 1e-3


def test_grid_out_weight(rg, sim, oracle, tmp_path):
    """grid.out -weight: uniform weighting (weight(), src/reference/grid.c:59-81,
    as main.c:153 calls it) before W-projection gridding and imaging."""
    obs = sim.wproj_plain(seed=8)
    n_bl, n_time = obs.uvw.shape[:2]
    d = tmp_path
    rg.write_vis_hdf5(str(d / "vis.h5"), obs.antenna1, obs.antenna2, np.broadcast_to(obs.time, (n_bl, n_time)),
                      obs.freq, obs.uvw, obs.vis)
    th, n = obs.meta["theta"], obs.meta["grid_size"]
    u, v, w, vis = obs.flat()
    wk = sim.wkernel_for(w, th, 10.0, size=16, oversampling=8)
    rg.write_wkern_hdf5(str(d / "wk.h5"), th, wk)
    wkr = rg.read_wkern_hdf5(str(d / "wk.h5"), th)
    binary = os.path.join(os.path.dirname(__file__), "..", "radio-gridders_b200", "bin", "grid.out")
    r = subprocess.run([binary, f"-vis={d}/vis.h5", f"-wkernel={d}/wk.h5", f"-theta={th}",
                        f"-lambda={obs.meta['lam']}", f"-image={d}/w.img", f"-grid={d}/w.grid", "-wproj", "-weight"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    wvis = oracle.weight(n, th, u, v, vis)
    assert not np.allclose(wvis, vis)  # the weighting does something on this data
    ref = oracle.grid_wprojection(n, th, u, v, w, wvis, wkr)
    grid = np.fromfile(f"{d}/w.grid", np.float64).view(np.complex128).reshape(n, n)
    assert rel_rms(grid, oracle.make_hermitian(ref.copy())) < TOL
    img = np.fromfile(f"{d}/w.img", np.float64).reshape(n, n)
    assert rel_rms(img, oracle.image_from_grid(ref.copy())) < TOL


def test_grid_out_simple(rg, sim, oracle, tmp_path):
    """grid.out -simple: grid_CPU.out's nearest-cell gridder (no w-kernel file,
    src/reference/main.c:200-206) from a visibility file, image as main.c
    forms it."""
    obs = sim.wproj_plain(seed=9, n_dump=16)
    n_bl, n_time = obs.uvw.shape[:2]
    rg.write_vis_hdf5(str(tmp_path / "vis.h5"), obs.antenna1, obs.antenna2, np.broadcast_to(obs.time, (n_bl, n_time)),
                      obs.freq, obs.uvw, obs.vis)
    th, n = obs.meta["theta"], obs.meta["grid_size"]
    u, v, w, vis = obs.flat()
    binary = os.path.join(os.path.dirname(__file__), "..", "radio-gridders_b200", "bin", "grid.out")
    r = subprocess.run([binary, f"-vis={tmp_path}/vis.h5", f"-theta={th}", f"-lambda={obs.meta['lam']}", "-simple",
                        f"-image={tmp_path}/s.img", f"-grid={tmp_path}/s.grid"], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and "Simple imaging" in r.stdout, r.stdout + r.stderr
    ref = oracle.grid_simple(n, th, u, v, vis)
    grid = np.fromfile(f"{tmp_path}/s.grid", np.float64).view(np.complex128).reshape(n, n)
    assert rel_rms(grid, oracle.make_hermitian(ref.copy())) < 1e-14
    img = np.fromfile(f"{tmp_path}/s.img", np.float64).reshape(n, n)
    assert rel_rms(img, oracle.image_from_grid(ref.copy())) < 1e-12
