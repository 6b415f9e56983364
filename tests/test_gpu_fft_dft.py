"""The project's FFT kernels against numpy and cuFFT, and the DFT imager's
precision modes against the FP64 DFT oracle."""
import importlib

import numpy as np
import pytest

from conftest import rel_rms

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [64, 128, 256, 512, 1024])
@pytest.mark.parametrize("sign", [-1, 1])
def test_fft32_vs_numpy_and_cufft(ctx, n, sign):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(n)
    x = (rng.normal(size=(3, n, n)) + 1j * rng.normal(size=(3, n, n))).astype(np.complex64)
    y = x.copy()
    ctx.fft2d(y, sign)
    ref = np.fft.fft2(x.astype(np.complex128)) if sign < 0 else np.fft.ifft2(x.astype(np.complex128)) * n * n
    assert rel_rms(y, ref) < 1e-6
    xt = torch.from_numpy(x).cuda()
    cu = torch.fft.fft2(xt) if sign < 0 else torch.fft.ifft2(xt) * (n * n)
    # our FP32 transform is at least as close to FP64 as cuFFT's
    assert rel_rms(y, ref) < 2.0 * rel_rms(cu.cpu().numpy(), ref) + 1e-7


@pytest.mark.parametrize("n", [2, 64, 1024, 4096])
def test_fft64_vs_numpy(ctx, n):
    rng = np.random.default_rng(n)
    x = rng.normal(size=(1, n, n)) + 1j * rng.normal(size=(1, n, n))
    y = x.copy()
    ctx.fft2d(y, -1)
    assert rel_rms(y, np.fft.fft2(x)) < 1e-13


@pytest.mark.parametrize("ny,nx", [(6, 10), (100, 250), (2500, 2500), (4094, 3)])
@pytest.mark.parametrize("sign", [-1, 1])
def test_fft64_any_length_vs_numpy(ctx, ny, nx, sign):
    """Lengths that are not powers of two (Bluestein's chirp-z over
    power-of-two transforms), both signs."""
    rng = np.random.default_rng(ny * 7 + nx)
    x = rng.normal(size=(1, ny, nx)) + 1j * rng.normal(size=(1, ny, nx))
    y = x.copy()
    ctx.fft2d(y, sign)
    ref = np.fft.fft2(x) if sign < 0 else np.fft.ifft2(x) * (nx * ny)
    assert rel_rms(y, ref) < 1e-12


def test_image_at_a_grid_size_that_is_not_a_power_of_two(rg, ctx, sim, oracle):
    """grid.out's grid size is floor(lambda * theta): theta 0.1, lambda 25000
    gives 2500.  W-projection grid against the oracle, and the dirty image
    (hermitian, shift, FFT sign -1, shift; src/reference/main.c:258-294)
    against the oracle's hermitian and shift with numpy's FFT."""
    obs = sim.wproj_plain(seed=3, lam=25000.0)
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    assert n == 2500
    u, v, w, vis = obs.flat()
    wk = sim.wkernel_for(w, th, 10.0, size=16, oversampling=8)
    g = np.zeros((n, n), np.complex128)
    ctx.grid_wprojection(g, n, th, rg.Visibilities(u, v, w, vis), wk)
    ref = oracle.grid_wprojection(n, th, u, v, w, vis, wk)
    assert rel_rms(g, ref) < 1e-5
    img = ctx.image_from_grid(g.copy())
    h = oracle.fft_shift(oracle.make_hermitian(g.copy()))
    img_ref = oracle.fft_shift(np.fft.fft2(h)).real
    assert rel_rms(img, img_ref) < 1e-12


@pytest.fixture(scope="module")
def dft_case(sim):
    obs = sim.dft_study(n_vis=20_000)
    u, v, w, vis = (a[:20_000] for a in obs.flat())
    return obs.meta, u, v, w, vis


def test_dft_precision_modes(rg, ctx, oracle, dft_case):
    meta, u, v, w, vis = dft_case
    n, th = 256, meta["theta"]
    ref = oracle.dft_image(n, th, u, v, w, vis, 2.0)
    V = rg.Visibilities(u, v, w, vis)
    peak = np.abs(ref).max()
    err = {}
    for mode in (rg.RG_DFT_FP32_NAIVE, rg.RG_DFT_FP64_REDUCED, rg.RG_DFT_FP64):
        img = ctx.dft_image(n, th, V, mode, 2.0)
        err[mode] = np.sqrt(np.mean((img - ref) ** 2)) / peak
    assert err[rg.RG_DFT_FP64] < 1e-12
    assert err[rg.RG_DFT_FP64_REDUCED] < 1e-6
    # the FP64 phase reduction is what buys the accuracy
    assert err[rg.RG_DFT_FP64_REDUCED] < err[rg.RG_DFT_FP32_NAIVE]


def test_dft_single_visibility_fringe(rg, ctx):
    n, th = 64, 0.1
    u, v, w = np.array([37.0]), np.array([-12.0]), np.array([3.0])
    vis = np.array([1.0 + 0.5j])
    img = ctx.dft_image(n, th, rg.Visibilities(u, v, w, vis), rg.RG_DFT_FP64, 2.0)
    lm = th * (np.arange(n) - n // 2) / n
    one_minus_n = 1 - np.sqrt(1 - lm[None, :] ** 2 - lm[:, None] ** 2)
    ph = u[0] * lm[None, :] + v[0] * lm[:, None] + w[0] * one_minus_n
    ref = 2 * (vis[0].real * np.cos(2 * np.pi * ph) + vis[0].imag * np.sin(2 * np.pi * ph))
    assert np.max(np.abs(img - ref)) < 1e-12


def test_dft_row_bands_make_the_image(rg, ctx, sim):
    """rg_dft_image_rows: bands starting on multiples of 32 (the partition of
    sharding.dft_row_ranges) give the whole image's rows bit for bit; a band
    starting elsewhere agrees to the mode's rounding; bad ranges are rejected."""
    sharding = importlib.import_module("radio-gridders_b200.sharding")
    obs = sim.wproj_plain(seed=5, n_dump=8)
    u, v, w, vis = obs.flat()
    n, th = 200, obs.meta["theta"]
    V = rg.Visibilities(u, v, w, vis)
    whole = ctx.dft_image(n, th, V)
    bands = [ctx.dft_image_rows(n, th, V, r0, k) for r0, k in sharding.dft_row_ranges(n, 3)]
    assert np.array_equal(np.concatenate(bands), whole)
    odd = ctx.dft_image_rows(n, th, V, 17, 50)
    assert np.max(np.abs(odd - whole[17:67])) < 1e-6 * np.abs(whole).max()
    for r0, k in ((-1, 4), (190, 20), (0, -2)):
        with pytest.raises(rg.RGError):
            ctx.dft_image_rows(n, th, V, r0, k, image=np.empty((max(k, 1), n)))
