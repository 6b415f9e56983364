"""Error behaviour: the C ABI returns a status and a message; nothing exits,
nothing faults.  Invalid inputs are rejected on the host or flagged by the
kernels' own range checks."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def vis_arrays(n=100, seed=0, wmax=4.0):
    rng = np.random.default_rng(seed)
    return (rng.uniform(-500, 500, n), rng.uniform(-500, 500, n), rng.uniform(-wmax, wmax, n),
            rng.normal(size=n) + 0j)


@pytest.fixture(scope="module")
def wkt(sim):
    return sim.generate_wkernel(0.1, np.arange(-5, 6, 1.0))


def test_margin_smaller_than_kernel(rg, ctx, wkt):
    g = np.zeros((256, 256), np.complex128)
    with pytest.raises(rg.RGError) as e:
        ctx.grid_wtowers(g, 256, 0.1, rg.Visibilities(*vis_arrays()), wkt, 128, 8, 10.0)
    assert e.value.status == 1 and "margin" in str(e.value)


def test_unsupported_subgrid(rg, ctx, wkt):
    g = np.zeros((256, 256), np.complex128)
    with pytest.raises(rg.RGError) as e:
        ctx.grid_wtowers(g, 256, 0.1, rg.Visibilities(*vis_arrays()), wkt, 96, 16, 10.0)
    assert e.value.status == 4


def test_nonfinite_w(rg, ctx, wkt):
    u, v, w, vis = vis_arrays()
    w[17] = np.nan
    g = np.zeros((256, 256), np.complex128)
    with pytest.raises(rg.RGError) as e:
        ctx.grid_wtowers(g, 256, 0.1, rg.Visibilities(u, v, w, vis), wkt, 128, 16, 10.0)
    assert e.value.status == 1 and "non-finite" in str(e.value)


def test_w_outside_kernel_table(rg, ctx, wkt):
    u, v, w, vis = vis_arrays(wmax=400.0)
    g = np.zeros((256, 256), np.complex128)
    with pytest.raises(rg.RGError) as e:
        ctx.grid_wprojection(g, 256, 0.1, rg.Visibilities(u, v, w, vis), wkt)
    assert e.value.status == 1 and "w-kernel" in str(e.value)


def test_footprint_outside_grid(rg, ctx, wkt):
    u, v, w, vis = vis_arrays()
    u[3] = 1e6
    g = np.zeros((256, 256), np.complex128)
    with pytest.raises(rg.RGError) as e:
        ctx.grid_wprojection(g, 256, 0.1, rg.Visibilities(u, v, w, vis), wkt)
    assert e.value.status == 1


def test_visibilities_outside_every_tower_are_counted(rg, ctx, wkt):
    u, v, w, vis = vis_arrays()
    u[5] = 1e6  # beyond the last tower: the reference grids nothing for it either
    g = np.zeros((256, 256), np.complex128)
    ctx.grid_wtowers(g, 256, 0.1, rg.Visibilities(u, v, w, vis), wkt, 128, 16, 10.0)
    st = ctx.last_stats()
    assert st["dropped"] == 1 and st["gridded"] == len(u) - 1


def test_context_still_usable_after_errors(rg, ctx, wkt, oracle):
    u, v, w, vis = vis_arrays()
    g = np.zeros((256, 256), np.complex128)
    ctx.grid_wtowers(g, 256, 0.1, rg.Visibilities(u, v, w, vis), wkt, 128, 16, 10.0)
    ref = oracle.grid_wtowers(256, 0.1, u, v, w, vis, wkt, 128, 16, 10.0)
    assert np.linalg.norm(g - ref) / np.linalg.norm(ref) < 1e-5


def test_null_and_bad_arguments(rg, ctx, wkt):
    import ctypes as ct
    L = rg.lib()
    assert L.rg_grid_wtowers(ctx.handle, None, 256, 0.1, None, None, 128, 16, 10.0, 0) == 1
    assert L.rg_fft2d(ctx.handle, None, 1, 64, 64, -1, 8) == 1
    assert L.rg_dft_image(ctx.handle, None, 64, 0.1, None, 1, 2.0) == 1
    assert b"NULL" in L.rg_last_error() or len(L.rg_last_error()) > 0
