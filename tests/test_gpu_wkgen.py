"""The w-kernel generator behind the C ABI (rg_wkern_generate) against the
Python generator the workloads use (simulate.generate_wkernel): the same
tables to FP64 rounding, for the benchmark's 16-tap 32x-oversampled planes and
a wide-w 8-tap table."""
import numpy as np
import pytest

from conftest import rel_rms

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("planes,size,ov", [(np.arange(-5.0, 6.0, 1.0), 16, 32),
                                            (np.arange(-2000.0, 2001.0, 500.0), 8, 4),
                                            (np.array([0.0, 37.5]), 16, 8)])
def test_generator_matches_python(ctx, sim, planes, size, ov):
    got = ctx.wkern_generate(0.1, planes, size, ov)
    ref = sim.generate_wkernel(0.1, planes, size, ov).data
    assert got.shape == ref.shape
    assert rel_rms(got, ref) < 1e-12
    # each plane on its own (the large-w planes have the smallest taps)
    for p in range(len(planes)):
        assert rel_rms(got[p], ref[p]) < 1e-12


def test_generated_table_grids_like_the_python_one(rg, ctx, sim, oracle):
    """A W-projection grid made with the generated table equals the oracle's
    with the Python table."""
    obs = sim.wproj_plain()
    u, v, w, vis = obs.flat()
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    ref_wk = sim.wkernel_for(w, th, 10.0, size=16, oversampling=8)
    planes = ref_wk.w_min + ref_wk.w_step * np.arange(ref_wk.plane_count)
    data = ctx.wkern_generate(th, planes, 16, 8)
    from types import SimpleNamespace
    wk = SimpleNamespace(data=data, w_min=ref_wk.w_min, w_step=ref_wk.w_step, plane_count=ref_wk.plane_count,
                         size=16, oversampling=8)
    g = np.zeros((n, n), np.complex128)
    ctx.grid_wprojection(g, n, th, rg.Visibilities(u, v, w, vis), wk)
    assert rel_rms(g, oracle.grid_wprojection(n, th, u, v, w, vis, ref_wk)) < 1e-5


def test_generator_rejects_bad_arguments(rg, ctx):
    with pytest.raises(rg.RGError):
        ctx.wkern_generate(0.1, np.array([0.0]), 7, 8)
    with pytest.raises(rg.RGError):
        ctx.wkern_generate(0.1, np.array([np.nan]), 16, 8)
    with pytest.raises(rg.RGError):
        ctx.wkern_generate(-0.1, np.array([0.0]), 16, 8)
