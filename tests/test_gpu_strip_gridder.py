"""The W-towers strip gridder (per-strip visibility lists, gridding in shared
memory fused with the backward column transform) against the oracle and
against Romein's gridder, chosen with rg_context_set_wtowers_gridder.

Bar: relative RMS of the uv grid <= 1e-5 against the FP64 CPU restatement of
grid.c; the two GPU gridders differ only in FP32 summation order."""
import numpy as np
import pytest

from conftest import rel_rms

pytestmark = pytest.mark.gpu
TOL = 1e-5
torch = pytest.importorskip("torch")


def V(rg, u, v, w, vis):
    return rg.Visibilities(u, v, w, vis)


@pytest.fixture(scope="module")
def wproj_data(sim):
    obs = sim.wproj_plain()
    u, v, w, vis = obs.flat()
    return obs, u, v, w, vis


def _ctx(rg, gridder):
    ctx = rg.Context(0)
    ctx.set_wtowers_gridder(gridder)
    return ctx


@pytest.mark.parametrize("sub,margin,winc,ksize,ov", [(256, 32, 20.0, 16, 16), (512, 16, 10.0, 16, 16),
                                                       (256, 16, 10.0, 8, 8), (512, 32, 5.0, 8, 4)])
def test_strip_gridder_vs_oracle(rg, sim, oracle, wproj_data, sub, margin, winc, ksize, ov):
    obs, u, v, w, vis = wproj_data
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    wkt = sim.generate_wkernel(th, np.arange(-winc / 2 - 1, winc / 2 + 1.5, 1.0), ksize, ov)
    ctx = _ctx(rg, rg.RG_WTOWERS_GRIDDER_STRIP)
    ref = oracle.grid_wtowers(n, th, u, v, w, vis, wkt, sub, margin, winc)
    g = np.zeros((n, n), np.complex128)
    for _ in range(2):  # sizing + tuning pass, then a pass of the tuned plan
        ctx.grid_wtowers(g, n, th, V(rg, u, v, w, vis), wkt, sub, margin, winc, flags=rg.RG_GRID_OVERWRITE)
        assert rel_rms(g, ref) < TOL
        assert ctx.last_stats()["strip_gridder"] == 1


def test_strip_and_romein_agree_at_full_size(rg, sim, oracle):
    """The benchmark workload (2048^2, S 512, margin 16, winc 10, 2,088,960
    visibilities, 32x oversampled 16-tap kernels) through both gridders and
    the CPU restatement of grid.c (about 20 s on the host).  Each gridder's
    FP32 rounding leaves ~1e-6 against FP64, independently, so the two agree
    to ~sqrt(2) of that."""
    obs = sim.wtowers_plain(seed=1)
    u, v, w, vis = obs.flat()
    wk = sim.generate_wkernel(0.1, np.arange(-5, 6, 1.0), 16, 32)
    out = {}
    for gridder in (rg.RG_WTOWERS_GRIDDER_ROMEIN, rg.RG_WTOWERS_GRIDDER_STRIP):
        ctx = _ctx(rg, gridder)
        g = np.zeros((2048, 2048), np.complex128)
        ctx.grid_wtowers(g, 2048, 0.1, V(rg, u, v, w, vis), wk, 512, 16, 10.0)
        st = ctx.last_stats()
        assert st["strip_gridder"] == (gridder == rg.RG_WTOWERS_GRIDDER_STRIP)
        assert st["gridded"] + st["dropped"] == len(u)
        out[gridder] = g
    ref = oracle.grid_wtowers(2048, 0.1, u, v, w, vis, wk, 512, 16, 10.0)
    assert rel_rms(out[rg.RG_WTOWERS_GRIDDER_STRIP], ref) < TOL
    assert rel_rms(out[rg.RG_WTOWERS_GRIDDER_STRIP], out[rg.RG_WTOWERS_GRIDDER_ROMEIN]) < 3e-6


def test_strip_gridder_ragged_and_edges(rg, sim, oracle):
    """Counts that are not multiples of the list batch (32) or of the CTA's
    four warps, and footprints crossing the sub-grid's edges (the linear
    index wraps a column past the right edge into the next row; rows past
    the top or bottom are dropped)."""
    th, n = 0.1, 512
    wkt = sim.generate_wkernel(th, np.arange(-6, 7, 1.0))
    ctx = _ctx(rg, rg.RG_WTOWERS_GRIDDER_STRIP)
    rng = np.random.default_rng(5)
    for count in (1, 2, 33, 257, 1025):
        u = rng.uniform(-2500, 2500, count)
        v = rng.uniform(-2500, 2500, count)
        w = rng.uniform(-40, 40, count)
        vis = rng.normal(size=count) + 1j * rng.normal(size=count)
        g = np.zeros((n, n), np.complex128)
        ctx.grid_wtowers(g, n, th, V(rg, u, v, w, vis), wkt, 256, 24, 10.0, flags=rg.RG_GRID_OVERWRITE)
        ref = oracle.grid_wtowers(n, th, u, v, w, vis, wkt, 256, 24, 10.0)
        assert rel_rms(g, ref) < TOL
        assert ctx.last_stats()["strip_gridder"] == 1


def test_strip_gridder_empty_and_accumulate(rg, sim, oracle, wproj_data):
    ctx = _ctx(rg, rg.RG_WTOWERS_GRIDDER_STRIP)
    wkt = sim.generate_wkernel(0.1, np.arange(-6, 7, 1.0))
    e = np.zeros(0)
    g = np.full((256, 256), 1.0 + 0j)
    ctx.grid_wtowers(g, 256, 0.1, V(rg, e, e, e, e.astype(np.complex128)), wkt, 256, 16, 10.0)
    assert np.all(g == 1.0)
    obs, u, v, w, vis = wproj_data
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    ref = oracle.grid_wtowers(n, th, u, v, w, vis, wkt, 256, 16, 10.0)
    g = np.zeros((n, n), np.complex128)
    for k in range(3):
        ctx.grid_wtowers(g, n, th, V(rg, u, v, w, vis), wkt, 256, 16, 10.0)
        assert rel_rms(g, (k + 1) * ref) < TOL


def test_strip_gridder_graph_replay(rg, sim, oracle, wproj_data):
    """Device buffers: eager (+ tuning + capture), then graph replays of the
    strip gridder's pass, tracking new data in the same buffers."""
    obs, u, v, w, vis = wproj_data
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    wkt = sim.generate_wkernel(th, np.arange(-6, 7, 1.0))
    ref = oracle.grid_wtowers(n, th, u, v, w, vis, wkt, 256, 32, 10.0)
    d = torch.device("cuda", 0)
    du, dv, dw, dvis = (torch.from_numpy(np.ascontiguousarray(a)).to(d) for a in (u, v, w, vis))
    dwk = torch.from_numpy(np.ascontiguousarray(wkt.data)).to(d)
    g = torch.zeros((n, n), dtype=torch.complex128, device=d)
    ctx = _ctx(rg, rg.RG_WTOWERS_GRIDDER_STRIP)
    Vd = rg.Visibilities(du, dv, dw, dvis)
    graph = []
    for _ in range(4):
        ctx.grid_wtowers(g, n, th, Vd, wkt, 256, 32, 10.0, flags=rg.RG_GRID_OVERWRITE, wkern_data=dwk)
        torch.cuda.synchronize()
        assert rel_rms(g.cpu().numpy(), ref) < TOL
        st = ctx.last_stats()
        graph.append(st["graph"])
        assert st["strip_gridder"] == 1
    assert graph == [0, 1, 1, 1]
    dvis.mul_(-3.0)
    ctx.grid_wtowers(g, n, th, Vd, wkt, 256, 32, 10.0, flags=rg.RG_GRID_OVERWRITE, wkern_data=dwk)
    torch.cuda.synchronize()
    assert rel_rms(g.cpu().numpy(), -3.0 * ref) < TOL


def test_gridder_choice(rg, sim, wproj_data):
    """AUTO lets the tuner pick; a shape the strip gridder does not cover
    (sub-grid 128) runs Romein's even when the strip gridder is chosen;
    switching the choice on a context re-tunes and stays correct."""
    obs, u, v, w, vis = wproj_data
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    wkt = sim.generate_wkernel(th, np.arange(-6, 7, 1.0))
    Vs = V(rg, u, v, w, vis)
    ctx = rg.Context(0)
    grids = []
    for gridder in (rg.RG_WTOWERS_GRIDDER_AUTO, rg.RG_WTOWERS_GRIDDER_STRIP, rg.RG_WTOWERS_GRIDDER_ROMEIN):
        ctx.set_wtowers_gridder(gridder)
        g = np.zeros((n, n), np.complex128)
        for _ in range(2):
            g[:] = 0
            ctx.grid_wtowers(g, n, th, Vs, wkt, 256, 16, 10.0)
        st = ctx.last_stats()
        if gridder == rg.RG_WTOWERS_GRIDDER_AUTO:
            assert st["strip_gridder"] in (0, 1)
        else:
            assert st["strip_gridder"] == (gridder == rg.RG_WTOWERS_GRIDDER_STRIP)
        grids.append(g)
    assert rel_rms(grids[1], grids[2]) < 3e-6 and rel_rms(grids[0], grids[2]) < 3e-6
    ctx.set_wtowers_gridder(rg.RG_WTOWERS_GRIDDER_STRIP)
    g = np.zeros((n, n), np.complex128)
    ctx.grid_wtowers(g, n, th, Vs, wkt, 128, 16, 10.0)
    assert ctx.last_stats()["strip_gridder"] == 0
    with pytest.raises(rg.RGError):
        ctx.set_wtowers_gridder(7)
