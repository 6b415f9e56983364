"""W-towers schedules: the autotuner's choices and graph replay of whole
passes (device buffers), including data that changes under the same buffers
and data that outgrows the sized capacities."""
import numpy as np
import pytest

from conftest import rel_rms

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def case(sim):
    obs = sim.wproj_plain()
    u, v, w, vis = obs.flat()
    th, n = obs.meta["theta"], obs.meta["grid_size"]
    wkt = sim.generate_wkernel(th, np.arange(-6, 7, 1.0))
    return n, th, u, v, w, vis, wkt


def _dev(*arrays):
    d = torch.device("cuda", 0)
    return [torch.from_numpy(np.ascontiguousarray(a)).to(d) for a in arrays]


def test_graph_replay_tracks_the_data(rg, sim, oracle, case):
    n, th, u, v, w, vis, wkt = case
    ctx = rg.Context(0)
    ref = oracle.grid_wtowers(n, th, u, v, w, vis, wkt, 128, 16, 10.0)
    du, dv, dw, dvis = _dev(u, v, w, vis)
    dwk = _dev(wkt.data)[0]
    g = torch.zeros((n, n), dtype=torch.complex128, device="cuda")
    V = rg.Visibilities(du, dv, dw, dvis)
    launches, graph = [], []
    for _ in range(4):  # eager (+ tuning + capture), then graph replays
        ctx.grid_wtowers(g, n, th, V, wkt, 128, 16, 10.0, flags=rg.RG_GRID_OVERWRITE, wkern_data=dwk)
        torch.cuda.synchronize()
        assert rel_rms(g.cpu().numpy(), ref) < 1e-5
        launches.append(ctx.last_stats()["launches"])
        graph.append(ctx.last_stats()["graph"])
    assert launches[-1] == launches[-2] > 0
    assert graph == [0, 1, 1, 1]
    # new values in the same buffers: the replayed graph reads them
    dvis.mul_(2.0)
    ctx.grid_wtowers(g, n, th, V, wkt, 128, 16, 10.0, flags=rg.RG_GRID_OVERWRITE, wkern_data=dwk)
    torch.cuda.synchronize()
    assert rel_rms(g.cpu().numpy(), 2 * ref) < 1e-5
    # accumulate mode through the graph
    ctx.grid_wtowers(g, n, th, V, wkt, 128, 16, 10.0, flags=rg.RG_GRID_ACCUMULATE, wkern_data=dwk)
    ctx.grid_wtowers(g, n, th, V, wkt, 128, 16, 10.0, flags=rg.RG_GRID_ACCUMULATE, wkern_data=dwk)
    torch.cuda.synchronize()
    assert rel_rms(g.cpu().numpy(), 6 * ref) < 1e-5


def test_graph_replay_outgrowing_the_plan(rg, sim, oracle, case):
    """The plan is sized on clustered data; the same buffers then hold the
    whole observation, whose sub-grids exceed the capacities: the replay
    detects the overflow, writes nothing, and the call reruns eagerly."""
    n, th, u, v, w, vis, wkt = case
    ctx = rg.Context(0)
    m = len(u)
    sel = np.argsort(np.hypot(u, v))[: m // 50]
    cu, cv, cw, cvis = (np.resize(a[sel], m) for a in (u, v, w, vis))
    du, dv, dw, dvis = _dev(cu, cv, cw, cvis)
    dwk = _dev(wkt.data)[0]
    g = torch.zeros((n, n), dtype=torch.complex128, device="cuda")
    V = rg.Visibilities(du, dv, dw, dvis)
    for _ in range(3):
        ctx.grid_wtowers(g, n, th, V, wkt, 128, 16, 10.0, flags=rg.RG_GRID_OVERWRITE, wkern_data=dwk)
    small = ctx.last_stats()["active_subgrids"]
    for t, a in zip((du, dv, dw, dvis), (u, v, w, vis)):
        t.copy_(torch.from_numpy(a))
    ctx.grid_wtowers(g, n, th, V, wkt, 128, 16, 10.0, flags=rg.RG_GRID_OVERWRITE, wkern_data=dwk)
    torch.cuda.synchronize()
    assert ctx.last_stats()["active_subgrids"] > small
    ref = oracle.grid_wtowers(n, th, u, v, w, vis, wkt, 128, 16, 10.0)
    assert rel_rms(g.cpu().numpy(), ref) < 1e-5


def test_autotune_choices_and_results(rg, sim, case):
    n, th, u, v, w, vis, wkt = case
    V = rg.Visibilities(u, v, w, vis)
    out = {}
    for tune in (False, True):
        ctx = rg.Context(0)
        ctx.set_autotune(tune)
        g = np.zeros((n, n), np.complex128)
        for _ in range(2):
            g[:] = 0
            ctx.grid_wtowers(g, n, th, V, wkt, 128, 16, 10.0)
        st = ctx.last_stats()
        out[tune] = g.copy()
        assert st["romein_points"] in (2, 4, 8) and st["group_items_per_sm"] in (4, 8, 16)
        if not tune:
            assert (st["romein_points"], st["group_items_per_sm"]) == (8, 8)
    assert rel_rms(out[True], out[False]) < 1e-6


def test_batch_matches_single_calls(rg, sim, oracle, case):
    """rg_grid_wtowers_batch over host buffers (pinned and pageable), device
    buffers, accumulate and overwrite: every grid equals the single-call one."""
    n, th, u, v, w, vis, wkt = case
    ctx = rg.Context(0)
    rng = np.random.default_rng(3)
    obs = []
    for k in range(5):  # same count, different data
        perm = rng.permutation(len(u))
        obs.append(tuple(np.ascontiguousarray(a[perm]) * (1.0 + 0.5 * k if j == 3 else 1.0)
                         for j, a in enumerate((u, v, w, vis))))
    ref = [oracle.grid_wtowers(n, th, *o, wkt, 128, 16, 10.0) for o in obs]
    pinned = [torch.from_numpy(np.stack([a.real if np.iscomplexobj(a) else a for a in o[:3]]))
              .pin_memory() for o in obs]
    vis_list = [rg.Visibilities(p[0].numpy(), p[1].numpy(), p[2].numpy(), o[3]) for p, o in zip(pinned, obs)]
    grids = [torch.zeros((n, n), dtype=torch.complex128).pin_memory().numpy() for _ in obs]
    ctx.grid_wtowers_batch(grids, n, th, vis_list, wkt, 128, 16, 10.0, flags=rg.RG_GRID_OVERWRITE)
    for g, r in zip(grids, ref):
        assert rel_rms(g, r) < 1e-5
    ctx.grid_wtowers_batch(grids, n, th, vis_list, wkt, 128, 16, 10.0)  # accumulate
    for g, r in zip(grids, ref):
        assert rel_rms(g, 2 * r) < 1e-5
    dvis = [rg.Visibilities(*_dev(*o)) for o in obs]
    dgrids = [torch.zeros((n, n), dtype=torch.complex128, device="cuda") for _ in obs]
    ctx.grid_wtowers_batch(dgrids, n, th, dvis, wkt, 128, 16, 10.0, flags=rg.RG_GRID_OVERWRITE)
    torch.cuda.synchronize()
    for g, r in zip(dgrids, ref):
        assert rel_rms(g.cpu().numpy(), r) < 1e-5


def test_batch_with_a_step_that_outgrows_the_plan(rg, sim, oracle, case):
    """Steps 0-1 clustered (the plan is sized on them), steps 2-3 the whole
    observation with the same visibility count: step 2 overflows inside the
    pipelined batch, stops the later steps' writes, and both are rerun."""
    n, th, u, v, w, vis, wkt = case
    m = len(u)
    sel = np.argsort(np.hypot(u, v))[: m // 50]
    clustered = tuple(np.ascontiguousarray(np.resize(a[sel], m)) for a in (u, v, w, vis))
    full = (u, v, w, vis)
    obs = [clustered, clustered, full, full]
    ctx = rg.Context(0)
    grids = [np.zeros((n, n), np.complex128) for _ in obs]
    ctx.grid_wtowers_batch(grids, n, th, [rg.Visibilities(*o) for o in obs], wkt, 128, 16, 10.0,
                           flags=rg.RG_GRID_OVERWRITE)
    for g, o in zip(grids, obs):
        assert rel_rms(g, oracle.grid_wtowers(n, th, *o, wkt, 128, 16, 10.0)) < 1e-5
