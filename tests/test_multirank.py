"""The multi-GPU partitions (radio-gridders_b200/sharding.py, used by
bench.py), run as world_size-2 gloo ranks on CPU.

W-towers: one observation's towers are split over the ranks by the library's
own partition (rg_wtowers_partition, a host function: balanced by
visibilities and active w-floors), each rank grids its share (the oracle's
W-towers restricted to those towers stands in for rg_grid_wtowers_part,
which needs a B200) and sharding.reduce_grid sums the FP64 master grids onto
rank 0.  The towers are independent until the add-back, so the sum must
equal gridding the whole observation on one rank to FP64 rounding.
W-projection: contiguous visibility shares, gridded and reduced the same way.
DFT: bands of image rows (the oracle's pixels stand in for
rg_dft_image_rows), gathered on every rank.  A rank that raises is reported
as a failure, not a hang (short process-group timeout)."""
import datetime
import importlib
import os
import socket
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


S, M, WINC = 128, 16, 10.0


def _observation(sim):
    obs = sim.wproj_plain(seed=0, n_dump=8)
    u, v, w, vis = obs.flat()
    wk = sim.generate_wkernel(obs.meta["theta"], np.arange(-6.0, 7.0, 1.0), 8, 4)
    return u, v, w, vis, obs.meta, wk


def _worker(rank, world, port, out_path, fail_rank):
    sys.path.insert(0, REPO)
    import torch
    import torch.distributed as dist

    import oracle
    sharding = importlib.import_module("radio-gridders_b200.sharding")
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=30))
    try:
        sim = importlib.import_module("radio-gridders_b200.simulate")
        u, v, w, vis, meta, wk = _observation(sim)
        if rank == fail_rank:
            raise RuntimeError("injected failure on rank %d" % rank)
        n, th = meta["grid_size"], meta["theta"]
        nv, nf = oracle.wtowers_census(n, th, u, v, w, S, M, WINC)
        parts = sharding.tower_parts(nv, nf, world)
        g = oracle.grid_wtowers(n, th, u, v, w, vis, wk, S, M, WINC, towers=(parts == rank))
        t = torch.from_numpy(g)
        sharding.reduce_grid(t, world)
        # W-projection over contiguous visibility shares
        b, e = sharding.vis_share(len(u), world, rank)
        wkp = sim.wkernel_for(w, th, 10.0, size=8, oversampling=4)  # planes over the whole w range
        gp = torch.from_numpy(oracle.grid_wprojection(n, th, u[b:e], v[b:e], w[b:e], vis[b:e], wkp))
        sharding.reduce_grid(gp, world)
        # DFT over bands of image rows, on a smaller image
        nd = 96
        ranges = sharding.dft_row_ranges(nd, world)
        row0, nrows = ranges[rank]
        py, px = np.divmod(np.arange(row0 * nd, (row0 + nrows) * nd), nd)
        band = oracle.dft_pixels(nd, th, u, v, w, vis, px, py).reshape(nrows, nd)
        img = sharding.gather_rows(torch.from_numpy(band), nd, ranges, world)
        if rank == 0:
            np.save(out_path, t.numpy())
            np.save(out_path + ".parts.npy", parts)
            np.save(out_path + ".wproj.npy", gp.numpy())
            np.save(out_path + ".dft.npy", img.numpy())
    finally:
        dist.destroy_process_group()


def _run(world, fail_rank, tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "master.npy")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, world, _free_port.port, out, fail_rank))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    return codes, out


def test_two_ranks_tower_shares_sum_to_the_whole(sim, oracle, tmp_path):
    _free_port.port = _free_port()
    codes, out = _run(2, -1, tmp_path)
    assert codes == [0, 0]
    got = np.load(out)
    u, v, w, vis, meta, wk = _observation(sim)
    n, th = meta["grid_size"], meta["theta"]
    ref = oracle.grid_wtowers(n, th, u, v, w, vis, wk, S, M, WINC)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12
    # both ranks had towers with data, and the loads are balanced
    parts = np.load(out + ".parts.npy")
    nv, nf = oracle.wtowers_census(n, th, u, v, w, S, M, WINC)
    cost = nv + 2400.0 * nf
    loads = [cost[parts == r].sum() for r in range(2)]
    assert min(loads) > 0 and max(loads) <= 1.25 * np.mean(loads) + cost.max()
    # W-projection shares sum to the whole, the DFT bands make the whole image
    gp = np.load(out + ".wproj.npy")
    refp = oracle.grid_wprojection(n, th, u, v, w, vis, sim.wkernel_for(w, th, 10.0, size=8, oversampling=4))
    assert np.linalg.norm(gp - refp) / np.linalg.norm(refp) < 1e-12
    img = np.load(out + ".dft.npy")
    assert np.max(np.abs(img - oracle.dft_image(96, th, u, v, w, vis))) < 1e-9 * np.abs(img).max()


def test_share_arithmetic():
    """Visibility shares tile [0, n) with sizes one apart; row bands tile the
    image, start on multiples of 32 and are as even as that allows."""
    sharding = importlib.import_module("radio-gridders_b200.sharding")
    for n, world in ((10, 3), (7, 8), (2_088_960, 8), (0, 2)):
        spans = [sharding.vis_share(n, world, r) for r in range(world)]
        assert spans[0][0] == 0 and spans[-1][1] == n
        assert all(spans[r][1] == spans[r + 1][0] for r in range(world - 1))
        sizes = [e - b for b, e in spans]
        assert max(sizes) - min(sizes) <= 1
    for n, world in ((2048, 8), (1000, 3), (96, 2), (50, 4)):
        ranges = sharding.dft_row_ranges(n, world)
        assert ranges[0][0] == 0 and sum(k for _, k in ranges) == n
        assert all(ranges[r][0] + ranges[r][1] == ranges[r + 1][0] for r in range(world - 1))
        assert all(r0 % 32 == 0 or k == 0 for r0, k in ranges)


def test_partition_is_deterministic_and_balanced(rg):
    """Largest first to the least loaded part: every tower gets a part in
    range, equal inputs give equal outputs, and no part exceeds the mean by
    more than the largest tower."""
    rng = np.random.default_rng(3)
    nv = rng.integers(0, 200_000, 81)
    nf = rng.integers(0, 60, 81)
    for parts_n in (1, 2, 3, 8):
        p1 = rg.partition_towers(nv, nf, parts_n)
        p2 = rg.partition_towers(nv.copy(), nf.copy(), parts_n)
        assert np.array_equal(p1, p2) and p1.min() >= 0 and p1.max() < parts_n
        cost = nv + 2400.0 * nf
        loads = np.array([cost[p1 == r].sum() for r in range(parts_n)])
        assert loads.max() <= loads.mean() + cost.max()
    with pytest.raises(rg.RGError):
        rg.partition_towers(nv, nf, 0)


def test_failing_rank_is_reported_not_hung(tmp_path):
    _free_port.port = _free_port()
    codes, _ = _run(2, 1, tmp_path)
    assert codes[1] != 0          # the failing rank exits with an error
    assert all(c is not None for c in codes)  # and nobody hangs past the timeout
