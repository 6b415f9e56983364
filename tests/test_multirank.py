"""The multi-GPU path of bench.py, run as world_size-2 gloo ranks on CPU.

Each rank grids its own snapshot (the oracle stands in for the GPU gridder,
which needs a B200) and bench.reduce_master sums the master grids onto rank 0.
By linearity the result must equal gridding both snapshots together; a rank
that raises is reported as a failure, not a hang (short process-group
timeout)."""
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


def _snapshot(sim, rank):
    obs = sim.wproj_plain(seed=0, n_dump=8)
    # each rank observes a later stretch of hour angle (same array and sky)
    u, v, w, vis = obs.flat()
    rot = 0.15 * rank
    c, s = np.cos(rot), np.sin(rot)
    uu, vv = c * u - s * v, s * u + c * v
    return uu, vv, w, vis, obs.meta


def _worker(rank, world, port, out_path, fail_rank):
    sys.path.insert(0, REPO)
    import torch
    import torch.distributed as dist

    import bench
    import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=30))
    try:
        sim = importlib.import_module("radio-gridders_b200.simulate")
        u, v, w, vis, meta = _snapshot(sim, rank)
        if rank == fail_rank:
            raise RuntimeError("injected failure on rank %d" % rank)
        wk = sim.generate_wkernel(meta["theta"], np.arange(-1800, 1801, 10.0), 8, 4)
        g = oracle.grid_wprojection(meta["grid_size"], meta["theta"], u, v, w, vis, wk)
        t = torch.from_numpy(g)
        bench.reduce_master(t, world)
        if rank == 0:
            np.save(out_path, t.numpy())
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


def test_two_ranks_reduce_equals_joint_gridding(sim, oracle, tmp_path):
    _free_port.port = _free_port()
    codes, out = _run(2, -1, tmp_path)
    assert codes == [0, 0]
    got = np.load(out)
    wk = sim.generate_wkernel(0.1, np.arange(-1800, 1801, 10.0), 8, 4)
    parts = [_snapshot(sim, r) for r in range(2)]
    u = np.concatenate([p[0] for p in parts])
    v = np.concatenate([p[1] for p in parts])
    w = np.concatenate([p[2] for p in parts])
    vis = np.concatenate([p[3] for p in parts])
    meta = parts[0][4]
    ref = oracle.grid_wprojection(meta["grid_size"], meta["theta"], u, v, w, vis, wk)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12


def test_failing_rank_is_reported_not_hung(tmp_path):
    _free_port.port = _free_port()
    codes, _ = _run(2, 1, tmp_path)
    assert codes[1] != 0          # the failing rank exits with an error
    assert all(c is not None for c in codes)  # and nobody hangs past the timeout
