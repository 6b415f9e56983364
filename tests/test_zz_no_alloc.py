"""rg_grid_wprojection_noalloc: W-projection for callers that cannot allocate.

Callers such as code running inside another framework's memory budget or a
real-time pipeline that forbids allocation after start-up cannot let the
library call cudaMalloc; this entry point keeps its intermediates in a fixed
device array instead.  The test allocates the inputs and the output itself (as
such a caller would), calls the entry point through the C ABI twice in a row,
and checks both results against rg_grid_wprojection and against the CPU
oracle (the restatement of the reference's grid_wprojection) within the
gridders' parity tolerance (relative RMS 1e-5).  The second call also shows
that the shared array is cleared between calls.  This file is collected last so that a
run stopping at the first failure has already run every other test."""
import ctypes as ct

import numpy as np
import pytest

from conftest import rel_rms

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.fixture(scope="module")
def case(sim):
    obs = sim.wproj_plain()
    u, v, w, vis = obs.flat()
    # 8x8 taps, 4x oversampling, planes every 10 lambda: 363,520 taps, under
    # the entry point's 524,288-tap limit
    wk = sim.wkernel_for(w, obs.meta["theta"], 10.0, size=8, oversampling=4)
    return obs.meta["grid_size"], obs.meta["theta"], (u, v, w, vis), wk


def _structs(rg, tensors, wk_dev, wk):
    u, v, w, vis = tensors
    vs = rg._Vis(u.data_ptr(), v.data_ptr(), w.data_ptr(), vis.data_ptr(), u.numel())
    ws = rg._WKern(wk_dev.data_ptr(), wk.plane_count, wk.size, wk.oversampling, wk.w_min, wk.w_step)
    return vs, ws


def test_noalloc_matches_wprojection_twice(rg, oracle, case):
    torch = pytest.importorskip("torch")
    n, th, arrays, wk = case
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(0)
    tensors = [torch.from_numpy(a).to(dev) for a in arrays]
    wk_dev = torch.from_numpy(np.ascontiguousarray(wk.data)).to(dev)
    vs, ws = _structs(rg, tensors, wk_dev, wk)

    ctx = rg.Context(0)
    ref = np.zeros((n, n), np.complex128)
    ctx.grid_wprojection(ref, n, th, rg.Visibilities(*arrays), wk)
    ctx.close()

    L = rg.lib()
    stream = torch.cuda.current_stream(dev).cuda_stream
    outs = []
    for _ in range(2):
        out = torch.full((n, n), 3.0 + 1.0j, dtype=torch.complex128, device=dev)
        st = L.rg_grid_wprojection_noalloc(ct.c_void_p(out.data_ptr()), n, th, ct.byref(vs),
                                           ct.byref(ws), rg.RG_GRID_OVERWRITE, ct.c_void_p(stream))
        assert st == 0, L.rg_last_error()
        torch.cuda.synchronize()
        outs.append(out.cpu().numpy())
    cpu = oracle.grid_wprojection(n, th, *arrays, wk)
    for o in outs:
        assert rel_rms(o, ref) < TOL
        assert rel_rms(o, cpu) < TOL
    assert rel_rms(outs[1], outs[0]) < TOL

    # accumulate semantics, as rg_grid_wprojection
    acc = torch.from_numpy(outs[0].copy()).to(dev)
    assert L.rg_grid_wprojection_noalloc(ct.c_void_p(acc.data_ptr()), n, th, ct.byref(vs),
                                         ct.byref(ws), rg.RG_GRID_ACCUMULATE,
                                         ct.c_void_p(stream)) == 0
    torch.cuda.synchronize()
    assert rel_rms(acc.cpu().numpy(), 2 * ref) < TOL


def test_noalloc_rejects_what_it_cannot_hold(rg, case):
    torch = pytest.importorskip("torch")
    n, th, arrays, wk = case
    dev = torch.device("cuda", 0)
    tensors = [torch.from_numpy(a).to(dev) for a in arrays]
    wk_dev = torch.from_numpy(np.ascontiguousarray(wk.data)).to(dev)
    vs, ws = _structs(rg, tensors, wk_dev, wk)
    L = rg.lib()
    big = torch.zeros((2048, 2048), dtype=torch.complex128, device=dev)
    assert L.rg_grid_wprojection_noalloc(ct.c_void_p(big.data_ptr()), 2048, th, ct.byref(vs),
                                         ct.byref(ws), 1, None) == 4
    assert b"1024" in L.rg_last_error()
    host = np.zeros((n, n), np.complex128)
    assert L.rg_grid_wprojection_noalloc(ct.c_void_p(host.ctypes.data), n, th, ct.byref(vs),
                                         ct.byref(ws), 1, None) == 1

    # the checks rg_grid_wprojection makes: a non-finite w_min is rejected on the host
    bad = rg._WKern(wk_dev.data_ptr(), wk.plane_count, wk.size, wk.oversampling, float("nan"), wk.w_step)
    assert L.rg_grid_wprojection_noalloc(ct.c_void_p(big.data_ptr()), n, th, ct.byref(vs),
                                         ct.byref(bad), 1, None) == 1
    assert L.rg_grid_wprojection_noalloc(ct.c_void_p(big.data_ptr()), n, float("nan"), ct.byref(vs),
                                         ct.byref(ws), 1, None) == 1


def test_noalloc_rejected_call_leaves_grid(rg, case):
    """A call rejected for its data (here every w lies beyond the kernel
    table) reports the error before it writes the caller's grid."""
    torch = pytest.importorskip("torch")
    n, th, arrays, wk = case
    dev = torch.device("cuda", 0)
    u, v, w, vis = arrays
    far = np.full_like(w, wk.w_min + wk.plane_count * wk.w_step + 1000.0)
    tensors = [torch.from_numpy(a).to(dev) for a in (u, v, far, vis)]
    wk_dev = torch.from_numpy(np.ascontiguousarray(wk.data)).to(dev)
    vs, ws = _structs(rg, tensors, wk_dev, wk)
    L = rg.lib()
    out = torch.full((n, n), 3.0 + 1.0j, dtype=torch.complex128, device=dev)
    st = L.rg_grid_wprojection_noalloc(ct.c_void_p(out.data_ptr()), n, th, ct.byref(vs), ct.byref(ws),
                                       rg.RG_GRID_OVERWRITE, None)
    assert st == 1 and b"w-kernel table" in L.rg_last_error()
    torch.cuda.synchronize()
    assert bool((out == (3.0 + 1.0j)).all())
