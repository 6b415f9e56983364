"""grid.out / dft.out end to end on the device: crocodile HDF5 files in, the
reference CPU pipeline's dirty image out (src/reference/main.c:261-294),
compared with the oracle."""
import os
import subprocess

import numpy as np
import pytest

from conftest import rel_rms

pytestmark = pytest.mark.gpu
BIN = os.path.join(os.path.dirname(__file__), "..", "radio-gridders_b200", "bin")


def run(name, *args):
    r = subprocess.run([os.path.join(BIN, name), *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    return r


@pytest.fixture(scope="module")
def files(rg, sim, tmp_path_factory):
    d = tmp_path_factory.mktemp("cli")
    obs = sim.wproj_plain(seed=7)
    n_bl, n_time = obs.uvw.shape[:2]
    rg.write_vis_hdf5(str(d / "vis.h5"), obs.antenna1, obs.antenna2,
                      np.broadcast_to(obs.time, (n_bl, n_time)), obs.freq, obs.uvw, obs.vis)
    th = obs.meta["theta"]
    u, v, w, vis = obs.flat()
    wk = sim.wkernel_for(w, th, 10.0, size=16, oversampling=8)
    rg.write_wkern_hdf5(str(d / "wk.h5"), th, wk)
    return d, obs, (u, v, w, vis), rg.read_wkern_hdf5(str(d / "wk.h5"), th)


def _load(path, n, complex_=False):
    a = np.fromfile(path, np.float64)
    return a.view(np.complex128).reshape(n, n) if complex_ else a.reshape(n, n)


@pytest.mark.parametrize("mode", ["wproj", "wtowers"])
def test_grid_out(oracle, files, mode):
    d, obs, (u, v, w, vis), wk = files
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    args = [f"-vis={d}/vis.h5", f"-wkernel={d}/wk.h5", f"-theta={th}", f"-lambda={obs.meta['lam']}",
            f"-image={d}/{mode}.img", f"-grid={d}/{mode}.grid"]
    if mode == "wproj":
        run("grid.out", *args, "-wproj")
        ref = oracle.grid_wprojection(n, th, u, v, w, vis, wk)
    else:
        run("grid.out", *args, "-subgrid=128", "-margin=16", "-winc=10")
        ref = oracle.grid_wtowers(n, th, u, v, w, vis, wk, 128, 16, 10.0)
    img_ref = oracle.image_from_grid(ref.copy())
    herm = oracle.make_hermitian(ref.copy())
    assert rel_rms(_load(f"{d}/{mode}.grid", n, True), herm) < 1e-5
    assert rel_rms(_load(f"{d}/{mode}.img", n), img_ref) < 1e-5


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("reduced", 2e-5)])
def test_dft_out(oracle, files, precision, tol):
    """At 64 pixels a 32-pixel tile spans |u| dl ~ 64 turns, so the
    FP64-reduced mode's FP32 increments leave ~3e-6; all-FP64 is exact."""
    d, obs, (u, v, w, vis), _ = files
    th, lam = obs.meta["theta"], 640.0
    n = int(np.floor(lam * th + 0.5))
    run("dft.out", f"-vis={d}/vis.h5", f"-theta={th}", f"-lambda={lam}", f"-image={d}/dft.img", "-hermitian",
        f"-precision={precision}")
    ref = oracle.dft_image(n, th, u, v, w, vis, factor=2.0)
    assert rel_rms(_load(f"{d}/dft.img", n), ref) < tol


def test_reference_wrapper_entry_points(rg, oracle, files):
    """rg_wtowers_cuda_flat / rg_wproj_cuda_flat / rg_image_dft_host_flat take
    the reference wrappers' argument lists (files, device grid, host grid,
    grid_size, theta, lambda, bl_min, bl_max, ...) and leave the dirty image
    as the real part of both complex buffers."""
    import ctypes as ct

    import torch
    d, obs, (u, v, w, vis), wk = files
    n, th, lam = obs.meta["grid_size"], obs.meta["theta"], obs.meta["lam"]
    L = rg.lib()
    for mode in ("wproj", "wtowers"):
        dev = torch.zeros((n, n), dtype=torch.complex128, device="cuda")
        host = np.zeros((n, n), np.complex128)
        args = [f"{d}/vis.h5".encode(), f"{d}/wk.h5".encode(), ct.c_void_p(dev.data_ptr()),
                host.ctypes.data_as(ct.c_void_p), n, th, lam, 0.0, 1e30]
        if mode == "wproj":
            st = L.rg_wproj_cuda_flat(*args, 256)
            ref = oracle.grid_wprojection(n, th, u, v, w, vis, wk)
        else:
            st = L.rg_wtowers_cuda_flat(*args, 128, 16, 10.0)
            ref = oracle.grid_wtowers(n, th, u, v, w, vis, wk, 128, 16, 10.0)
        assert st == 0, rg.lib().rg_last_error()
        img_ref = oracle.image_from_grid(ref.copy())
        assert rel_rms(host.real, img_ref) < 1e-5
        assert np.all(host.imag == 0)
        assert np.array_equal(dev.cpu().numpy(), host)
    lam_dft = 640.0
    m = int(np.floor(lam_dft * th + 0.5))
    host = np.zeros((m, m), np.complex128)
    st = L.rg_image_dft_host_flat(f"{d}/vis.h5".encode(), host.ctypes.data_as(ct.c_void_p), None, m, th,
                                  lam_dft, 0.0, 1e30, 64, 256)
    assert st == 0, rg.lib().rg_last_error()
    assert rel_rms(host.real, oracle.dft_image(m, th, u, v, w, vis, factor=1.0)) < 2e-5
    # errors come back as a status, not an exit
    assert L.rg_wtowers_cuda_flat(b"/nonexistent.h5", f"{d}/wk.h5".encode(), ct.c_void_p(dev.data_ptr()), None,
                                  n, th, lam, 0.0, 1e30, 128, 16, 10.0) != 0
