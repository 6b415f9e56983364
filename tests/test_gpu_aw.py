"""AW-projection on the device (rg_grid_awprojection) against the
restatement of the reference's convolve_aw_kernels + grid_awprojection
(src/reference/grid.c:557-637), which tests/test_oracle_pin.py pins
bit-identical to the reference's own build; from arrays, and from files
through grid.out -akern."""
import os
import subprocess

import numpy as np
import pytest

from conftest import rel_rms

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.fixture(scope="module")
def aw_case(sim):
    obs = sim.wtowers_plain(seed=3, n_st=30, n_dump=8, n_chan=4, lam=5120.0)
    u, v, w, vis = obs.flat()
    th = obs.meta["theta"]
    wk = sim.wkernel_for(w * 1.01, th, 2.0, size=8, oversampling=4)
    ak = sim.akern_for(obs, 3, 2, 8, jitter=0.1)
    return obs, wk, ak


def test_awprojection_matches_oracle(rg, ctx, oracle, aw_case):
    obs, wk, ak = aw_case
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    hv = rg.HierVis.of(obs)
    A = rg.AKernels(ak.freq, ak.time, ak.data, ak.t_min, ak.t_step, ak.f_min, ak.f_step)
    g = np.zeros((n, n), np.complex128)
    ctx.grid_awprojection(g, n, th, hv, wk, A)
    ref = oracle.grid_awprojection(n, th, hv, wk, ak)
    assert rel_rms(g, ref) < TOL
    # a baseline range, accumulated: two halves sum to the whole
    half = hv.uvw.shape[0] // 2
    g2 = np.zeros((n, n), np.complex128)
    ctx.grid_awprojection(g2, n, th, hv, wk, A, 0, half)
    ctx.grid_awprojection(g2, n, th, hv, wk, A, half, None)
    assert rel_rms(g2, ref) < TOL
    # a time outside the A-kernel axes is an error, not a wild read
    bad = rg.AKernels(ak.freq, ak.time, ak.data, ak.t_min + 100 * ak.t_step, ak.t_step, ak.f_min, ak.f_step)
    with pytest.raises(rg.RGError):
        ctx.grid_awprojection(g, n, th, hv, wk, bad)


def test_grid_out_akern(rg, oracle, aw_case, tmp_path):
    obs, wk, ak = aw_case
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    n_bl, n_time = obs.uvw.shape[:2]
    rg.write_vis_hdf5(str(tmp_path / "vis.h5"), obs.antenna1, obs.antenna2,
                      np.broadcast_to(obs.time, (n_bl, n_time)), obs.freq, obs.uvw, obs.vis)
    rg.write_wkern_hdf5(str(tmp_path / "wk.h5"), th, wk)
    A = rg.AKernels(ak.freq, ak.time, ak.data, ak.t_min, ak.t_step, ak.f_min, ak.f_step)
    rg.write_akern_hdf5(str(tmp_path / "ak.h5"), th, A)
    binary = os.path.join(os.path.dirname(__file__), "..", "radio-gridders_b200", "bin", "grid.out")
    r = subprocess.run([binary, f"-vis={tmp_path}/vis.h5", f"-wkernel={tmp_path}/wk.h5", f"-akern={tmp_path}/ak.h5",
                        f"-theta={th}", f"-lambda={obs.meta['lam']}", f"-grid={tmp_path}/aw.grid",
                        f"-image={tmp_path}/aw.img"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Gridder: AW-projection" in r.stdout
    wkr = rg.read_wkern_hdf5(str(tmp_path / "wk.h5"), th)
    akr = rg.read_akern_hdf5(str(tmp_path / "ak.h5"), th)
    ref = oracle.grid_awprojection(n, th, rg.HierVis.of(obs), wkr, akr)
    grid = np.fromfile(f"{tmp_path}/aw.grid", np.float64).view(np.complex128).reshape(n, n)
    assert rel_rms(grid, oracle.make_hermitian(ref.copy())) < TOL
    img = np.fromfile(f"{tmp_path}/aw.img", np.float64).reshape(n, n)
    assert rel_rms(img, oracle.image_from_grid(ref.copy())) < TOL
