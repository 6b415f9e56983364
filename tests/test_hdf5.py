"""Crocodile HDF5 subset: the project's reader and writer behind the C ABI.

Host only (no device).  Round trips check that a written file reads back
bit-identically through load_vis/flatten_visibilities_CUDA's conventions
(src/reference/hdf5.c:173-318, src/common/hdf5.c:827-872) and load_wkern's
(src/reference/hdf5.c:321-413); files written by libhdf5 itself (the
reference's separable-kernel files, read by src/common/hdf5.c:372-500) pin the
reader against another writer when the reference tree is present."""
import os

import numpy as np
import pytest

C_LIGHT = 299792458.0
# the reference checkout (its root directory), when the caller provides one
REF = os.environ.get("RG_REFERENCE_ROOT")


@pytest.fixture(scope="module")
def obs(sim):
    return sim.wproj_plain(seed=5, n_dump=8)


def _write(rg, path, o):
    n_bl, n_time = o.uvw.shape[:2]
    rg.write_vis_hdf5(str(path), o.antenna1, o.antenna2, np.broadcast_to(o.time, (n_bl, n_time)),
                      o.freq, o.uvw, o.vis)


def test_vis_round_trip_bit_exact(rg, obs, tmp_path):
    p = tmp_path / "vis.h5"
    _write(rg, p, obs)
    vis, n_bl = rg.read_vis_hdf5(str(p))
    u, v, w, x = obs.flat()
    assert n_bl == obs.uvw.shape[0]
    assert vis.n == u.size
    for a, b in ((vis.u, u), (vis.v, v), (vis.w, w), (vis.vis, x)):
        np.testing.assert_array_equal(a, b)


def test_vis_baseline_length_filter(rg, obs, tmp_path):
    """Baselines are kept when the first uvw sample's (u, v) length lies in
    [bl_min, bl_max) metres (src/reference/hdf5.c:77-79)."""
    p = tmp_path / "vis.h5"
    _write(rg, p, obs)
    length = np.sqrt((obs.uvw[:, 0, :2] ** 2).sum(-1))
    lo, hi = np.quantile(length, [0.25, 0.75])
    vis, n_bl = rg.read_vis_hdf5(str(p), lo, hi)
    keep = (length >= lo) & (length < hi)
    assert n_bl == keep.sum()
    f = obs.freq[keep][:, None, :]
    np.testing.assert_array_equal(vis.u, (obs.uvw[keep][:, :, 0:1] * f / C_LIGHT).ravel())
    np.testing.assert_array_equal(vis.vis, obs.vis[keep].ravel())
    empty, n0 = rg.read_vis_hdf5(str(p), 1e12, 2e12)
    assert n0 == 0 and empty.n == 0


def test_vis_datasets_readable_generically(rg, obs, tmp_path):
    p = tmp_path / "vis.h5"
    _write(rg, p, obs)
    a1, a2 = int(obs.antenna1[0]), int(obs.antenna2[0])
    uvw = rg.hdf5_read(str(p), f"vis/{a1}/{a2}/uvw")
    np.testing.assert_array_equal(uvw, obs.uvw[0])
    vis = rg.hdf5_read(str(p), f"vis/{a1}/{a2}/vis")
    assert vis.shape[-1] == 2
    np.testing.assert_array_equal(vis.reshape(-1, 2)[:, 0], obs.vis[0].real.ravel())
    np.testing.assert_array_equal(vis.reshape(-1, 2)[:, 1], obs.vis[0].imag.ravel())


def test_wkern_round_trip(rg, sim, tmp_path):
    theta = 0.1
    wk = sim.generate_wkernel(theta, np.arange(-3, 4) * 40.0, size=8, oversampling=4)
    p = tmp_path / "wk.h5"
    rg.write_wkern_hdf5(str(p), theta, wk)
    back = rg.read_wkern_hdf5(str(p), theta)
    assert back.data.shape == wk.data.shape
    np.testing.assert_array_equal(back.data, wk.data)
    assert back.w_min == pytest.approx(wk.w_min, abs=1e-12)
    assert back.w_step == pytest.approx(wk.w_step, rel=1e-12)
    with pytest.raises(rg.RGError) as e:
        rg.read_wkern_hdf5(str(p), 0.2)  # no wkern/0.2 group
    assert e.value.status == 5


def test_missing_and_corrupt_files_are_io_errors(rg, obs, tmp_path):
    with pytest.raises(rg.RGError) as e:
        rg.read_vis_hdf5(str(tmp_path / "absent.h5"))
    assert e.value.status == 5
    p = tmp_path / "vis.h5"
    _write(rg, p, obs)
    raw = p.read_bytes()
    for cut in (0, 7, 100, len(raw) // 3, len(raw) - 9):
        q = tmp_path / f"cut{cut}.h5"
        q.write_bytes(raw[:cut])
        with pytest.raises(rg.RGError) as e:
            rg.read_vis_hdf5(str(q))
        assert e.value.status == 5
    junk = tmp_path / "junk.h5"
    junk.write_bytes(np.random.default_rng(0).integers(0, 256, 4096, dtype=np.uint8).tobytes())
    with pytest.raises(rg.RGError):
        rg.read_vis_hdf5(str(junk))


SEPKERN = [("src/wstack/sepkern_uv.hdf5", (4096, 8)), ("src/wstack/sepkern_w.hdf5", (4096, 4)),
           ("test/kernels/sze/sepkern_lm_highres.hdf5", (1, 100001)),
           ("test/kernels/sze/sepkern_n.hdf5", (1, 10001))]


@pytest.mark.parametrize("rel,shape", SEPKERN)
def test_reads_libhdf5_written_files(rg, rel, shape):
    """Separable-kernel files written by libhdf5 (read by
    src/common/hdf5.c:372-500: dataset sepkern/kern, root attributes du, dw,
    x0)."""
    if not REF:
        pytest.skip("set RG_REFERENCE_ROOT to the reference checkout to read its libhdf5-written files")
    path = os.path.join(REF, rel)
    if not os.path.exists(path):
        pytest.skip(f"{rel} not found under RG_REFERENCE_ROOT")
    kern = rg.hdf5_read(path, "sepkern/kern")
    assert kern.shape == shape
    assert np.isfinite(kern).all() and np.abs(kern).max() > 0
    for name in ("du", "dw", "x0"):
        assert np.isfinite(rg.hdf5_attr(path, "/", name))


def test_legacy_flat_layout_round_trip(rg, obs, tmp_path):
    """The legacy flat /vis group (rows of one time sample, a shared frequency
    axis, type attribute "Visibility"; src/common/hdf5.c:199-300): every row is
    its own baseline for the length cut."""
    n_bl, n_time = obs.uvw.shape[:2]
    rows = n_bl * n_time
    p = tmp_path / "flat.h5"
    rg.write_vis_flat_hdf5(str(p), np.repeat(obs.antenna1, n_time), np.repeat(obs.antenna2, n_time),
                           np.tile(obs.time, n_bl), obs.freq[0], obs.uvw.reshape(rows, 3),
                           obs.vis.reshape(rows, -1))
    vis, n_rows = rg.read_vis_hdf5(str(p))
    u, v, w, x = obs.flat()
    assert n_rows == rows
    for a, b in ((vis.u, u), (vis.v, v), (vis.w, w), (vis.vis, x)):
        np.testing.assert_array_equal(a, b)
    import ctypes as ct
    buf = ct.c_double()
    assert rg.lib().rg_hdf5_attr_f64(str(p).encode(), b"vis", b"type", ct.byref(buf)) == 5  # a string
    length = np.sqrt((obs.uvw.reshape(rows, 3)[:, :2] ** 2).sum(-1))
    lo = np.quantile(length, 0.5)
    _, kept = rg.read_vis_hdf5(str(p), lo)
    assert kept == int((length >= lo).sum())


def test_akern_round_trip(rg, sim, tmp_path):
    """A-kernel files (load_akern's layout, src/common/hdf5.c:652-820:
    akern/<theta>/<antenna>/<time>/<freq>/kern): written and read back with
    the same axes, frequencies and kernel values."""
    obs = sim.wtowers_plain(seed=3, n_st=6, n_dump=4, n_chan=3, lam=5120.0)
    ak = sim.akern_for(obs, 3, 3, 8)
    A = rg.AKernels(ak.freq, ak.time, ak.data, ak.t_min, ak.t_step, ak.f_min, ak.f_step)
    p = str(tmp_path / "ak.h5")
    rg.write_akern_hdf5(p, 0.1, A)
    back = rg.read_akern_hdf5(p, 0.1)
    np.testing.assert_array_equal(back.data, A.data)
    np.testing.assert_array_equal(back.freq, A.freq)
    np.testing.assert_array_equal(back.time, A.time)
    assert back.t_min == A.t_min and back.f_min == A.f_min
    assert abs(back.t_step - A.t_step) < 1e-12 * abs(A.t_step)
    with pytest.raises(rg.RGError):
        rg.read_akern_hdf5(p, 0.2)  # no akern/0.2 group


def test_hierarchical_read_keeps_baselines(rg, sim, tmp_path):
    """rg_read_vis_bl_hdf5: the same baselines, antennas, times, channels,
    uvw and visibilities as written, in the flat reader's order."""
    obs = sim.wtowers_plain(seed=3, n_st=6, n_dump=4, n_chan=3, lam=5120.0)
    p = tmp_path / "vis.h5"
    _write(rg, p, obs)
    hv = rg.read_vis_bl_hdf5(str(p))
    np.testing.assert_array_equal(hv.antenna1, obs.antenna1)
    np.testing.assert_array_equal(hv.antenna2, obs.antenna2)
    np.testing.assert_array_equal(hv.uvw, obs.uvw)
    np.testing.assert_array_equal(hv.freq, obs.freq)
    np.testing.assert_array_equal(hv.vis, obs.vis)
    np.testing.assert_array_equal(hv.time, np.broadcast_to(obs.time, hv.time.shape))
    flat, _ = rg.read_vis_hdf5(str(p))
    np.testing.assert_array_equal(flat.vis, hv.vis.ravel())
