"""The project's synthetic-data and w-kernel generator (CPU)."""
import importlib

import numpy as np
import pytest


def test_pswf_matches_scipy(sim):
    special = pytest.importorskip("scipy.special")
    for c in (3.0, 4 * np.pi, 7 * np.pi):
        x = np.linspace(-0.99, 0.99, 41)
        ref = special.pro_ang1(0, 0, c, x)[0] / special.pro_ang1(0, 0, c, 0.0)[0]
        assert np.max(np.abs(sim.pswf0(c, x) - ref)) < 1e-9


def test_kernel_w0_is_real_and_symmetric(sim):
    wk = sim.generate_wkernel(0.1, np.array([0.0]), 16, 8)
    k0 = wk.data[0, 0, 0]  # sub-cell offset 0: taps at integer offsets -8..7
    assert np.max(np.abs(k0.imag)) < 1e-12 * np.abs(k0).max()
    # symmetric about the centre tap (index 8): K(p) = K(-p)
    assert np.allclose(k0[1:, 1:], k0[1:, 1:][::-1, ::-1], atol=1e-14)


def test_kernel_w_symmetry(sim):
    """K_{-w}(p) = conj(K_w(-p)): the screen of -w is the conjugate screen
    (real, even taper).  Checked on the integer-offset taps, where -p is again
    a tap; the one-sample asymmetry of the even-length screen (l = -theta/2 is
    sampled, +theta/2 is not) sits where the taper is ~1e-8."""
    wk = sim.generate_wkernel(0.1, np.array([-40.0, 40.0]), 16, 4)
    neg, pos = wk.data[0, 0, 0, 1:, 1:], wk.data[1, 0, 0, 1:, 1:]
    assert np.max(np.abs(neg - np.conj(pos[::-1, ::-1]))) < 1e-6 * np.abs(pos).max()


def test_kernel_normalisation(sim):
    """Sum of the integer-offset taps equals the taper at l = 0 (1)."""
    wk = sim.generate_wkernel(0.1, np.array([0.0]), 16, 8)
    assert abs(wk.data[0, 0, 0].sum() - 1.0) < 1e-6


def test_workloads_fit_the_grid(sim):
    obs = sim.wproj_plain()
    u, v, w, _ = obs.flat()
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    assert obs.nvis == 22464
    assert max(np.abs(u).max(), np.abs(v).max()) * th + 8 < n / 2


def test_generator_is_seeded(sim):
    a = sim.wproj_plain(seed=3, n_dump=4).flat()
    b = sim.wproj_plain(seed=3, n_dump=4).flat()
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("c", [3.0 * np.pi, 7.0 * np.pi, 5.0, 40.0])
def test_library_pswf_matches_generator(c):
    """rg_pswf0 (the C ABI generator's taper: Sturm bisection and inverse
    iteration for the Legendre coefficients) against the Python generator's
    psi_0 (dense symmetric eigensolver), which is itself checked against
    scipy.special.pro_ang1 above."""
    rg = importlib.import_module("radio-gridders_b200")
    sim = importlib.import_module("radio-gridders_b200.simulate")
    x = np.linspace(-1.0, 1.0, 301)
    assert np.abs(rg.pswf0(c, x) - sim.pswf0(c, x)).max() < 1e-13
    with pytest.raises(rg.RGError):
        rg.pswf0(c, np.array([1.5]))
