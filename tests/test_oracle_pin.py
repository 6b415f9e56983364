"""The C restatement (oracle/rg_oracle.c) against the reference's own code.

Pinned two ways: against the committed golden fixture (outputs of the
reference's grid.c, tests/golden/make_golden.py), and, when the reference build
oracle/_ref is present, against it directly on fresh seeded inputs.  The bar is
bit-identity: the restatement keeps the reference's operation order."""
import numpy as np
import pytest

from conftest import rel_rms


def test_golden_wprojection(oracle, golden, golden_kernels):
    wk, _ = golden_kernels
    g = oracle.grid_wprojection(int(golden["grid_size"]), float(golden["theta"]), golden["u"],
                                golden["v"], golden["w"], golden["vis"], wk)
    assert np.array_equal(g, golden["grid_wprojection"])


def test_golden_wtowers(oracle, golden, golden_kernels):
    _, wkt = golden_kernels
    g, counts = oracle.grid_wtowers(int(golden["grid_size"]), float(golden["theta"]), golden["u"],
                                    golden["v"], golden["w"], golden["vis"], wkt,
                                    int(golden["subgrid"]), int(golden["margin"]),
                                    float(golden["winc"]), return_counts=True)
    assert np.array_equal(g, golden["grid_wtowers"])
    # every visibility gridded exactly once (src/reference/grid.c:519-530)
    assert counts.min() == 1 and counts.max() == 1


def test_golden_weight_hermitian_shift(oracle, golden):
    n, th = int(golden["grid_size"]), float(golden["theta"])
    assert np.array_equal(oracle.weight(n, th, golden["u"], golden["v"], golden["vis"]),
                          golden["weighted_vis"])
    assert np.array_equal(oracle.make_hermitian(golden["grid_wprojection"]), golden["hermitian"])
    assert np.array_equal(oracle.fft_shift(golden["grid_wprojection"]), golden["shifted"])


def test_frac_coord_matches_definition(oracle):
    # x = 3.26 cells, ov 8: cell floor(3.26 + 1/16) = 3, frac floor(0.26*8 + .5) = 2
    go, so = oracle.frac_coord(64, 8, 8, 0.1, 32.6, -10.0)
    assert go == (-1 + 32 - 4) * 64 + (3 + 32 - 4)
    assert so == 8 * 8 * (0 * 8 + 2)


@pytest.fixture(scope="module")
def wproj_case(sim):
    obs = sim.wproj_plain(seed=5, n_dump=24)
    u, v, w, vis = obs.flat()
    wk = sim.wkernel_for(w, obs.meta["theta"], 10.0)
    return obs, (u, v, w, vis), wk


def test_restated_equals_reference_wprojection(oracle, wproj_case):
    if not oracle.reference_available():
        pytest.skip("reference build (oracle/_ref) not present")
    obs, (u, v, w, vis), wk = wproj_case
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    a = oracle.grid_wprojection(n, th, u, v, w, vis, wk)
    b = oracle.ref_grid_wprojection(n, th, obs, wk)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("sub,margin,winc", [(128, 18, 10.0), (64, 20, 25.0), (256, 32, 5.0)])
def test_restated_equals_reference_wtowers(oracle, sim, wproj_case, sub, margin, winc):
    if not oracle.reference_available():
        pytest.skip("reference build (oracle/_ref) not present")
    obs, (u, v, w, vis), _ = wproj_case
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    wkt = sim.generate_wkernel(th, np.arange(-winc / 2 - 1, winc / 2 + 1.5, 1.0))
    mask = oracle.reference_safe_baselines(obs, n, th, sub, margin, 16, 8)
    o2 = oracle.subset_baselines(obs, mask)
    uu, vv, ww, vz = o2.flat()
    a = oracle.grid_wtowers(n, th, uu, vv, ww, vz, wkt, sub, margin, winc)
    b = oracle.ref_grid_wtowers(n, th, o2, wkt, sub, margin, winc)
    assert np.array_equal(a, b)


def test_restated_equals_reference_weight(oracle, wproj_case):
    if not oracle.reference_available():
        pytest.skip("reference build (oracle/_ref) not present")
    obs, (u, v, w, vis), _ = wproj_case
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    assert np.array_equal(oracle.weight(n, th, u, v, vis), oracle.ref_weight(n, th, obs))


def test_wtowers_equals_wprojection_for_small_w(oracle, sim):
    """Known answer: with every |w| < winc/2 all visibilities sit on floor 0 and
    W-towers must reproduce W-projection (up to the FFT round trip)."""
    obs = sim.wproj_plain(seed=7, n_dump=8)
    u, v, w, vis = obs.flat()
    w = w * (4.0 / np.abs(w).max())
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    wkt = sim.generate_wkernel(th, np.arange(-5, 6, 1.0))
    a = oracle.grid_wprojection(n, th, u, v, w, vis, wkt)
    # margin > kernel support: only the FFT round trip separates the two
    b = oracle.grid_wtowers(n, th, u, v, w, vis, wkt, 128, 18, 10.0)
    assert rel_rms(b, a) < 1e-13
    # margin == kernel support: footprints of visibilities within 1/(2 ov) cell of
    # a tower's low edge wrap to the previous sub-grid row (reference behaviour),
    # moving only the kernel's outermost taps
    b16 = oracle.grid_wtowers(n, th, u, v, w, vis, wkt, 128, 16, 10.0)
    assert rel_rms(b16, a) < 1e-9


def test_dft_single_visibility_is_a_fringe(oracle):
    n, th = 64, 0.1
    u, v, w = np.array([37.0]), np.array([-12.0]), np.array([0.0])
    vis = np.array([1.0 + 0.5j])
    img = oracle.dft_image(n, th, u, v, w, vis, factor=2.0)
    lm = th * (np.arange(n) - n // 2) / n
    ph = u[0] * lm[None, :] + v[0] * lm[:, None]
    ref = 2 * (vis[0].real * np.cos(2 * np.pi * ph) + vis[0].imag * np.sin(2 * np.pi * ph))
    assert np.max(np.abs(img - ref)) < 1e-12


def test_dft_point_source_at_centre(oracle, sim):
    """A unit source at the phase centre: constant visibilities, image peak at
    the centre pixel equal to 2 * number of visibilities."""
    obs = sim.wproj_plain(seed=3, n_dump=4)
    u, v, w, _ = obs.flat()
    vis = np.ones(len(u), np.complex128)
    n = 64
    img = oracle.dft_image(n, 0.1, u, v, w, vis, factor=2.0)
    assert abs(img[n // 2, n // 2] - 2 * len(u)) < 1e-9 * len(u)
    assert img.argmax() == (n // 2) * n + n // 2


def test_gridded_image_matches_dft_for_point_source(oracle, sim):
    """End-to-end convention check: W-projection grid -> image (hermitian,
    shift, FFT -1, shift) / taper agrees with the DFT oracle for a point source."""
    obs = sim.wproj_plain(seed=9, n_dump=32)
    u, v, w, _ = obs.flat()
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    l0, m0 = 0.012, -0.007
    vis = np.exp(-2j * np.pi * (u * l0 + v * m0 + w * (np.sqrt(1 - l0 * l0 - m0 * m0) - 1)))
    w = w * (300.0 / np.abs(w).max())  # keep the w-spread inside the 16-tap support
    vis = np.exp(-2j * np.pi * (u * l0 + v * m0 + w * (np.sqrt(1 - l0 * l0 - m0 * m0) - 1)))
    wk = sim.wkernel_for(w, th, 2.0, size=16, oversampling=32)
    g = oracle.grid_wprojection(n, th, u, v, w, vis, wk)
    img = oracle.image_from_grid(g)
    t = sim.taper_1d(th, n, wk.c)
    img = img / np.outer(t, t)
    ref = oracle.dft_image(n, th, u, v, w, vis, factor=2.0)
    c = slice(n // 4, 3 * n // 4)
    err = np.sqrt(np.mean((img[c, c] - ref[c, c]) ** 2)) / np.abs(ref).max()
    assert err < 1e-3
    # the source appears at (-l0, -m0) in this convention
    y, x = np.unravel_index(np.argmax(ref), ref.shape)
    assert abs((x - n // 2) * th / n + l0) < th / n and abs((y - n // 2) * th / n + m0) < th / n


def test_awprojection_restatement_matches_reference(sim, oracle, rg):
    """grid_awprojection after convolve_aw_kernels (src/reference/grid.c:
    557-637), the reference's own build against the restatement: bit-identical
    grids, and different from plain W-projection (the A-kernel channels'
    frequencies pick the planes)."""
    if not oracle.reference_available():
        pytest.skip("reference build absent")
    obs = sim.wtowers_plain(seed=3, n_st=30, n_dump=8, n_chan=4, lam=5120.0)
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    u, v, w, vis = obs.flat()
    wk = sim.wkernel_for(w * 1.01, th, 2.0, size=8, oversampling=4)
    ak = sim.akern_for(obs, 3, 2, 8, jitter=0.1)
    got = oracle.grid_awprojection(n, th, rg.HierVis.of(obs), wk, ak)
    ref = oracle.ref_grid_awprojection(n, th, obs, wk, ak)
    assert np.array_equal(got, ref)
    wp = oracle.grid_wprojection(n, th, u, v, w, vis, wk)
    assert np.linalg.norm(got - wp) / np.linalg.norm(wp) > 1e-6


def test_grid_simple_restatement_matches_reference(sim, oracle):
    """grid_simple (src/reference/grid.c:83-99): the restatement and the
    reference's build give bit-identical grids."""
    if not oracle.reference_available():
        pytest.skip("reference build absent")
    obs = sim.wproj_plain(seed=4, n_dump=8)
    u, v, w, vis = obs.flat()
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    assert np.array_equal(oracle.grid_simple(n, th, u, v, vis), oracle.ref_grid_simple(n, th, obs))
