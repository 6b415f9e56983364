"""CUDA gridders against the oracle and the reference's golden outputs.

Bar (north star): relative RMS of the uv grid <= 1e-5 against the FP64 CPU
gridder; the FP32 sub-grids and atomics leave ~1e-7."""
import numpy as np
import pytest

from conftest import rel_rms

pytestmark = pytest.mark.gpu
TOL = 1e-5


def V(rg, u, v, w, vis):
    return rg.Visibilities(u, v, w, vis)


def test_wprojection_golden(rg, ctx, golden, golden_kernels):
    wk, _ = golden_kernels
    n = int(golden["grid_size"])
    g = np.zeros((n, n), np.complex128)
    ctx.grid_wprojection(g, n, float(golden["theta"]),
                         V(rg, golden["u"], golden["v"], golden["w"], golden["vis"]), wk)
    assert rel_rms(g, golden["grid_wprojection"]) < TOL


def test_wtowers_golden(rg, ctx, golden, golden_kernels):
    _, wkt = golden_kernels
    n = int(golden["grid_size"])
    g = np.zeros((n, n), np.complex128)
    ctx.grid_wtowers(g, n, float(golden["theta"]),
                     V(rg, golden["u"], golden["v"], golden["w"], golden["vis"]), wkt,
                     int(golden["subgrid"]), int(golden["margin"]), float(golden["winc"]))
    assert rel_rms(g, golden["grid_wtowers"]) < TOL
    st = ctx.last_stats()
    assert st["gridded"] == len(golden["u"]) and st["dropped"] == 0


@pytest.fixture(scope="module")
def wproj_data(sim):
    obs = sim.wproj_plain()
    u, v, w, vis = obs.flat()
    return obs, u, v, w, vis


@pytest.mark.parametrize("ksize,ov", [(16, 8), (8, 4), (32, 2)])
def test_wprojection_vs_oracle(rg, ctx, sim, oracle, wproj_data, ksize, ov):
    obs, u, v, w, vis = wproj_data
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    if ksize == 32:  # keep the 32-tap footprint inside the grid
        keep = (np.abs(u) * th < n / 2 - 18) & (np.abs(v) * th < n / 2 - 18)
        u, v, w, vis = u[keep], v[keep], w[keep], vis[keep]
    wk = sim.wkernel_for(w, th, 10.0, size=ksize, oversampling=ov)
    g = np.zeros((n, n), np.complex128)
    ctx.grid_wprojection(g, n, th, V(rg, u, v, w, vis), wk)
    ref = oracle.grid_wprojection(n, th, u, v, w, vis, wk)
    assert rel_rms(g, ref) < TOL


def test_wprojection_fp64_and_converted_taps(rg, ctx, sim, oracle, wproj_data):
    """A call with fewer taps to read than its table holds reads the FP64
    table directly; a larger one converts the table to FP32 first.  The same
    visibilities sent twice take the second path; the grid must be twice the
    first call's, and both must match the oracle."""
    obs, u, v, w, vis = wproj_data
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    wk = sim.wkernel_for(w, th, 10.0, size=16, oversampling=8)
    ntaps = wk.plane_count * wk.oversampling ** 2 * wk.size ** 2
    assert len(u) * 16 * 16 * 16 < 24 * ntaps <= 2 * len(u) * 16 * 16 * 16  # one call each side
    g1 = np.zeros((n, n), np.complex128)
    ctx.grid_wprojection(g1, n, th, V(rg, u, v, w, vis), wk)
    dup = lambda a: np.ascontiguousarray(np.concatenate([a, a]))
    g2 = np.zeros((n, n), np.complex128)
    ctx.grid_wprojection(g2, n, th, V(rg, dup(u), dup(v), dup(w), dup(vis)), wk)
    assert rel_rms(g2, 2 * g1) < 1e-6
    assert rel_rms(g1, oracle.grid_wprojection(n, th, u, v, w, vis, wk)) < TOL


@pytest.mark.parametrize("sub,margin,winc", [(128, 16, 10.0), (64, 16, 10.0), (256, 32, 20.0),
                                             (512, 16, 10.0), (128, 24, 3.0)])
def test_wtowers_vs_oracle(rg, ctx, sim, oracle, wproj_data, sub, margin, winc):
    obs, u, v, w, vis = wproj_data
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    wkt = sim.generate_wkernel(th, np.arange(-winc / 2 - 1, winc / 2 + 1.5, 1.0))
    g = np.zeros((n, n), np.complex128)
    ctx.grid_wtowers(g, n, th, V(rg, u, v, w, vis), wkt, sub, margin, winc)
    ref, counts = oracle.grid_wtowers(n, th, u, v, w, vis, wkt, sub, margin, winc, return_counts=True)
    assert rel_rms(g, ref) < TOL
    st = ctx.last_stats()
    assert st["gridded"] == int((counts > 0).sum()) and st["dropped"] == int((counts == 0).sum())


def test_device_and_host_buffers_agree(rg, ctx, sim, wproj_data):
    torch = pytest.importorskip("torch")
    obs, u, v, w, vis = wproj_data
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    wkt = sim.generate_wkernel(th, np.arange(-6, 7, 1.0))
    g_host = np.zeros((n, n), np.complex128)
    ctx.grid_wtowers(g_host, n, th, V(rg, u, v, w, vis), wkt, 128, 16, 10.0)
    dev = torch.device("cuda", 0)
    t = [torch.from_numpy(a).to(dev) for a in (u, v, w, vis)]
    g_dev = torch.zeros((n, n), dtype=torch.complex128, device=dev)
    ctx.grid_wtowers(g_dev, n, th, V(rg, *t), wkt, 128, 16, 10.0,
                     wkern_data=torch.from_numpy(wkt.data).to(dev))
    torch.cuda.synchronize()
    assert rel_rms(g_dev.cpu().numpy(), g_host) < 1e-6


def test_accumulate_and_overwrite(rg, ctx, sim, wproj_data):
    obs, u, v, w, vis = wproj_data
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    wk = sim.wkernel_for(w, th, 10.0)
    once = np.zeros((n, n), np.complex128)
    ctx.grid_wprojection(once, n, th, V(rg, u, v, w, vis), wk)
    twice = once.copy()
    ctx.grid_wprojection(twice, n, th, V(rg, u, v, w, vis), wk)  # accumulates
    assert rel_rms(twice, 2 * once) < 1e-6
    junk = np.full((n, n), 7.0 + 1j)
    ctx.grid_wprojection(junk, n, th, V(rg, u, v, w, vis), wk, flags=rg.RG_GRID_OVERWRITE)
    assert rel_rms(junk, once) < 1e-6


def test_empty_input(rg, ctx, sim):
    wkt = sim.generate_wkernel(0.1, np.arange(-6, 7, 1.0))
    e = np.zeros(0)
    g = np.full((256, 256), 1.0 + 0j)
    ctx.grid_wtowers(g, 256, 0.1, V(rg, e, e, e, e.astype(np.complex128)), wkt, 128, 16, 10.0)
    assert np.all(g == 1.0)
    ctx.grid_wprojection(g, 256, 0.1, V(rg, e, e, e, e.astype(np.complex128)), wkt,
                         flags=rg.RG_GRID_OVERWRITE)
    assert np.all(g == 0.0)


def test_single_visibility_ragged(rg, ctx, sim, oracle):
    """One visibility, and counts that are not multiples of any batch size."""
    th, n = 0.1, 256
    wkt = sim.generate_wkernel(th, np.arange(-6, 7, 1.0))
    rng = np.random.default_rng(4)
    for count in (1, 2, 255, 257, 1025):
        u = rng.uniform(-1000, 1000, count)
        v = rng.uniform(-1000, 1000, count)
        w = rng.uniform(-40, 40, count)
        vis = rng.normal(size=count) + 1j * rng.normal(size=count)
        g = np.zeros((n, n), np.complex128)
        ctx.grid_wtowers(g, n, th, V(rg, u, v, w, vis), wkt, 128, 16, 10.0)
        ref = oracle.grid_wtowers(n, th, u, v, w, vis, wkt, 128, 16, 10.0)
        assert rel_rms(g, ref) < TOL


def test_wtowers_linearity_full_size(rg, ctx, sim):
    """Size-independent property at the benchmark size: G(a V1 + V2) = a G(V1) + G(V2)."""
    obs = sim.wtowers_plain()
    u, v, w, vis = obs.flat()
    wkt = sim.generate_wkernel(0.1, np.arange(-5, 6, 1.0))
    rng = np.random.default_rng(0)
    v2 = rng.normal(size=len(u)) + 1j * rng.normal(size=len(u))
    a = 0.37 - 1.1j

    def grid(x):
        g = np.zeros((2048, 2048), np.complex128)
        ctx.grid_wtowers(g, 2048, 0.1, V(rg, u, v, w, x), wkt, 512, 16, 10.0)
        return g

    g1, g2, g12 = grid(vis), grid(v2), grid(a * vis + v2)
    assert rel_rms(g12, a * g1 + g2) < 1e-5
    assert ctx.last_stats()["gridded"] == len(u)


def test_weight_hermitian_shift_image_exact(rg, ctx, oracle, wproj_data, golden):
    obs, u, v, w, vis = wproj_data
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    out = ctx.weight(n, th, V(rg, u, v, w, vis))
    assert np.array_equal(out, oracle.weight(n, th, u, v, vis))
    g = golden["grid_wprojection"]
    assert np.array_equal(ctx.make_hermitian(g.copy()), golden["hermitian"])
    assert np.array_equal(ctx.fft_shift(g.copy()), golden["shifted"])
    img = ctx.image_from_grid(g.copy())
    assert rel_rms(img, oracle.image_from_grid(g)) < 1e-13


def test_wtowers_subgrid_1024(rg, ctx, sim, oracle):
    """The largest sub-grid (1024: 128 column strips, two mask words per half)
    on a 1024-cell grid, against the oracle."""
    obs = sim.wtowers_plain(seed=6, n_st=40, n_dump=8, n_chan=2, lam=10240.0)
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    u, v, w, vis = obs.flat()
    wkt = sim.generate_wkernel(th, np.arange(-6, 7, 1.0))
    g = np.zeros((n, n), np.complex128)
    ctx.grid_wtowers(g, n, th, V(rg, u, v, w, vis), wkt, 1024, 32, 10.0)
    ref = oracle.grid_wtowers(n, th, u, v, w, vis, wkt, 1024, 32, 10.0)
    assert rel_rms(g, ref) < TOL


def test_wtowers_full_benchmark_workload(rg, ctx, sim, oracle):
    """Parity at the benchmark's full size (2048^2, S 512, margin 16, winc 10,
    2,088,960 visibilities, 32x oversampled 16-tap kernels) against the CPU
    restatement of grid.c (about 20 s on the host)."""
    obs = sim.wtowers_plain(seed=1)
    u, v, w, vis = obs.flat()
    wk = sim.generate_wkernel(0.1, np.arange(-5, 6, 1.0), 16, 32)
    g = np.zeros((2048, 2048), np.complex128)
    ctx.grid_wtowers(g, 2048, 0.1, V(rg, u, v, w, vis), wk, 512, 16, 10.0)
    ref = oracle.grid_wtowers(2048, 0.1, u, v, w, vis, wk, 512, 16, 10.0)
    assert rel_rms(g, ref) < TOL
    st = ctx.last_stats()
    assert st["gridded"] + st["dropped"] == len(u) and st["active_subgrids"] > 900


def test_wtowers_tower_shares_sum_to_the_whole(rg, ctx, sim, oracle, wproj_data):
    """One observation's towers split three ways (rg_wtowers_tower_loads +
    rg_wtowers_partition): the device census equals the oracle's, and the
    three shares gridded by rg_grid_wtowers_part sum to rg_grid_wtowers'
    grid and to the oracle's."""
    obs, u, v, w, vis = wproj_data
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    S, M, winc = 128, 16, 10.0
    wkt = sim.generate_wkernel(th, np.arange(-6, 7, 1.0))
    Vs = V(rg, u, v, w, vis)
    nv, nf = ctx.tower_loads(n, th, Vs, S, M, winc)
    onv, onf = oracle.wtowers_census(n, th, u, v, w, S, M, winc)
    assert np.array_equal(nv, onv) and np.array_equal(nf, onf)
    parts = rg.partition_towers(nv, nf, 3)
    total = np.zeros((n, n), np.complex128)
    gridded = 0
    for p in range(3):
        g = np.zeros((n, n), np.complex128)
        ctx.grid_wtowers_part(g, n, th, Vs, wkt, S, M, winc, parts, p)
        gridded += ctx.last_stats()["gridded"]
        total += g
    whole = np.zeros((n, n), np.complex128)
    ctx.grid_wtowers(whole, n, th, Vs, wkt, S, M, winc)
    assert gridded == ctx.last_stats()["gridded"] == int(nv.sum())
    assert rel_rms(total, whole) < 1e-6
    assert rel_rms(total, oracle.grid_wtowers(n, th, u, v, w, vis, wkt, S, M, winc)) < TOL


def test_grid_simple_matches_oracle(rg, ctx, oracle, wproj_data):
    """Nearest-cell gridding (grid_simple, src/reference/grid.c:83-99) with
    FP64 atomics against the sequential oracle; accumulate and overwrite; a
    visibility off the grid is an error that leaves the grid untouched."""
    obs, u, v, w, vis = wproj_data
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    ref = oracle.grid_simple(n, th, u, v, vis)
    g = np.full((n, n), 2.0 + 0j)
    ctx.grid_simple(g, n, th, V(rg, u, v, w, vis), flags=rg.RG_GRID_OVERWRITE)
    assert rel_rms(g, ref) < 1e-14
    ctx.grid_simple(g, n, th, V(rg, u, v, w, vis))
    assert rel_rms(g, 2 * ref) < 1e-14
    keep = g.copy()
    far = u.copy()
    far[3] = 1e9
    with pytest.raises(rg.RGError):
        ctx.grid_simple(g, n, th, V(rg, far, v, w, vis))
    assert np.array_equal(g, keep)


def test_wtowers_grid_size_not_a_power_of_two(rg, ctx, sim, oracle):
    """grid.out's grid size floor(lambda * theta) is rarely a power of two:
    W-towers at N = 2500 (6 x 6 towers of 496 cells, the last ones clipped at
    the grid edge) against the oracle."""
    obs = sim.wtowers_plain(seed=7, n_st=48, n_dump=8, n_chan=2, lam=25000.0)
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    assert n == 2500
    u, v, w, vis = obs.flat()
    wkt = sim.generate_wkernel(th, np.arange(-6, 7, 1.0), 16, 16)
    g = np.zeros((n, n), np.complex128)
    ctx.grid_wtowers(g, n, th, V(rg, u, v, w, vis), wkt, 512, 16, 10.0)
    ref = oracle.grid_wtowers(n, th, u, v, w, vis, wkt, 512, 16, 10.0)
    assert rel_rms(g, ref) < TOL


def test_wtowers_equals_wprojection_for_small_w_on_gpu(rg, ctx, sim):
    """Known answer on the device: with every |w| < winc/2 all visibilities
    sit on floor 0, so the CUDA W-towers pass must reproduce the CUDA
    W-projection grid up to the FP32 sub-grid FFT round trip (margin larger
    than the kernel support, so no footprint wraps)."""
    obs = sim.wproj_plain(seed=7, n_dump=8)
    u, v, w, vis = obs.flat()
    w = w * (4.0 / np.abs(w).max())
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    wkt = sim.generate_wkernel(th, np.arange(-5, 6, 1.0))
    a = np.zeros((n, n), np.complex128)
    ctx.grid_wprojection(a, n, th, V(rg, u, v, w, vis), wkt)
    b = np.zeros((n, n), np.complex128)
    ctx.grid_wtowers(b, n, th, V(rg, u, v, w, vis), wkt, 128, 18, 10.0)
    assert ctx.last_stats()["floors"] == 1
    assert rel_rms(b, a) < TOL


def test_point_source_at_phase_centre_image_on_gpu(rg, ctx, sim):
    """Known answer: a unit source at the phase centre gives constant
    visibilities; the dirty image from the CUDA W-towers grid (hermitian,
    shift, FFT, shift) peaks at the centre pixel."""
    obs = sim.wproj_plain(seed=3, n_dump=16)
    u, v, w, _ = obs.flat()
    vis = np.ones(len(u), np.complex128)
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    wkt = sim.generate_wkernel(th, np.arange(-6, 7, 1.0))
    g = np.zeros((n, n), np.complex128)
    ctx.grid_wtowers(g, n, th, V(rg, u, v, w, vis), wkt, 128, 16, 10.0)
    img = ctx.image_from_grid(g)
    assert np.unravel_index(np.argmax(img), img.shape) == (n // 2, n // 2)
    assert img[n // 2, n // 2] > 0


@pytest.mark.parametrize("ksize,ov,sub,margin", [(8, 8, 256, 16), (32, 4, 256, 32)])
def test_wtowers_kernel_sizes_vs_oracle(rg, ctx, sim, oracle, wproj_data, ksize, ov, sub, margin):
    """W-towers with 8- and 32-tap kernels (the gridder's other footprint
    sizes) against the oracle, visibility counts included."""
    obs, u, v, w, vis = wproj_data
    n, th = obs.meta["grid_size"], obs.meta["theta"]
    wkt = sim.generate_wkernel(th, np.arange(-6.0, 7.0, 1.0), ksize, ov)
    g = np.zeros((n, n), np.complex128)
    ctx.grid_wtowers(g, n, th, V(rg, u, v, w, vis), wkt, sub, margin, 10.0)
    ref, counts = oracle.grid_wtowers(n, th, u, v, w, vis, wkt, sub, margin, 10.0, return_counts=True)
    assert rel_rms(g, ref) < TOL
    st = ctx.last_stats()
    assert st["gridded"] == int(counts.sum()) and st["gridded"] + st["dropped"] == len(u)


def test_wtowers_cuts_on_the_boundaries(rg, ctx, sim, oracle):
    """Visibilities exactly on the half-open tower cuts in u and v and on the
    w-floor cuts, and one ulp either side, formed in FP64 as the reference
    forms them (grid.c:425-458 for the towers, :244-254 for the floors): the
    device bins every one as the oracle does."""
    n, th, S, M, winc = 512, 0.1, 128, 16, 10.0
    chunk = S - M
    nchunk = n // chunk + 1
    cuts = np.array([(chunk * c - n // 2 - 0.5) / th for c in range(nchunk)])
    fcuts = np.array([(wp - 0.5) * winc for wp in range(-4, 5)])
    rng = np.random.default_rng(11)
    m = 4000

    def near(x):  # on the value, or one ulp below or above
        step = rng.integers(-1, 2, len(x))
        return np.where(step < 0, np.nextafter(x, -np.inf), np.where(step > 0, np.nextafter(x, np.inf), x))

    u = near(cuts[rng.integers(1, nchunk, m)])
    v = near(cuts[rng.integers(1, nchunk, m)])
    w = near(fcuts[rng.integers(0, len(fcuts), m)])
    # half of them off the cuts in one axis only
    free = rng.random(m) < 0.5
    u[free] = rng.uniform(-200, 200, free.sum()) / th
    vis = rng.normal(size=m) + 1j * rng.normal(size=m)
    wkt = sim.generate_wkernel(th, np.arange(-6.0, 7.0, 1.0))
    g = np.zeros((n, n), np.complex128)
    ctx.grid_wtowers(g, n, th, V(rg, u, v, w, vis), wkt, S, M, winc)
    ref, counts = oracle.grid_wtowers(n, th, u, v, w, vis, wkt, S, M, winc, return_counts=True)
    assert rel_rms(g, ref) < TOL
    st = ctx.last_stats()
    assert st["gridded"] == int(counts.sum()) and st["gridded"] + st["dropped"] == m
