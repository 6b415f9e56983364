"""Learned w-kernel: the CUDA forward/backward kernels against the FP64 CPU
oracle (oracle/mlp_oracle.py), training on the GPU, the learned-tap gridder,
and what the trained network gains over the oversampled table."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def MO():
    return importlib.import_module("oracle.mlp_oracle")


@pytest.fixture(scope="module")
def learned():
    return importlib.import_module("radio-gridders_b200.learned")


def _random_batch(rng, n, ksize=16, wmax=2000.0):
    w = rng.uniform(-wmax, wmax, n)
    du, dv = rng.uniform(0, 1, n), rng.uniform(0, 1, n)
    tx, ty = rng.integers(0, ksize, n).astype(float), rng.integers(0, ksize, n).astype(float)
    return w, du, dv, tx, ty


def test_forward_matches_oracle(rg, ctx, MO):
    rng = np.random.default_rng(0)
    mlp = rg.LearnedKernel(ctx, 16, 2000.0, 0.05)
    mlp.set_params(MO.pack(MO.init_params(3)).astype(np.float32))
    P = MO.unpack(mlp.get_params().astype(np.float64))
    b = _random_batch(rng, 1000)
    y, _ = MO.forward(P, MO.features(*b, 16, 2000.0))
    ref = (y[:, 0] + 1j * y[:, 1]) * 0.05
    got = mlp.eval(rg.LearnedKernel.samples(*b))
    # BF16-rounded weights, FP16 activations (tcgen05), FP32 accumulation
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 2e-2


def test_gradient_matches_oracle(rg, ctx, MO):
    rng = np.random.default_rng(1)
    mlp = rg.LearnedKernel(ctx, 16, 2000.0, 0.05)
    mlp.set_params(MO.pack(MO.init_params(4)).astype(np.float32))
    P = MO.unpack(mlp.get_params().astype(np.float64))
    b = _random_batch(rng, 700)  # not a multiple of the 64-sample tile
    tg = (rng.normal(size=700) + 1j * rng.normal(size=700)) * 0.05
    loss, g = mlp.gradient(rg.LearnedKernel.samples(*b), rg.LearnedKernel.targets(tg))
    ref_loss, ref_g = MO.loss_and_grads(P, MO.features(*b, 16, 2000.0),
                                        np.stack([tg.real, tg.imag], -1) / 0.05)
    assert abs(loss - ref_loss) / ref_loss < 2e-2
    gu = MO.unpack(g.astype(np.float64))
    for name, _ in MO.SIZES:
        assert np.linalg.norm(gu[name] - ref_g[name]) / np.linalg.norm(ref_g[name]) < 5e-2, name


def test_training_beats_the_table(rg, ctx, sim, learned):
    """Trained on the GPU, the network's taps at continuous (w, du, dv) are more
    accurate than nearest-plane / nearest-sub-cell lookup in an 8x oversampled
    table with planes every 10 lambda — from 37.5k parameters instead of a
    ~52 MB table."""
    mlp, losses = learned.train(ctx, n_triples=2048, steps=12000, batch=16384, lr_max=4e-3)
    assert losses[-1] < 0.05 * losses[0]
    err, held = learned.tap_error(mlp, n_triples=128)
    wk = sim.generate_wkernel(0.1, np.arange(-2010.0, 2011.0, 10.0), 16, 8)
    table = learned.table_tap_error(wk, held)
    assert err < table, (err, table)


def test_learned_gridder_matches_cpu_evaluation(rg, ctx, MO):
    """The learned-tap W-projection gridder against a CPU gridding with the
    oracle network (same parameters) at each visibility's exact sub-cell
    offset: footprint at floor(theta u) - K/2, grid += vis * conj(tap)."""
    rng = np.random.default_rng(5)
    mlp = rg.LearnedKernel(ctx, 16, 2000.0, 0.05)
    mlp.set_params(MO.pack(MO.init_params(6)).astype(np.float32) * 0.5)
    P = MO.unpack(mlp.get_params().astype(np.float64))
    n, th, nv, K = 128, 0.1, 200, 16
    u, v = rng.uniform(-500, 500, nv), rng.uniform(-500, 500, nv)
    w = rng.uniform(-1500, 1500, nv)
    vis = rng.normal(size=nv) + 1j * rng.normal(size=nv)
    g = np.zeros((n, n), np.complex128)
    rg.grid_wprojection_learned(ctx, mlp, g, n, th, rg.Visibilities(u, v, w, vis))
    ref = np.zeros((n, n), np.complex128)
    tyy, txx = np.meshgrid(np.arange(K), np.arange(K), indexing="ij")
    for i in range(nv):
        x, y = th * u[i], th * v[i]
        cx, cy = np.floor(x), np.floor(y)
        f = MO.features(np.full(K * K, w[i]), np.full(K * K, x - cx), np.full(K * K, y - cy),
                        txx.ravel(), tyy.ravel(), K, 2000.0)
        yv, _ = MO.forward(P, f)
        tap = ((yv[:, 0] + 1j * yv[:, 1]) * 0.05).reshape(K, K)
        r0, c0 = int(cy) - K // 2 + n // 2, int(cx) - K // 2 + n // 2
        ref[r0:r0 + K, c0:c0 + K] += vis[i] * np.conj(tap)
    assert np.linalg.norm(g - ref) / np.linalg.norm(ref) < 3e-2


def test_learned_wtowers_equals_table_wtowers_on_the_lattice(rg, ctx, MO):
    """W-towers with learned taps against W-towers with a table made from the
    same network.  With theta = 1/8, integer u, v and w on the table planes,
    every visibility's offsets fall exactly on the 8x oversampling lattice, so
    the table's nearest sub-cell/plane lookup and the network's continuous
    evaluation see the same inputs and the two grids agree to the gridders'
    atomic-ordering noise — the learned path is the table pipeline with only
    the taps replaced."""
    from types import SimpleNamespace
    rng = np.random.default_rng(11)
    K, ov, th, n, S, M, winc = 8, 8, 0.125, 256, 128, 16, 5.0
    planes = np.arange(-2.0, 3.0)
    mlp = rg.LearnedKernel(ctx, K, 4.0, 0.05)
    mlp.set_params(MO.pack(MO.init_params(12)).astype(np.float32) * 0.5)
    # table[p][yf][xf][ty][tx] = network(w_p, xf/ov, yf/ov, tx, ty)
    P_, YF, XF, TY, TX = np.meshgrid(np.arange(5), np.arange(ov), np.arange(ov), np.arange(K), np.arange(K),
                                      indexing="ij")
    taps = mlp.eval(rg.LearnedKernel.samples(planes[P_].ravel(), XF.ravel() / ov, YF.ravel() / ov,
                                             TX.ravel(), TY.ravel()))
    table = SimpleNamespace(data=taps.reshape(5, ov, ov, K, K), w_min=-2.0, w_step=1.0)
    nv = 3000
    u = rng.integers(-900, 900, nv).astype(np.float64)
    v = rng.integers(-900, 900, nv).astype(np.float64)
    w = rng.integers(-8, 9, nv) * winc + rng.integers(-2, 3, nv)
    vis = rng.normal(size=nv) + 1j * rng.normal(size=nv)
    V = rg.Visibilities(u, v, w.astype(np.float64), vis)
    g_table = np.zeros((n, n), np.complex128)
    ctx.grid_wtowers(g_table, n, th, V, table, S, M, winc)
    g_learned = np.zeros((n, n), np.complex128)
    rg.grid_wtowers_learned(ctx, mlp, g_learned, n, th, V, S, M, winc)
    assert np.abs(g_table).max() > 0
    assert np.linalg.norm(g_learned - g_table) / np.linalg.norm(g_table) < 1e-5
    with pytest.raises(rg.RGError):  # network w range narrower than winc / 2
        rg.grid_wtowers_learned(ctx, mlp, g_learned, n, th, V, S, M, 10.0)


def test_bounded_wait_times_out_and_context_survives(rg, ctx):
    """The tensor-core kernels' waits are bounded: a wait on an mbarrier that
    nothing arrives on gives up, the error reaches the host as RG_ERR_CUDA
    ("timed out"), and the context keeps working afterwards."""
    with pytest.raises(rg.RGError) as e:
        ctx.selftest_wait_timeout()
    assert e.value.status == 2 and "timed out" in str(e.value)
    mlp = rg.LearnedKernel(ctx, 16, 10.0, 0.05)
    taps = mlp.eval(rg.LearnedKernel.samples(np.zeros(4), np.full(4, 0.5), np.full(4, 0.5), np.arange(4.0),
                                            np.arange(4.0)))
    assert np.all(np.isfinite(taps))
