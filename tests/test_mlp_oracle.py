"""The CPU oracle of the learned w-kernel network: analytic gradients against
central finite differences (FP64), and the feature definition's ranges."""
import numpy as np

from oracle import mlp_oracle as MO


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    P = MO.init_params(1)
    for k in P:
        P[k] = P[k] + 0.01 * rng.normal(size=P[k].shape) * (k != "W1")
    B = 16
    f = MO.features(rng.uniform(-2000, 2000, B), rng.uniform(0, 1, B), rng.uniform(0, 1, B),
                    rng.integers(0, 16, B), rng.integers(0, 16, B), 16, 2000.0)
    t = rng.normal(size=(B, 2))
    _, g = MO.loss_and_grads(P, f, t)
    flat, gflat = MO.pack(P), MO.pack(g)
    live = [i for i in range(len(flat)) if not (i < 32 * 128 and i // 128 >= MO.NFEAT)]
    for i in rng.choice(live, 40, replace=False):
        e = 1e-6
        fp, fm = flat.copy(), flat.copy()
        fp[i] += e
        fm[i] -= e
        num = (MO.loss_and_grads(MO.unpack(fp), f, t)[0] - MO.loss_and_grads(MO.unpack(fm), f, t)[0]) / (2 * e)
        assert abs(num - gflat[i]) <= 1e-6 + 1e-5 * abs(num)


def test_features_bounded():
    rng = np.random.default_rng(1)
    f = MO.features(rng.uniform(-2000, 2000, 500), rng.uniform(0, 1, 500), rng.uniform(0, 1, 500),
                    rng.integers(0, 16, 500), rng.integers(0, 16, 500), 16, 2000.0)
    assert f.shape == (500, 32)
    assert np.all(np.abs(f[:, :MO.NFEAT]) <= 1.13) and np.all(f[:, MO.NFEAT:] == 0)
