"""W-stacking predict on the device (rg_wstack_predict) against the oracle's
restatement of the reference's wstack_predict (src/wstack/predict.cpp:
396-562) with the same kernels: FP64 on both sides, so the visibilities
agree to rounding; and against the direct sum over the quantised sky."""
import numpy as np
import pytest

from test_wstack_oracle import case

pytestmark = pytest.mark.gpu


def _run(ctx, c, **kw):
    return ctx.wstack_predict(c["theta"], c["lam"], c["points"], c["u"], c["v"], c["w"], c["du"], c["dw"], c["x0"],
                              c["conv_uv"], c["conv_w"], c["corr_lm"], c["corr_n"], **kw)


@pytest.mark.parametrize("lam,nv,npts,sw", [(2560.0, 3000, 10, 6), (5120.0, 20000, 25, 4), (2500.0, 777, 3, 6)])
def test_predict_matches_oracle(ctx, sim, oracle, lam, nv, npts, sw):
    c = case(sim, seed=int(lam) + nv, lam=lam, nv=nv, npts=npts, sw=sw)
    got = _run(ctx, c)
    ref = oracle.wstack_predict(c["theta"], c["lam"], c["points"], c["u"], c["v"], c["w"], c["du"], c["dw"],
                                c["x0"], c["conv_uv"], c["conv_w"], c["corr_lm"], c["corr_n"])
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-11
    dft = oracle.predict_dft_quantized(c["theta"], c["lam"], c["points"], c["u"], c["v"], c["w"])
    assert np.linalg.norm(got - dft) / np.linalg.norm(dft) < 2e-3


def test_predict_device_buffers_and_errors(rg, ctx, sim):
    torch = pytest.importorskip("torch")
    c = case(sim, seed=5, nv=500)
    host = _run(ctx, c)
    dev = torch.device("cuda", 0)
    d = dict(c)
    for k in ("u", "v", "w"):
        d[k] = torch.from_numpy(c[k]).to(dev)
    out = torch.zeros(500, dtype=torch.complex128, device=dev)
    _run(ctx, d, out=out)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), host)
    bad = dict(c)
    bad["u"] = c["u"] * 10.0  # taps far outside the stack
    with pytest.raises(rg.RGError):
        _run(ctx, bad)
    bad = dict(c)
    bad["points"] = np.array([[0.9 * c["theta"], 0.0]])  # outside the image
    with pytest.raises(rg.RGError):
        _run(ctx, bad)
