"""The W-stacking predict oracle (the C restatement of the reference's
wstack_predict, src/wstack/predict.cpp:396-562) against the direct sum over
the quantised sky it approximates (predict_visibility_quantized_vec,
src/wstack/predict.cpp:89-129), with the project's PSWF separable kernels
(simulate.sepkern_pswf).  CPU only.

The reference's own predict cannot be built here (it needs libhdf5, FFTW's
guru interface and its HDF5 kernel files), so its parity is pinned by this
property — a predict equal to the DFT of the same sky within the kernel's
accuracy — and the GPU predict is checked against this oracle."""
import numpy as np
import pytest


def case(sim, seed=0, theta=0.1, lam=2560.0, nv=2000, npts=10, dw=50.0, suv=8, sw=6):
    import oracle
    rng = np.random.default_rng(seed)
    n = int(np.floor(theta * lam))
    du = 1.0 / (2.0 * theta)
    pts = rng.uniform(-0.45 * theta, 0.45 * theta, (npts, 2))
    planes = oracle.wstack_planes(theta, lam, dw, sw)
    lim_u = (n - suv // 2 - 2) * du
    wl = (planes // 2 - sw // 2 - 1) * dw
    u, v = rng.uniform(-lim_u, lim_u, (2, nv))
    w = rng.uniform(-wl, wl, nv)
    cu, ku = sim.sepkern_pswf(suv, 1024, 0.25, corr_oversampling=1024)
    cw, kw = sim.sepkern_pswf(sw, 1024, 0.25, corr_oversampling=1024)
    return dict(theta=theta, lam=lam, points=pts, u=u, v=v, w=w, du=du, dw=dw, x0=0.25, conv_uv=cu, conv_w=cw,
                corr_lm=ku, corr_n=kw)


def test_oracle_predict_matches_quantised_dft(sim, oracle):
    c = case(sim)
    got = oracle.wstack_predict(c["theta"], c["lam"], c["points"], c["u"], c["v"], c["w"], c["du"], c["dw"],
                                c["x0"], c["conv_uv"], c["conv_w"], c["corr_lm"], c["corr_n"])
    ref = oracle.predict_dft_quantized(c["theta"], c["lam"], c["points"], c["u"], c["v"], c["w"])
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 2e-3


def test_oracle_predict_is_linear_in_the_sky(sim, oracle):
    """Two source lists predicted together equal the sum of each alone."""
    c = case(sim, seed=1, npts=6)
    args = (c["u"], c["v"], c["w"], c["du"], c["dw"], c["x0"], c["conv_uv"], c["conv_w"], c["corr_lm"], c["corr_n"])
    a = oracle.wstack_predict(c["theta"], c["lam"], c["points"][:3], *args)
    b = oracle.wstack_predict(c["theta"], c["lam"], c["points"][3:], *args)
    ab = oracle.wstack_predict(c["theta"], c["lam"], c["points"], *args)
    assert np.linalg.norm(ab - (a + b)) / np.linalg.norm(ab) < 1e-12
