"""Generate the golden fixtures in this directory from the reference itself.

Run in a checkout where the reference sources are present (the oracle Makefile
compiles src/reference/grid.c from them into oracle/_ref/libref_grid.so):

    python tests/golden/make_golden.py

Each fixture holds seeded inputs (flat visibilities, the hierarchical layout
they came from, a w-kernel table) and the reference's own outputs for them:
grid_wprojection, grid_wtowers, weight, make_hermitian and fft_shift.  Sizes
are kept small so the files stay a few hundred KB.
"""
import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

import oracle  # noqa: E402

sim = importlib.import_module("radio-gridders_b200.simulate")


def small_obs(seed, n_ant, n_dump, theta, lam, ksize, w_limit):
    rng = np.random.default_rng(seed)
    enu = sim.uniform_disc(rng, n_ant, 10_000.0)
    lat, dec = 10.0, -30.0
    ha = np.linspace(-2.0, 2.0, n_dump)
    freqs = np.array([1.4e9, 1.401e9])
    n_grid = int(theta * lam)
    limit = (n_grid / 2 - ksize / 2 - 2) / theta
    scale = sim.fit_scale(enu, lat, dec, ha, freqs, limit)
    enu = enu * scale
    xyz = sim.enu_to_xyz(enu, np.radians(lat))
    a1, a2 = np.triu_indices(n_ant, k=1)
    uvw = sim.baseline_uvw(xyz[a2] - xyz[a1], ha * np.pi / 12, np.radians(dec))
    wmax = np.abs(uvw[:, :, 2]).max() * freqs.max() / sim.C_LIGHT
    src = sim.random_sources(rng, 5, theta, "uniform")
    return sim.observe(enu, lat, dec, ha, freqs, src, w_scale=w_limit / wmax)


def main():
    oracle.build(reference=True)
    theta, lam, ksize, ov = 0.1, 1280.0, 8, 4
    n = int(theta * lam)
    obs = small_obs(11, 12, 24, theta, lam, ksize, w_limit=38.0)
    u, v, w, vis = obs.flat()
    wk = sim.generate_wkernel(theta, np.arange(-50.0, 51.0, 10.0), ksize, ov)
    wkt = sim.generate_wkernel(theta, np.arange(-5.0, 6.0, 1.0), ksize, ov)
    g_wproj = oracle.ref_grid_wprojection(n, theta, obs, wk)
    sub, margin, winc = 64, 16, 10.0
    mask = oracle.reference_safe_baselines(obs, n, theta, sub, margin, ksize, ov)
    assert mask.all(), "fixture must not contain footprints outside the reference's buffer"
    g_tow = oracle.ref_grid_wtowers(n, theta, obs, wkt, sub, margin, winc)
    vis_w = oracle.ref_weight(n, theta, obs)
    herm = oracle.ref_make_hermitian(g_wproj)
    shift = oracle.ref_fft_shift(g_wproj)
    np.savez_compressed(
        os.path.join(HERE, "small_128.npz"),
        theta=theta, grid_size=n, subgrid=sub, margin=margin, winc=winc,
        u=u, v=v, w=w, vis=vis,
        uvw=obs.uvw, freq=obs.freq, time=obs.time, vis_h=obs.vis,
        antenna1=obs.antenna1, antenna2=obs.antenna2,
        wk_data=wk.data, wk_wmin=wk.w_min, wk_wstep=wk.w_step,
        wkt_data=wkt.data, wkt_wmin=wkt.w_min, wkt_wstep=wkt.w_step,
        grid_wprojection=g_wproj, grid_wtowers=g_tow, weighted_vis=vis_w,
        hermitian=herm, shifted=shift)
    print("wrote small_128.npz:", len(u), "visibilities")


if __name__ == "__main__":
    main()
