"""Seeded synthetic observations and the project's own w-kernel generator.

The reference reads crocodile HDF5 datasets (src/common/hdf5.c:64-96 for
visibilities, :513-550 for w-kernels); those datasets are Git-LFS pointers in
the reference tree and no public dataset is named for the benchmark, so every
workload here is generated from a seed:

* uvw from Earth-rotation synthesis (Thompson, Moran & Swenson, eq. 4.1) of a
  station layout at a site latitude, hour angles and frequencies;
* visibilities from point sources, V = sum_s A_s exp(-2 pi i (u l + v m + w (n-1)))
  (the convention of the reference's predict_visibility,
  src/wstack/predict.cpp:27-45);
* w-kernels as the Fourier transform of a PSWF-tapered w-screen, oversampled,
  in the table layout the reference gridder indexes
  (kern_by_w[plane].data[(yf*ov + xf)*S*S + y*S + x], src/reference/grid.c:53-56).

All quantities are float64.  The data layout is the reference's
"hierarchical" one (baseline -> time -> frequency, uvw in metres per
(baseline, time)) and its flattened form (u, v, w in wavelengths), as produced
by flatten_visibilities_CUDA (src/common/hdf5.c:827-872, without its
off-by-one write).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

C_LIGHT = 299792458.0  # src/reference/grid.c:19


# ----------------------------------------------------------------------------
# Prolate spheroidal wave function psi_0(c, x) on [-1, 1]
# ----------------------------------------------------------------------------

def pswf0(c: float, x: np.ndarray, nterms: int = 0) -> np.ndarray:
    """Zeroth-order angular prolate spheroidal function, normalised psi(0) = 1.

    Method: expansion in normalised Legendre polynomials; the expansion
    coefficients are the eigenvector of the symmetric tridiagonal matrix of
    the differential operator (1-x^2) d2/dx2 - 2x d/dx - c^2 x^2 restricted to
    even degrees (Bouwkamp 1947; Xiao, Rokhlin & Yarvin 2001).  Tests compare
    against scipy.special.pro_ang1.
    """
    x = np.asarray(x, dtype=np.float64)
    if nterms <= 0:
        nterms = int(2 * c + 40)
    ks = np.arange(0, 2 * nterms, 2)  # even degrees
    # matrix elements of c^2 x^2 in normalised Legendre basis P_k*sqrt(k+1/2)
    diag = ks * (ks + 1) + c * c * (2 * ks * (ks + 1) - 1) / ((2 * ks + 3) * (2 * ks - 1))
    kk = ks[:-1]
    off = c * c * (kk + 1) * (kk + 2) / ((2 * kk + 3) * np.sqrt((2 * kk + 1) * (2 * kk + 5)))
    mat = np.diag(diag) + np.diag(off, 1) + np.diag(off, -1)
    evals, evecs = np.linalg.eigh(mat)
    coef = evecs[:, np.argmin(evals)]
    # evaluate sum coef_j sqrt(k_j + 1/2) P_{k_j}(x) by the Legendre recurrence
    flat = x.ravel()
    p_prev = np.ones_like(flat)
    p_cur = flat.copy()
    out = coef[0] * math.sqrt(0.5) * p_prev
    at0 = coef[0] * math.sqrt(0.5)
    p0_prev, p0_cur = 1.0, 0.0
    deg = 1
    for j in range(1, len(ks)):
        while deg < ks[j]:
            p_next = ((2 * deg + 1) * flat * p_cur - deg * p_prev) / (deg + 1)
            p0_next = ((2 * deg + 1) * 0.0 * p0_cur - deg * p0_prev) / (deg + 1)
            p_prev, p_cur = p_cur, p_next
            p0_prev, p0_cur = p0_cur, p0_next
            deg += 1
        out = out + coef[j] * math.sqrt(ks[j] + 0.5) * p_cur
        at0 += coef[j] * math.sqrt(ks[j] + 0.5) * p0_cur
    return (out / at0).reshape(x.shape)


# ----------------------------------------------------------------------------
# w-kernel generator
# ----------------------------------------------------------------------------

@dataclasses.dataclass
class WKernel:
    """An oversampled w-kernel table (the reference's struct w_kernel_data,
    src/reference/grid.h:34-49, with planes evenly spaced from w_min)."""
    data: np.ndarray  # complex128 [planes, ov, ov, size, size]
    w_min: float
    w_step: float
    theta: float
    c: float

    @property
    def plane_count(self) -> int:
        return int(self.data.shape[0])

    @property
    def oversampling(self) -> int:
        return int(self.data.shape[1])

    @property
    def size(self) -> int:
        return int(self.data.shape[3])

    @property
    def w_max(self) -> float:
        return self.w_min + (self.plane_count - 1) * self.w_step


def screen_coords(theta: float, m_pix: int) -> np.ndarray:
    return theta * (np.arange(m_pix) - m_pix // 2) / m_pix


def w_screen(theta: float, w: float, c: float, m_pix: int) -> np.ndarray:
    """PSWF-tapered w-screen s_w(l, m) = A(l) A(m) exp(+2 pi i w (1 - n)).

    The sign makes conj(taps) undo the w-term of the visibility model in the
    image convention of the reference's CPU pipeline (hermitian, shift,
    FFT sign -1, shift: src/reference/main.c:258-294) and agrees with the
    W-towers Fresnel transfer pattern exp(+2 pi i winc (1 - n))
    (src/reference/grid.c:304-319).
    """
    lm = screen_coords(theta, m_pix)
    a = pswf0(c, 2.0 * lm / theta)
    l2 = lm[None, :] ** 2 + lm[:, None] ** 2
    one_minus_n = 1.0 - np.sqrt(1.0 - l2)
    return (a[None, :] * a[:, None]) * np.exp(2j * np.pi * w * one_minus_n)


def kernel_taps(theta: float, w: float, c: float, size: int,
                offsets_x: np.ndarray, offsets_y: np.ndarray, m_pix: int = 128) -> np.ndarray:
    """Continuous kernel K_w(p, q) at cell offsets p (x) and q (y), measured as
    (grid cell - visibility position):
        K(p, q) = 1/M^2 sum_ij s_w(l_i, m_j) exp(-2 pi i (p l_i + q m_j) / theta)
    Returns [len(offsets_y), len(offsets_x)] complex128.
    """
    lm = screen_coords(theta, m_pix)
    s = w_screen(theta, w, c, m_pix)  # [m (y), l (x)]
    ex = np.exp(-2j * np.pi * np.outer(offsets_x, lm) / theta)  # [px, i]
    ey = np.exp(-2j * np.pi * np.outer(offsets_y, lm) / theta)  # [qy, j]
    return (ey @ s @ ex.T) / (m_pix * m_pix)


def generate_wkernel(theta: float, w_planes: np.ndarray, size: int = 16,
                     oversampling: int = 8, c: float | None = None,
                     m_pix: int = 128) -> WKernel:
    """Oversampled table for evenly spaced w planes.

    tap[plane, yf, xf, ty, tx] = K_w(tx - size/2 - xf/ov, ty - size/2 - yf/ov),
    matching frac_coord's split of a position into cell + sub-cell index
    (src/reference/grid.c:37-57): the footprint starts size/2 cells left of the
    nearest cell and the sub-cell index xf means a shift of +xf/ov cells.
    """
    w_planes = np.asarray(w_planes, dtype=np.float64)
    if c is None:
        c = math.pi * (size - 2) / 2.0
    ov = oversampling
    taps = np.arange(size)
    data = np.empty((len(w_planes), ov, ov, size, size), dtype=np.complex128)
    # offsets for all sub-cell shifts at once: [ov*size]
    offs = (taps[None, :] - size // 2 - np.arange(ov)[:, None] / ov).ravel()
    for p, w in enumerate(w_planes):
        k = kernel_taps(theta, float(w), c, size, offs, offs, m_pix)  # [(yf,ty),(xf,tx)]
        data[p] = k.reshape(ov, size, ov, size).transpose(0, 2, 1, 3)
    w_step = float(w_planes[1] - w_planes[0]) if len(w_planes) > 1 else 1.0
    return WKernel(data=data, w_min=float(w_planes[0]), w_step=w_step, theta=theta, c=c)


def taper_1d(theta: float, n: int, c: float) -> np.ndarray:
    """Image-plane taper A(l) at the n pixels of an n-point image of width theta
    (pixel x at l = theta (x - n/2) / n), used for grid correction."""
    lm = theta * (np.arange(n) - n // 2) / n
    return pswf0(c, 2.0 * lm / theta)


# ----------------------------------------------------------------------------
# Observations
# ----------------------------------------------------------------------------

@dataclasses.dataclass
class Observation:
    """Hierarchical visibilities (reference struct vis_data, grid.h:7-30):
    uvw [bl, time, 3] metres, freq [bl, freq] Hz, vis [bl, time, freq]."""
    uvw: np.ndarray
    freq: np.ndarray
    time: np.ndarray
    vis: np.ndarray
    antenna1: np.ndarray
    antenna2: np.ndarray
    meta: dict

    @property
    def nvis(self) -> int:
        return int(self.vis.size)

    def flat(self):
        """(u, v, w, vis) in wavelengths, order baseline -> time -> frequency,
        computed as uvw * freq / c exactly as uvw_lambda (grid.c:21-24)."""
        f = self.freq[:, None, :]
        u = (self.uvw[:, :, 0:1] * f / C_LIGHT).ravel()
        v = (self.uvw[:, :, 1:2] * f / C_LIGHT).ravel()
        w = (self.uvw[:, :, 2:3] * f / C_LIGHT).ravel()
        return (np.ascontiguousarray(u), np.ascontiguousarray(v),
                np.ascontiguousarray(w), np.array(self.vis.ravel(), copy=True))


def enu_to_xyz(enu: np.ndarray, lat_rad: float) -> np.ndarray:
    e, n, up = enu[:, 0], enu[:, 1], enu[:, 2]
    x = -math.sin(lat_rad) * n + math.cos(lat_rad) * up
    y = e
    z = math.cos(lat_rad) * n + math.sin(lat_rad) * up
    return np.stack([x, y, z], axis=1)


def baseline_uvw(xyz_bl: np.ndarray, ha_rad: np.ndarray, dec_rad: float) -> np.ndarray:
    """[bl, time, 3] from equatorial baselines (TMS eq. 4.1)."""
    sh, ch = np.sin(ha_rad)[None, :], np.cos(ha_rad)[None, :]
    sd, cd = math.sin(dec_rad), math.cos(dec_rad)
    x, y, z = (xyz_bl[:, i][:, None] for i in range(3))
    u = sh * x + ch * y
    v = -sd * ch * x + sd * sh * y + cd * z
    w = cd * ch * x - cd * sh * y + sd * z
    return np.stack([u, v, w], axis=2)


def predict(u, v, w, sources: np.ndarray, chunk: int = 1 << 18) -> np.ndarray:
    """V = sum_s A_s exp(-2 pi i (u l + v m + w (n - 1))), sources [S, 3] (l, m, A)."""
    out = np.zeros(len(u), dtype=np.complex128)
    l, m, a = sources[:, 0], sources[:, 1], sources[:, 2]
    nm1 = np.sqrt(1.0 - l * l - m * m) - 1.0
    for s0 in range(0, len(u), chunk):
        sl = slice(s0, s0 + chunk)
        ph = np.outer(u[sl], l) + np.outer(v[sl], m) + np.outer(w[sl], nm1)
        out[sl] = (np.exp(-2j * np.pi * ph) * a[None, :]).sum(axis=1)
    return out


def _pairs(n_ant: int):
    a1, a2 = np.triu_indices(n_ant, k=1)
    return a1.astype(np.int64), a2.astype(np.int64)


def observe(enu: np.ndarray, lat_deg: float, dec_deg: float, ha_hours: np.ndarray,
            freqs: np.ndarray, sources: np.ndarray, w_scale: float = 1.0) -> Observation:
    lat, dec = math.radians(lat_deg), math.radians(dec_deg)
    xyz = enu_to_xyz(enu, lat)
    a1, a2 = _pairs(len(enu))
    bl = xyz[a2] - xyz[a1]
    ha = np.asarray(ha_hours, dtype=np.float64) * (math.pi / 12.0)
    uvw = baseline_uvw(bl, ha, dec)
    if w_scale != 1.0:
        uvw[:, :, 2] *= w_scale
    nbl, nt = uvw.shape[0], uvw.shape[1]
    freq = np.broadcast_to(np.asarray(freqs, dtype=np.float64), (nbl, len(freqs))).copy()
    obs = Observation(uvw=uvw, freq=freq, time=np.asarray(ha_hours, dtype=np.float64),
                      vis=np.zeros((nbl, nt, len(freqs)), np.complex128),
                      antenna1=a1, antenna2=a2, meta={})
    u, v, w, _ = obs.flat()
    obs.vis = predict(u, v, w, sources).reshape(nbl, nt, len(freqs))
    return obs


def fit_scale(enu, lat_deg, dec_deg, ha_hours, freqs, limit_lambda: float) -> float:
    """Array scale putting the largest |u|, |v| (wavelengths) at limit_lambda."""
    lat, dec = math.radians(lat_deg), math.radians(dec_deg)
    xyz = enu_to_xyz(enu, lat)
    a1, a2 = _pairs(len(enu))
    uvw = baseline_uvw(xyz[a2] - xyz[a1], np.asarray(ha_hours) * math.pi / 12.0, dec)
    peak = np.max(np.abs(uvw[:, :, :2])) * np.max(freqs) / C_LIGHT
    return limit_lambda / peak


def random_sources(rng: np.random.Generator, count: int, theta: float, flux: str,
                   extent: float = 0.8) -> np.ndarray:
    lm = rng.uniform(-0.5 * extent * theta, 0.5 * extent * theta, size=(count, 2))
    if flux == "uniform":
        a = rng.uniform(0.1, 1.0, size=count)
    else:  # power law dN/dS ~ S^-1.5 between 0.01 and 1 Jy (inverse CDF)
        lo, hi, k = 0.01, 1.0, -1.5
        r = rng.uniform(size=count)
        a = (lo ** (k + 1) + r * (hi ** (k + 1) - lo ** (k + 1))) ** (1.0 / (k + 1))
    return np.column_stack([lm, a])


def uniform_disc(rng, count, radius):
    r = radius * np.sqrt(rng.uniform(size=count))
    phi = rng.uniform(0, 2 * math.pi, size=count)
    return np.column_stack([r * np.cos(phi), r * np.sin(phi), np.zeros(count)])


def log_radial(rng, count, r_min, r_max):
    r = r_min * (r_max / r_min) ** rng.uniform(size=count)
    phi = rng.uniform(0, 2 * math.pi, size=count)
    return np.column_stack([r * np.cos(phi), r * np.sin(phi), np.zeros(count)])


# ----------------------------------------------------------------------------
# Named workloads
# ----------------------------------------------------------------------------

def wproj_plain(seed: int = 0, n_ant: int = 27, n_dump: int = 64, theta: float = 0.1,
                lam: float = 5120.0, ksize: int = 16, n_src: int = 10):
    """W-projection workload: 512x512 grid (theta 0.1, lambda 5120), 27 stations
    uniform within a disc, 351 baselines x 64 dumps = 22,464 visibilities at
    1.4 GHz, dec -30 deg, phase centre 40 deg from zenith at transit (site
    latitude +10 deg), hour angles -2 h .. +2 h.  Recorded knob: the disc
    radius is scaled (from 10 km) so the longest |u|, |v| keeps the whole
    16-tap footprint inside the grid."""
    rng = np.random.default_rng(seed)
    enu = uniform_disc(rng, n_ant, 10_000.0)
    lat, dec = 10.0, -30.0
    ha = np.linspace(-2.0, 2.0, n_dump)
    freqs = np.array([1.4e9])
    n_grid = int(theta * lam)
    limit = (n_grid / 2 - ksize / 2 - 2) / theta
    scale = fit_scale(enu, lat, dec, ha, freqs, limit)
    enu = enu * scale
    src = random_sources(rng, n_src, theta, "uniform")
    obs = observe(enu, lat, dec, ha, freqs, src)
    obs.meta = dict(name="wproj_plain", theta=theta, lam=lam, grid_size=n_grid,
                    array_scale=scale, lat=lat, dec=dec, sources=src, seed=seed)
    return obs


def wtowers_plain(seed: int = 1, n_st: int = 256, n_dump: int = 16, n_chan: int = 4,
                  theta: float = 0.1, lam: float = 20480.0, ksize: int = 16,
                  n_src: int = 50, dump_s: float = 120.0, r_max: float = 20_000.0,
                  ha_offset_hours: float = 0.0):
    """W-towers workload: 2048x2048 grid (theta 0.1, lambda 20480), SKA-Low-like
    256 stations on a seeded log-radial layout (20 m .. 20 km radius, i.e.
    baselines to 40 km), 32,640 baselines x 16 dumps x 4 channels = 2,088,960
    visibilities, zenith phase centre (dec = site latitude -26.8 deg), 2-minute
    dumps centred on transit, 50 power-law sources.  Recorded knob: the base
    frequency is set so the longest |u|, |v| fits the grid (channels 0.5%
    apart)."""
    rng = np.random.default_rng(seed)
    enu = log_radial(rng, n_st, 20.0, r_max)
    lat = dec = -26.8
    ha = (np.arange(n_dump) - (n_dump - 1) / 2) * dump_s / 3600.0 + ha_offset_hours
    n_grid = int(theta * lam)
    limit = (n_grid / 2 - ksize / 2 - 2) / theta
    rel = 1.0 + 0.005 * np.arange(n_chan)
    f0 = fit_scale(enu, lat, dec, ha, rel, limit)  # frequency knob: base frequency in Hz
    freqs = rel * f0
    src = random_sources(rng, n_src, theta, "powerlaw")
    obs = observe(enu, lat, dec, ha, freqs, src)
    obs.meta = dict(name="wtowers_plain", theta=theta, lam=lam, grid_size=n_grid,
                    freq0=float(freqs[0]), lat=lat, dec=dec, sources=src, seed=seed)
    return obs


def wtowers_full(seed: int = 4, n_st: int = 512, n_dump: int = 32, n_chan: int = 2,
                 theta: float = 0.1, lam: float = 40960.0, ksize: int = 16,
                 n_src: int = 100, dump_s: float = 60.0, r_max: float = 20_000.0,
                 ha_offset_hours: float = 0.0):
    """Full-scale W-towers workload: 4096x4096 grid (theta 0.1, lambda 40960),
    512 stations -> 130,816 baselines x 32 dumps x 2 channels = 8,372,224
    visibilities, 100 power-law sources; same knobs as wtowers_plain."""
    return _rename(wtowers_plain(seed, n_st, n_dump, n_chan, theta, lam, ksize, n_src,
                                 dump_s, r_max, ha_offset_hours), "wtowers_full")


def _rename(obs, name):
    obs.meta["name"] = name
    return obs


def dft_study(seed: int = 2, n_vis: int = 200_000, theta: float = 0.05,
              lam: float = 20480.0):
    """Direct-DFT precision workload: 1024x1024 image at theta 0.05 against
    200,000 visibilities from the W-projection generator (27 stations,
    351 baselines x 570 dumps, truncated), scaled so max |u|, |v| = 10,240 lambda,
    with w scaled (recorded knob) so max |w| = 2,000 lambda."""
    rng = np.random.default_rng(seed)
    enu = uniform_disc(rng, 27, 10_000.0)
    lat, dec = 10.0, -30.0
    n_dump = -(-n_vis // 351)
    ha = np.linspace(-4.0, 4.0, n_dump)
    freqs = np.array([1.4e9])
    scale = fit_scale(enu, lat, dec, ha, freqs, 10_240.0)
    enu = enu * scale
    xyz = enu_to_xyz(enu, math.radians(lat))
    a1, a2 = _pairs(27)
    uvw = baseline_uvw(xyz[a2] - xyz[a1], ha * math.pi / 12, math.radians(dec))
    wmax = np.max(np.abs(uvw[:, :, 2])) * freqs[0] / C_LIGHT
    src = random_sources(rng, 10, theta, "uniform")
    obs = observe(enu, lat, dec, ha, freqs, src, w_scale=2000.0 / wmax)
    obs.meta = dict(name="dft_study", theta=theta, lam=lam, grid_size=int(theta * lam),
                    array_scale=scale, w_scale=2000.0 / wmax, sources=src, seed=seed,
                    n_vis=n_vis)
    return obs


def learned_wproj(seed: int = 3, n_vis: int = 1_000_000, theta: float = 0.1,
                  lam: float = 20480.0, ksize: int = 16, w_limit: float = 2000.0):
    """Learned-kernel W-projection workload: the W-projection generator scaled to
    a 2048x2048 grid (theta 0.1, lambda 20480) with 1,000,000 visibilities
    (351 baselines x 2850 dumps, truncated).  Recorded knob: w is scaled so
    max |w| = w_limit (the learned kernel's training range)."""
    rng = np.random.default_rng(seed)
    enu = uniform_disc(rng, 27, 10_000.0)
    lat, dec = 10.0, -30.0
    n_dump = -(-n_vis // 351)
    ha = np.linspace(-2.0, 2.0, n_dump)
    freqs = np.array([1.4e9])
    n_grid = int(theta * lam)
    scale = fit_scale(enu, lat, dec, ha, freqs, (n_grid / 2 - ksize / 2 - 2) / theta)
    src = random_sources(rng, 10, theta, "uniform")
    xyz = enu_to_xyz(enu * scale, math.radians(lat))
    a1, a2 = _pairs(len(enu))
    uvw = baseline_uvw(xyz[a2] - xyz[a1], ha * math.pi / 12, math.radians(dec))
    wmax = np.max(np.abs(uvw[:, :, 2])) * freqs[0] / C_LIGHT
    obs = observe(enu * scale, lat, dec, ha, freqs, src, w_scale=w_limit / wmax)
    obs.meta = dict(name="learned_wproj", theta=theta, lam=lam, grid_size=n_grid,
                    array_scale=scale, w_scale=w_limit / wmax, sources=src, seed=seed, n_vis=n_vis)
    return obs


def flat_truncate(flat, n):
    return tuple(np.ascontiguousarray(a[:n]) for a in flat)


def wkernel_for(flat_w: np.ndarray, theta: float, w_step: float, size: int = 16,
                oversampling: int = 8, c: float | None = None) -> WKernel:
    """Table covering the w range of the data with planes every w_step."""
    lo = math.floor(min(float(np.min(flat_w)), 0.0) / w_step) - 1
    hi = math.ceil(max(float(np.max(flat_w)), 0.0) / w_step) + 1
    planes = np.arange(lo, hi + 1) * w_step
    return generate_wkernel(theta, planes, size, oversampling, c)


def learned_training_set(n_triples: int, wmax: float, theta: float, size: int = 16,
                         c: float | None = None, seed: int = 0, m_pix: int = 128,
                         batch: int = 128):
    """Training taps for the learned w-kernel: n_triples random (w, du, dv) with
    w uniform in [-wmax, wmax] and du, dv uniform in [0, 1), each with all
    size x size taps of the generator's continuous kernel
        K_w(tx - size/2 - du, ty - size/2 - dv)   (kernel_taps).
    Returns (w, du, dv, tx, ty) float arrays and complex128 targets, one entry
    per tap (n_triples * size^2)."""
    if c is None:
        c = math.pi * (size - 2) / 2.0
    rng = np.random.default_rng(seed)
    w = rng.uniform(-wmax, wmax, n_triples)
    du = rng.uniform(0.0, 1.0, n_triples)
    dv = rng.uniform(0.0, 1.0, n_triples)
    lm = screen_coords(theta, m_pix)
    a = pswf0(c, 2.0 * lm / theta)
    taper = a[None, :] * a[:, None]
    one_minus_n = 1.0 - np.sqrt(1.0 - (lm[None, :] ** 2 + lm[:, None] ** 2))
    taps = np.arange(size) - size // 2
    out = np.empty((n_triples, size, size), np.complex128)
    for b0 in range(0, n_triples, batch):
        sl = slice(b0, min(b0 + batch, n_triples))
        s = taper[None] * np.exp(2j * np.pi * w[sl, None, None] * one_minus_n[None])
        px = taps[None, :] - du[sl, None]
        qy = taps[None, :] - dv[sl, None]
        ex = np.exp(-2j * np.pi * px[:, :, None] * lm[None, None, :] / theta)
        ey = np.exp(-2j * np.pi * qy[:, :, None] * lm[None, None, :] / theta)
        out[sl] = ey @ s @ np.transpose(ex, (0, 2, 1)) / (m_pix * m_pix)
    ty, tx = np.meshgrid(np.arange(size), np.arange(size), indexing="ij")
    rep = size * size
    return (np.repeat(w, rep), np.repeat(du, rep), np.repeat(dv, rep),
            np.tile(tx.ravel(), n_triples).astype(np.float64),
            np.tile(ty.ravel(), n_triples).astype(np.float64), out.reshape(-1))


# ----------------------------------------------------------------------------
# Separable kernels for W-stacking predict
# ----------------------------------------------------------------------------

def sepkern_pswf(support: int, oversampling: int, x0: float = 0.25, c: float | None = None,
                 corr_size: int = 64, corr_oversampling: int = 64):
    """A separable gridding kernel and its grid correction in the table
    layouts the W-stacking predict indexes (src/wstack/wstack_common.h:460-478
    for the convolution, src/wstack/predict.cpp:219-234 for the correction):

    * conv[j, t] = C(t - support/2 + (j + 1/2)/oversampling), C(x) =
      psi_0(c, 2x/support) on |x| <= support/2: the predict maps a visibility
      f of a cell before its first grid point (0 <= f < 1) to j = floor(f ov),
      so row j holds the kernel at the middle of [j/ov, (j+1)/ov);
    * corr[k] = C^(nu_k), nu_k = (k - T/2) / T, T = corr_size * corr_oversampling:
      the kernel's continuous Fourier transform (what the gridded sky is
      divided by), by Simpson quadrature.

    The reference reads Sze-Tan kernels from HDF5 files instead
    (load_sep_kern, src/common/hdf5.c:372-497); this is a PSWF stand-in with
    the same meaning, c = 3 pi support x0 by default."""
    if c is None:
        c = 3.0 * math.pi * support * x0
    ov = oversampling
    t = np.arange(support)[None, :] - support // 2 + (np.arange(ov)[:, None] + 0.5) / ov
    conv = np.where(np.abs(t) <= support / 2, pswf0(c, np.clip(2.0 * t / support, -1.0, 1.0)), 0.0)
    T = corr_size * corr_oversampling
    nu = (np.arange(T) - T // 2) / T
    xq = np.linspace(0.0, support / 2, 4001)
    cq = pswf0(c, 2.0 * xq / support)
    wq = np.full(xq.size, 2.0)
    wq[1::2] = 4.0
    wq[0] = wq[-1] = 1.0
    wq *= (xq[1] - xq[0]) / 3.0
    corr = 2.0 * (np.cos(2 * np.pi * np.outer(nu, xq)) * (cq * wq)[None, :]).sum(axis=1)
    return np.ascontiguousarray(conv), np.ascontiguousarray(corr.reshape(corr_oversampling, corr_size))


def akern_for(obs, n_time: int = 3, n_freq: int = 2, size: int = 16, seed: int = 0, jitter: float = 0.0):
    """An A-kernel table (rg_akern layout) for an observation: per antenna,
    n_time slots spanning its times and n_freq channels spanning its
    frequencies (each kernel's own time and frequency, optionally jittered by
    `jitter` of a step so the nearest-slot search has something to decide),
    smooth seeded complex kernel values.  The reference's AW-projection reads
    only the kernels' frequencies (src/reference/grid.c:571-590)."""
    rng = np.random.default_rng(seed)
    n_ant = int(max(obs.antenna1.max(), obs.antenna2.max())) + 1
    t = np.asarray(obs.time, np.float64)
    f = np.asarray(obs.freq, np.float64)
    t_min, t_max = float(t.min()), float(t.max())
    f_min, f_max = float(f.min()), float(f.max())
    t_step = (t_max - t_min) / (n_time - 1) if n_time > 1 else 1.0
    f_step = (f_max - f_min) / (n_freq - 1) if n_freq > 1 else 1.0
    ta = t_min + np.arange(n_time) * t_step
    fa = f_min + np.arange(n_freq) * f_step
    time = np.broadcast_to(ta[None, :, None], (n_ant, n_time, n_freq)).copy()
    freq = np.broadcast_to(fa[None, None, :], (n_ant, n_time, n_freq)).copy()
    if jitter:
        freq = freq + jitter * f_step * rng.uniform(-1, 1, freq.shape)
    y, x = np.mgrid[:size, :size] - size / 2
    base = np.exp(-(x * x + y * y) / (size * size / 8.0))
    data = base[None, None, None] * np.exp(1j * rng.uniform(0, 2 * np.pi, (n_ant, n_time, n_freq, 1, 1)))
    from types import SimpleNamespace
    return SimpleNamespace(freq=freq, time=time, data=data, t_min=t_min, t_step=t_step, f_min=f_min, f_step=f_step)
