"""ORACLE — test infrastructure, not the product.

Only tests/, __graft_entry__.smoke() and bench.py (its CPU-baseline leg and its
``--impl reference`` arm) import this package, and only as the checker.

Two CPU implementations of the reference gridder are exposed through ctypes:

* ``restated``: oracle/rg_oracle.c, a plain-C FP64 restatement of
  src/reference/grid.c on flat visibility arrays, plus the FP64 DFT oracle;
* ``reference``: the reference's own src/reference/grid.c compiled from its
  sources here (oracle/Makefile -> oracle/_ref/libref_grid.so, IEEE build;
  libref_grid_omp.so with the reference's flags and -DOMP_TOWERS for timing),
  driven through in-memory struct vis_data / struct w_kernel_data mirrors of
  src/reference/grid.h:7-49.

Parity pin: tests/test_oracle_pin.py checks ``restated`` == ``reference``
bit-for-bit; tests/golden/ holds fixtures produced by ``reference``.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF = os.path.join(HERE, "_ref")
# Directory of the reference's src/reference sources (read in place); set by
# the caller, no default.
REFERENCE_SRC = os.environ.get("RG_REFERENCE_SRC")

_c_double_p = ct.POINTER(ct.c_double)


def build(reference: bool = True, reference_src: str | None = None) -> None:
    """Compile the restatement (always) and the reference build from the
    reference's src/reference directory (``reference_src``, else the
    RG_REFERENCE_SRC environment variable) when one is given and present."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    src = reference_src or REFERENCE_SRC
    if reference and src and os.path.isdir(src):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_SRC={src}"], check=True)


def _ptr(a):
    return a.ctypes.data_as(ct.c_void_p)


# --------------------------------------------------------------------------
# restatement
# --------------------------------------------------------------------------

class _Wk(ct.Structure):
    _fields_ = [("data", ct.c_void_p), ("plane_count", ct.c_int), ("size", ct.c_int),
                ("oversampling", ct.c_int), ("w_min", ct.c_double), ("w_step", ct.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(BUILD, "librgoracle.so")
        if not os.path.exists(path):
            build(reference=False)
        L = ct.CDLL(path)
        i64, vp, d, i = ct.c_int64, ct.c_void_p, ct.c_double, ct.c_int
        L.rgo_grid_wprojection.argtypes = [vp, i, d, i64, vp, vp, vp, vp, ct.POINTER(_Wk)]
        L.rgo_grid_wprojection.restype = ct.c_uint64
        L.rgo_grid_wtowers.argtypes = [vp, i, d, i64, vp, vp, vp, vp, ct.POINTER(_Wk), i, i, d, vp, vp]
        L.rgo_wtowers_census.argtypes = [i, d, i64, vp, vp, vp, i, i, d, vp, vp]
        L.rgo_grid_wtowers.restype = ct.c_uint64
        L.rgo_weight.argtypes = [i, d, i64, vp, vp, vp]
        L.rgo_grid_simple.argtypes = [vp, i, d, i64, vp, vp, vp]
        L.rgo_grid_simple.restype = i
        L.rgo_make_hermitian.argtypes = [vp, i]
        L.rgo_fft_shift.argtypes = [vp, i]
        L.rgo_image_from_grid.argtypes = [vp, i, vp]
        L.rgo_dft_image.argtypes = [vp, i, d, i64, vp, vp, vp, vp, d]
        L.rgo_dft_pixels.argtypes = [vp, i, vp, vp, i, d, i64, vp, vp, vp, vp, d]
        L.rgo_wstack_planes.argtypes = [d, d, d, i]
        L.rgo_wstack_planes.restype = i
        L.rgo_wstack_predict.argtypes = [d, d, i, vp, i64, vp, vp, vp, d, d, d, vp, i, i, vp, i, i, vp, i, i,
                                         vp, i, i, vp]
        L.rgo_wstack_predict.restype = i
        L.rgo_predict_dft_quantized.argtypes = [d, d, i, vp, i64, vp, vp, vp, vp]
        L.rgo_grid_awprojection.argtypes = [vp, i, d, i, i, i, i, vp, vp, vp, vp, vp, ct.POINTER(_Wk), i, i, i,
                                            d, d, d, d, vp]
        L.rgo_grid_awprojection.restype = i
        L.rgo_frac_coord.argtypes = [i, i, i, d, d, d, d, d, ct.POINTER(i), ct.POINTER(i)]
        _lib = L
    return _lib


def _wk_struct(wk):
    data = np.ascontiguousarray(wk.data, dtype=np.complex128)
    s = _Wk(data.ctypes.data, wk.plane_count, wk.size, wk.oversampling, wk.w_min, wk.w_step)
    return s, data


def _flat(u, v, w, vis):
    return (np.ascontiguousarray(u, np.float64), np.ascontiguousarray(v, np.float64),
            np.ascontiguousarray(w, np.float64), np.ascontiguousarray(vis, np.complex128))


def grid_wprojection(grid_size, theta, u, v, w, vis, wk):
    u, v, w, vis = _flat(u, v, w, vis)
    grid = np.zeros((grid_size, grid_size), np.complex128)
    s, keep = _wk_struct(wk)
    lib().rgo_grid_wprojection(_ptr(grid), grid_size, theta, len(u), _ptr(u), _ptr(v),
                               _ptr(w), _ptr(vis), ct.byref(s))
    return grid


def grid_wtowers(grid_size, theta, u, v, w, vis, wk, subgrid, margin, winc,
                 return_counts=False, towers=None):
    """towers: optional boolean array over the towers (row-major): grid only
    those (one share of a tower-partitioned observation)."""
    u, v, w, vis = _flat(u, v, w, vis)
    grid = np.zeros((grid_size, grid_size), np.complex128)
    s, keep = _wk_struct(wk)
    counts = np.zeros(len(u), np.int32)
    sel = None if towers is None else np.ascontiguousarray(towers, np.uint8)
    lib().rgo_grid_wtowers(_ptr(grid), grid_size, theta, len(u), _ptr(u), _ptr(v),
                           _ptr(w), _ptr(vis), ct.byref(s), subgrid, margin, winc,
                           _ptr(counts), None if sel is None else _ptr(sel))
    return (grid, counts) if return_counts else grid


def wtowers_census(grid_size, theta, u, v, w, subgrid, margin, winc):
    """(visibilities per tower int64, active w-floors per tower int32)."""
    u, v, w, _ = _flat(u, v, w, np.zeros(0))
    nc = grid_size // (subgrid - margin) + 1
    nv = np.zeros(nc * nc, np.int64)
    nf = np.zeros(nc * nc, np.int32)
    lib().rgo_wtowers_census(grid_size, theta, len(u), _ptr(u), _ptr(v), _ptr(w), subgrid, margin, winc,
                             _ptr(nv), _ptr(nf))
    return nv, nf


def grid_simple(grid_size, theta, u, v, vis):
    """grid.c:83-99 restated (nearest-cell gridding)."""
    u, v, _, vis = _flat(u, v, u, vis)
    grid = np.zeros((grid_size, grid_size), np.complex128)
    if lib().rgo_grid_simple(_ptr(grid), grid_size, theta, len(u), _ptr(u), _ptr(v), _ptr(vis)):
        raise ValueError("a visibility's cell lies off the grid")
    return grid


def weight(grid_size, theta, u, v, vis):
    u, v, _, vis = _flat(u, v, u, vis)
    out = vis.copy()
    lib().rgo_weight(grid_size, theta, len(u), _ptr(u), _ptr(v), _ptr(out))
    return out


def make_hermitian(grid):
    g = np.ascontiguousarray(grid, np.complex128).copy()
    lib().rgo_make_hermitian(_ptr(g), g.shape[0])
    return g


def fft_shift(grid):
    g = np.ascontiguousarray(grid, np.complex128).copy()
    lib().rgo_fft_shift(_ptr(g), g.shape[0])
    return g


def image_from_grid(grid):
    g = np.ascontiguousarray(grid, np.complex128).copy()
    img = np.zeros(g.shape, np.float64)
    lib().rgo_image_from_grid(_ptr(g), g.shape[0], _ptr(img))
    return img


def dft_image(grid_size, theta, u, v, w, vis, factor=2.0):
    u, v, w, vis = _flat(u, v, w, vis)
    img = np.zeros((grid_size, grid_size), np.float64)
    lib().rgo_dft_image(_ptr(img), grid_size, theta, len(u), _ptr(u), _ptr(v), _ptr(w),
                        _ptr(vis), factor)
    return img


def dft_pixels(grid_size, theta, u, v, w, vis, px, py, factor=2.0):
    """The FP64 DFT oracle at pixels (px[k], py[k]) (column, row) only."""
    u, v, w, vis = _flat(u, v, w, vis)
    px = np.ascontiguousarray(px, np.int32)
    py = np.ascontiguousarray(py, np.int32)
    out = np.zeros(len(px), np.float64)
    lib().rgo_dft_pixels(_ptr(out), len(px), _ptr(px), _ptr(py), grid_size, theta, len(u), _ptr(u), _ptr(v),
                         _ptr(w), _ptr(vis), factor)
    return out


def wstack_predict(theta, lam, points, u, v, w, du, dw, x0, conv_uv, conv_w, corr_lm, corr_n):
    """src/wstack/predict.cpp:396-562.  points: [npts, 2] (l, m); each table
    a 2-D float64 array [oversampling, size] (data[ov_index * size + tap])."""
    u, v, w, _ = _flat(u, v, w, np.zeros(0))
    pts = np.ascontiguousarray(points, np.float64).reshape(-1, 2)
    tabs = [np.ascontiguousarray(t, np.float64) for t in (conv_uv, conv_w, corr_lm, corr_n)]
    out = np.zeros(len(u), np.complex128)
    args = []
    for t in tabs:
        args += [_ptr(t), t.shape[1], t.shape[0]]
    st = lib().rgo_wstack_predict(theta, lam, len(pts), _ptr(pts), len(u), _ptr(u), _ptr(v), _ptr(w), du, dw, x0,
                                  *args, _ptr(out))
    if st != 0:
        raise ValueError(f"wstack_predict oracle failed ({st})")
    return out


def wstack_planes(theta, lam, dw, support_w):
    return lib().rgo_wstack_planes(theta, lam, dw, support_w)


def predict_dft_quantized(theta, lam, points, u, v, w):
    """src/wstack/predict.cpp:89-129."""
    u, v, w, _ = _flat(u, v, w, np.zeros(0))
    pts = np.ascontiguousarray(points, np.float64).reshape(-1, 2)
    out = np.zeros(len(u), np.complex128)
    lib().rgo_predict_dft_quantized(theta, lam, len(pts), _ptr(pts), len(u), _ptr(u), _ptr(v), _ptr(w), _ptr(out))
    return out


def grid_awprojection(grid_size, theta, hv, wk, ak, bl_min=0, bl_max=None):
    """src/reference/grid.c:557-637 restated (convolve_aw_kernels +
    grid_awprojection).  hv: HierVis-like (antenna1, time [bl, nt], freq
    [bl, nf], uvw, vis); ak: AKernels-like (freq [ant, nt, nf], axes)."""
    nbl, nt = hv.uvw.shape[:2]
    nf = hv.freq.shape[1]
    a1 = np.ascontiguousarray(hv.antenna1, np.int32)
    tm = np.ascontiguousarray(np.broadcast_to(np.asarray(hv.time, np.float64), (nbl, nt)))
    fr = np.ascontiguousarray(hv.freq, np.float64)
    uvw = np.ascontiguousarray(hv.uvw, np.float64)
    vis = np.ascontiguousarray(hv.vis, np.complex128)
    akf = np.ascontiguousarray(ak.freq, np.float64)
    grid = np.zeros((grid_size, grid_size), np.complex128)
    s, keep = _wk_struct(wk)
    st = lib().rgo_grid_awprojection(_ptr(grid), grid_size, theta, bl_min, nbl if bl_max is None else bl_max, nt, nf,
                                     _ptr(a1), _ptr(tm), _ptr(fr), _ptr(uvw), _ptr(vis), ct.byref(s),
                                     akf.shape[0], akf.shape[1], akf.shape[2], ak.t_min, ak.t_step, ak.f_min,
                                     ak.f_step, _ptr(akf))
    if st != 0:
        raise ValueError("AW-projection oracle: an index leaves its table")
    return grid


def frac_coord(grid_size, ksize, ov, theta, u, v, du=0.0, dv=0.0):
    go, so = ct.c_int(), ct.c_int()
    lib().rgo_frac_coord(grid_size, ksize, ov, theta, u, v, du, dv, ct.byref(go), ct.byref(so))
    return go.value, so.value


# --------------------------------------------------------------------------
# the reference's own grid.c (struct mirrors of src/reference/grid.h:7-49)
# --------------------------------------------------------------------------

class BlData(ct.Structure):
    _fields_ = [("antenna1", ct.c_int), ("antenna2", ct.c_int),
                ("time_count", ct.c_int), ("freq_count", ct.c_int),
                ("time", _c_double_p), ("freq", _c_double_p), ("uvw", _c_double_p),
                ("vis", ct.c_void_p), ("awkern", ct.c_void_p),
                ("u_min", ct.c_double), ("u_max", ct.c_double),
                ("v_min", ct.c_double), ("v_max", ct.c_double),
                ("w_min", ct.c_double), ("w_max", ct.c_double),
                ("t_min", ct.c_double), ("t_max", ct.c_double),
                ("f_min", ct.c_double), ("f_max", ct.c_double),
                ("flops", ct.c_uint64)]


class VisData(ct.Structure):
    _fields_ = [("antenna_count", ct.c_int), ("bl_count", ct.c_int),
                ("bl", ct.POINTER(BlData))]


class WKern(ct.Structure):
    _fields_ = [("data", ct.c_void_p), ("w", ct.c_double)]


class WKernData(ct.Structure):
    _fields_ = [("plane_count", ct.c_int), ("kern", ct.POINTER(WKern)),
                ("kern_by_w", ct.POINTER(WKern)), ("w_min", ct.c_double),
                ("w_max", ct.c_double), ("w_step", ct.c_double),
                ("size_x", ct.c_int), ("size_y", ct.c_int), ("oversampling", ct.c_int)]


class AKernelC(ct.Structure):  # struct a_kernel, src/reference/grid.h:70-76
    _fields_ = [("data", ct.c_void_p), ("antenna", ct.c_int), ("time", ct.c_double), ("freq", ct.c_double)]


class AKernelData(ct.Structure):  # struct a_kernel_data, src/reference/grid.h:77-85
    _fields_ = [("antenna_count", ct.c_int), ("time_count", ct.c_int), ("freq_count", ct.c_int),
                ("kern", ct.POINTER(AKernelC)), ("kern_by_atf", ct.POINTER(AKernelC)),
                ("t_min", ct.c_double), ("t_max", ct.c_double), ("t_step", ct.c_double),
                ("f_min", ct.c_double), ("f_max", ct.c_double), ("f_step", ct.c_double),
                ("size_x", ct.c_int), ("size_y", ct.c_int)]


_ref_libs = {}


class quiet_stdout:
    """Silence C-level stdout (the reference prints progress with printf,
    e.g. grid.c:406) so it cannot mix into a caller's output."""

    def __enter__(self):
        import sys
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *exc):
        ct.CDLL(None).fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)
        return False


def reference_available(omp=False):
    return os.path.exists(os.path.join(REF, "libref_grid_omp.so" if omp else "libref_grid.so"))


def ref_lib(omp=False):
    name = "libref_grid_omp.so" if omp else "libref_grid.so"
    if name not in _ref_libs:
        path = os.path.join(REF, name)
        if not os.path.exists(path):
            build(reference=True)
        L = ct.CDLL(path)
        vp = ct.c_void_p
        L.grid_wprojection.argtypes = [vp, ct.c_int, ct.c_double, ct.POINTER(VisData),
                                       ct.POINTER(WKernData)]
        L.grid_wprojection.restype = ct.c_uint64
        L.grid_wtowers.argtypes = [vp, ct.c_int, ct.c_double, ct.POINTER(VisData),
                                   ct.POINTER(WKernData), ct.c_int, ct.c_int, ct.c_double]
        L.grid_wtowers.restype = ct.c_uint64
        L.weight.argtypes = [vp, ct.c_int, ct.c_double, ct.POINTER(VisData)]
        L.grid_simple.argtypes = [vp, ct.c_int, ct.c_double, ct.POINTER(VisData)]
        L.grid_simple.restype = ct.c_uint64
        L.make_hermitian.argtypes = [vp, ct.c_int]
        L.convolve_aw_kernels.argtypes = [ct.POINTER(BlData), ct.POINTER(WKernData), ct.POINTER(AKernelData)]
        L.grid_awprojection.argtypes = [vp, ct.c_int, ct.c_double, ct.POINTER(VisData), ct.POINTER(WKernData),
                                        ct.POINTER(AKernelData), ct.c_int, ct.c_int]
        L.grid_awprojection.restype = ct.c_uint64
        L.fft_shift.argtypes = [vp, ct.c_int]
        _ref_libs[name] = L
    return _ref_libs[name]


class RefInputs:
    """Keeps the numpy buffers alive behind the ctypes structs."""

    def __init__(self, obs, wk=None):
        nbl = obs.uvw.shape[0]
        self.arrays = []
        self.bl = (BlData * nbl)()
        c = 299792458.0
        vis = np.array(obs.vis, dtype=np.complex128, order="C", copy=True)  # weight() writes it
        self.vis = vis
        for b in range(nbl):
            uvw = np.ascontiguousarray(obs.uvw[b], np.float64)
            fr = np.ascontiguousarray(obs.freq[b], np.float64)
            tm = np.ascontiguousarray(obs.time, np.float64)
            vb = np.ascontiguousarray(vis[b])
            self.arrays += [uvw, fr, tm, vb]
            e = self.bl[b]
            e.antenna1, e.antenna2 = int(obs.antenna1[b]), int(obs.antenna2[b])
            e.time_count, e.freq_count = uvw.shape[0], fr.shape[0]
            e.time = tm.ctypes.data_as(_c_double_p)
            e.freq = fr.ctypes.data_as(_c_double_p)
            e.uvw = uvw.ctypes.data_as(_c_double_p)
            e.vis = vb.ctypes.data
            e.awkern = None
            # per-baseline statistics as load_vis_group computes them
            # (src/reference/hdf5.c:143-171)
            e.u_min, e.u_max = float(uvw[:, 0].min()), float(uvw[:, 0].max())
            e.v_min, e.v_max = float(uvw[:, 1].min()), float(uvw[:, 1].max())
            e.w_min, e.w_max = float(uvw[:, 2].min()), float(uvw[:, 2].max())
            e.t_min, e.t_max = float(tm.min()), float(tm.max())
            e.f_min, e.f_max = float(fr.min()), float(fr.max())
            e.flops = 0
        self.vd = VisData(int(max(obs.antenna2.max(), obs.antenna1.max()) + 1), nbl, self.bl)
        if wk is not None:
            self.wk_data = np.ascontiguousarray(wk.data, np.complex128)
            n = wk.plane_count
            self.kern = (WKern * n)()
            per = wk.oversampling * wk.oversampling * wk.size * wk.size
            for p in range(n):
                self.kern[p].data = self.wk_data.ctypes.data + p * per * 16
                self.kern[p].w = wk.w_min + p * wk.w_step
            self.wkd = WKernData(n, self.kern, self.kern, wk.w_min, wk.w_max, wk.w_step,
                                 wk.size, wk.size, wk.oversampling)

    def vis_out(self):
        return np.ascontiguousarray(self.vis).ravel()


def ref_grid_wprojection(grid_size, theta, obs, wk):
    r = RefInputs(obs, wk)
    grid = np.zeros((grid_size, grid_size), np.complex128)
    with quiet_stdout():
        ref_lib().grid_wprojection(_ptr(grid), grid_size, theta, ct.byref(r.vd), ct.byref(r.wkd))
    return grid


def ref_grid_wtowers(grid_size, theta, obs, wk, subgrid, margin, winc, omp=False):
    r = RefInputs(obs, wk)
    grid = np.zeros((grid_size, grid_size), np.complex128)
    with quiet_stdout():
        ref_lib(omp).grid_wtowers(_ptr(grid), grid_size, theta, ct.byref(r.vd), ct.byref(r.wkd),
                                  subgrid, margin, winc)
    return grid


def ref_grid_awprojection(grid_size, theta, obs, wk, ak):
    """The reference's convolve_aw_kernels for every baseline, then its
    grid_awprojection (src/reference/grid.c:557-637), on an Observation and
    an AKernels-like table."""
    r = RefInputs(obs, wk)
    a, t, f = ak.freq.shape
    slots = (AKernelC * (a * t * f))()
    zeros = np.zeros(wk.size * wk.size, np.complex128)  # the reference never reads the A-kernel values
    for ai in range(a):
        for ti in range(t):
            for fi in range(f):
                k = slots[(ai * t + ti) * f + fi]
                k.data = zeros.ctypes.data
                k.antenna, k.time, k.freq = ai, float(ak.time[ai, ti, fi]), float(ak.freq[ai, ti, fi])
    akd = AKernelData(a, t, f, slots, slots, ak.t_min, ak.t_min + (t - 1) * ak.t_step, ak.t_step,
                      ak.f_min, ak.f_min + (f - 1) * ak.f_step, ak.f_step, wk.size, wk.size)
    L = ref_lib()
    for b in range(r.vd.bl_count):
        L.convolve_aw_kernels(ct.byref(r.bl[b]), ct.byref(r.wkd), ct.byref(akd))
    grid = np.zeros((grid_size, grid_size), np.complex128)
    L.grid_awprojection(_ptr(grid), grid_size, theta, ct.byref(r.vd), ct.byref(r.wkd), ct.byref(akd), 0,
                        r.vd.bl_count)
    libc = ct.CDLL(None)
    libc.free.argtypes = [ct.c_void_p]
    for b in range(r.vd.bl_count):  # the kernels convolve_aw_kernels allocated
        libc.free(r.bl[b].awkern)
        r.bl[b].awkern = None
    return grid


def ref_grid_simple(grid_size, theta, obs):
    r = RefInputs(obs)
    grid = np.zeros((grid_size, grid_size), np.complex128)
    ref_lib().grid_simple(_ptr(grid), grid_size, theta, ct.byref(r.vd))
    return grid


def ref_weight(grid_size, theta, obs):
    r = RefInputs(obs)
    wgrid = np.zeros(grid_size * grid_size, np.uint32)
    ref_lib().weight(_ptr(wgrid), grid_size, theta, ct.byref(r.vd))
    return r.vis_out()


def ref_make_hermitian(grid):
    g = np.ascontiguousarray(grid, np.complex128).copy()
    ref_lib().make_hermitian(_ptr(g), g.shape[0])
    return g


def ref_fft_shift(grid):
    g = np.ascontiguousarray(grid, np.complex128).copy()
    ref_lib().fft_shift(_ptr(g), g.shape[0])
    return g


def reference_safe_baselines(obs, grid_size, theta, subgrid, margin, ksize, ov):
    """Boolean mask of baselines the reference's grid_wtowers can grid without
    writing outside its sub-grid buffer.

    With margin == kernel support, a visibility within 1/(2 ov) cell of a
    tower's low edge gets a footprint origin on row -1 (or row 0, column -1) of
    the sub-grid; grid.c's w_project has no bounds check (grid.c:177-182) and
    writes before the buffer.  Such baselines are left out when the reference
    itself is run; the restatement and the GPU path drop only the taps that
    leave the buffer."""
    u, v, w, _ = obs.flat()
    chunk = subgrid - margin
    row0 = _origin(v, theta, grid_size, chunk, subgrid, ksize, ov)
    col0 = _origin(u, theta, grid_size, chunk, subgrid, ksize, ov)
    bad = (row0 <= 0) | (col0 <= 0)
    nbl = obs.uvw.shape[0]
    return ~bad.reshape(nbl, -1).any(axis=1)


def _origin(x, theta, n, chunk, s, k, ov):
    c = np.floor((x * theta + 0.5 + n // 2) / chunk)
    mid = (c * chunk - n // 2 + chunk // 2) / theta
    cell = np.floor(theta * (x - mid) + 0.5 / ov)
    return cell + s // 2 - k // 2


def subset_baselines(obs, mask):
    import copy
    o = copy.copy(obs)
    o.uvw = obs.uvw[mask]
    o.freq = obs.freq[mask]
    o.vis = obs.vis[mask]
    o.antenna1 = obs.antenna1[mask]
    o.antenna2 = obs.antenna2[mask]
    return o
