"""B200-native radio imager: Python mirror of the reference's gridder interface.

The compute path is the CUDA library ``librg_b200.so`` built from ``csrc/``
(sm_100a) and bound here with ctypes; there is no CPU fallback — if the
library is missing or no B200 is present, every call raises.

Function names and argument meaning follow the reference's CPU gridder API
(src/reference/grid.h:113-137): ``grid_wprojection``, ``grid_wtowers``,
``weight``, ``make_hermitian``, ``fft_shift``, plus the image pipeline of
src/reference/main.c:258-294 (``image_from_grid``) and the direct DFT imager of
src/dft/dft_cuda.cu (``dft_image``).  Like the reference, the gridders
accumulate into ``uvgrid``; errors raise :class:`RGError` instead of exiting.

Buffers may be numpy arrays (host; staged through device memory) or CUDA
tensors / any object with ``data_ptr()`` (used in place).
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librg_b200.so")

RG_GRID_ACCUMULATE = 0
RG_GRID_OVERWRITE = 1
RG_DFT_FP32_NAIVE = 0
RG_DFT_FP64_REDUCED = 1
RG_DFT_FP64 = 2

STATUS = {0: "RG_OK", 1: "RG_ERR_INVALID_ARGUMENT", 2: "RG_ERR_CUDA", 3: "RG_ERR_OUT_OF_MEMORY",
          4: "RG_ERR_UNSUPPORTED", 5: "RG_ERR_IO", 6: "RG_ERR_NO_DEVICE"}

# every symbol include/radio_gridders.h declares
EXPORTS = [
    "rg_context_create", "rg_context_destroy", "rg_context_set_stream", "rg_last_error",
    "rg_last_stats", "rg_context_set_profiling", "rg_context_set_autotune", "rg_context_set_graphs",
    "rg_last_timings", "rg_grid_wprojection", "rg_grid_wtowers", "rg_weight",
    "rg_make_hermitian", "rg_fft_shift", "rg_image_from_grid", "rg_fft2d", "rg_dft_image", "rg_dft_image_rows",
    "rg_grid_wprojection_noalloc", "rg_mlp_param_count", "rg_mlp_create", "rg_mlp_destroy",
    "rg_mlp_set_params", "rg_mlp_get_params", "rg_mlp_gradient", "rg_mlp_train", "rg_mlp_eval",
    "rg_grid_wprojection_learned", "rg_grid_wtowers_learned", "rg_grid_wtowers_batch", "rg_read_vis_hdf5", "rg_free_vis_data", "rg_read_wkern_hdf5",
    "rg_free_wkern_data", "rg_write_vis_hdf5", "rg_write_vis_flat_hdf5", "rg_write_wkern_hdf5", "rg_hdf5_read_f64",
    "rg_hdf5_attr_f64", "rg_selftest_wait_timeout", "rg_wtowers_cuda_flat", "rg_wproj_cuda_flat",
    "rg_image_dft_host_flat", "rg_wtowers_tower_count", "rg_wtowers_tower_loads", "rg_wtowers_partition",
    "rg_grid_wtowers_part", "rg_wkern_generate", "rg_pswf0", "rg_wstack_predict", "rg_grid_awprojection",
    "rg_read_vis_bl_hdf5", "rg_free_vis_bl_data", "rg_read_akern_hdf5", "rg_free_akern_data",
    "rg_write_akern_hdf5", "rg_grid_simple",
]


class _SepKern(ct.Structure):
    _fields_ = [("data", ct.c_void_p), ("size", ct.c_int), ("oversampling", ct.c_int)]


class RGError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


def build() -> None:
    """Compile csrc/ for sm_100a into librg_b200.so (make, in-tree)."""
    subprocess.run(["make", "-s", "-C", HERE, "-j", str(min(8, os.cpu_count() or 1))], check=True)


class _Vis(ct.Structure):
    _fields_ = [("u", ct.c_void_p), ("v", ct.c_void_p), ("w", ct.c_void_p),
                ("vis", ct.c_void_p), ("n", ct.c_int64)]


class _WKern(ct.Structure):
    _fields_ = [("data", ct.c_void_p), ("plane_count", ct.c_int), ("size", ct.c_int),
                ("oversampling", ct.c_int), ("w_min", ct.c_double), ("w_step", ct.c_double)]


class _VisData(ct.Structure):
    _fields_ = [("u", ct.POINTER(ct.c_double)), ("v", ct.POINTER(ct.c_double)),
                ("w", ct.POINTER(ct.c_double)), ("vis", ct.POINTER(ct.c_double)),
                ("n", ct.c_int64), ("bl_count", ct.c_int64)]


class _WKernData(ct.Structure):
    _fields_ = [("data", ct.POINTER(ct.c_double)), ("plane_count", ct.c_int), ("size", ct.c_int),
                ("oversampling", ct.c_int), ("w_min", ct.c_double), ("w_step", ct.c_double)]


_dp = ct.POINTER(ct.c_double)


class _VisBL(ct.Structure):
    _fields_ = [("bl_count", ct.c_int), ("time_count", ct.c_int), ("freq_count", ct.c_int),
                ("antenna1", ct.POINTER(ct.c_int32)), ("antenna2", ct.POINTER(ct.c_int32)),
                ("time", _dp), ("freq", _dp), ("uvw", _dp), ("vis", _dp)]


class _AKern(ct.Structure):
    _fields_ = [("antenna_count", ct.c_int), ("time_count", ct.c_int), ("freq_count", ct.c_int),
                ("size_x", ct.c_int), ("size_y", ct.c_int), ("t_min", ct.c_double), ("t_step", ct.c_double),
                ("f_min", ct.c_double), ("f_step", ct.c_double), ("freq", _dp), ("time", _dp), ("data", _dp)]


class HierVis:
    """Hierarchical visibilities (rg_vis_bl): antenna1/antenna2 [bl], time
    [bl, nt] (or [nt], shared), freq [bl, nf] Hz, uvw [bl, nt, 3] metres, vis
    [bl, nt, nf] complex."""

    def __init__(self, antenna1, antenna2, time, freq, uvw, vis):
        self.uvw = np.ascontiguousarray(uvw, np.float64)
        nbl, nt = self.uvw.shape[:2]
        self.antenna1 = np.ascontiguousarray(antenna1, np.int32)
        self.antenna2 = np.ascontiguousarray(antenna2, np.int32)
        self.time = np.ascontiguousarray(np.broadcast_to(np.asarray(time, np.float64), (nbl, nt)))
        self.freq = np.ascontiguousarray(freq, np.float64)
        self.vis = np.ascontiguousarray(vis, np.complex128)

    @classmethod
    def of(cls, obs):
        return cls(obs.antenna1, obs.antenna2, obs.time, obs.freq, obs.uvw, obs.vis)

    def struct(self):
        nbl, nt = self.uvw.shape[:2]
        return _VisBL(nbl, nt, self.freq.shape[1], self.antenna1.ctypes.data_as(ct.POINTER(ct.c_int32)),
                      self.antenna2.ctypes.data_as(ct.POINTER(ct.c_int32)), self.time.ctypes.data_as(_dp),
                      self.freq.ctypes.data_as(_dp), self.uvw.ctypes.data_as(_dp), self.vis.ctypes.data_as(_dp))


class AKernels:
    """A-kernel table (rg_akern): freq, time [ant, nt, nf], data [ant, nt, nf,
    size_y, size_x] complex, evenly spaced axes t_min + i t_step,
    f_min + j f_step."""

    def __init__(self, freq, time, data, t_min, t_step, f_min, f_step):
        self.freq = np.ascontiguousarray(freq, np.float64)
        self.time = np.ascontiguousarray(time, np.float64)
        self.data = np.ascontiguousarray(data, np.complex128)
        self.t_min, self.t_step, self.f_min, self.f_step = float(t_min), float(t_step), float(f_min), float(f_step)

    def struct(self):
        a, t, f, sy, sx = self.data.shape
        return _AKern(a, t, f, sx, sy, self.t_min, self.t_step, self.f_min, self.f_step,
                      self.freq.ctypes.data_as(_dp), self.time.ctypes.data_as(_dp), self.data.ctypes.data_as(_dp))


_lib = None


def lib():
    """Load librg_b200.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RGError(4, f"{LIB_PATH} is not built; run radio-gridders_b200 build()")
        L = ct.CDLL(LIB_PATH)
        vp, i, d, i64 = ct.c_void_p, ct.c_int, ct.c_double, ct.c_int64
        L.rg_context_create.argtypes = [i, ct.POINTER(vp)]
        L.rg_context_destroy.argtypes = [vp]
        L.rg_context_set_stream.argtypes = [vp, vp]
        L.rg_last_error.restype = ct.c_char_p
        L.rg_last_stats.argtypes = [vp, ct.POINTER(i64), i]
        L.rg_last_stats.restype = i
        L.rg_context_set_profiling.argtypes = [vp, i]
        L.rg_context_set_autotune.argtypes = [vp, i]
        L.rg_context_set_graphs.argtypes = [vp, i]
        L.rg_last_timings.argtypes = [vp, ct.POINTER(ct.c_char_p), ct.POINTER(ct.c_float), i]
        L.rg_last_timings.restype = i
        L.rg_grid_wprojection.argtypes = [vp, vp, i, d, ct.POINTER(_Vis), ct.POINTER(_WKern), i]
        L.rg_grid_wtowers.argtypes = [vp, vp, i, d, ct.POINTER(_Vis), ct.POINTER(_WKern), i, i, d, i]
        L.rg_wtowers_tower_count.argtypes = [i, i, i]
        L.rg_wtowers_tower_count.restype = i
        L.rg_wtowers_tower_loads.argtypes = [vp, i, d, ct.POINTER(_Vis), i, i, d, vp, vp, i]
        L.rg_wtowers_partition.argtypes = [vp, vp, i, i, d, vp]
        L.rg_grid_wtowers_part.argtypes = [vp, vp, i, d, ct.POINTER(_Vis), ct.POINTER(_WKern), i, i, d, i, vp, i]
        L.rg_wkern_generate.argtypes = [vp, d, vp, i, i, i, d, i, vp]
        L.rg_grid_simple.argtypes = [vp, vp, i, d, ct.POINTER(_Vis), i]
        L.rg_grid_awprojection.argtypes = [vp, vp, i, d, ct.POINTER(_VisBL), ct.POINTER(_WKern), ct.POINTER(_AKern),
                                           i, i, i]
        L.rg_read_vis_bl_hdf5.argtypes = [ct.c_char_p, d, d, ct.POINTER(_VisBL)]
        L.rg_free_vis_bl_data.argtypes = [ct.POINTER(_VisBL)]
        L.rg_read_akern_hdf5.argtypes = [ct.c_char_p, d, ct.POINTER(_AKern)]
        L.rg_free_akern_data.argtypes = [ct.POINTER(_AKern)]
        L.rg_write_akern_hdf5.argtypes = [ct.c_char_p, d, ct.POINTER(_AKern)]
        L.rg_wstack_predict.argtypes = [vp, d, d, vp, i, vp, vp, vp, i64, d, d, d, ct.POINTER(_SepKern),
                                        ct.POINTER(_SepKern), ct.POINTER(_SepKern), ct.POINTER(_SepKern), vp]
        L.rg_pswf0.argtypes = [d, vp, i64, vp]
        L.rg_grid_wtowers_batch.argtypes = [vp, i, ct.POINTER(vp), i, d, ct.POINTER(_Vis), ct.POINTER(_WKern),
                                            i, i, d, i]
        L.rg_weight.argtypes = [vp, i, d, ct.POINTER(_Vis), vp]
        L.rg_make_hermitian.argtypes = [vp, vp, i]
        L.rg_fft_shift.argtypes = [vp, vp, i]
        L.rg_image_from_grid.argtypes = [vp, vp, i, vp, vp]
        L.rg_fft2d.argtypes = [vp, vp, i, i, i, i, i]
        L.rg_dft_image.argtypes = [vp, vp, i, d, ct.POINTER(_Vis), i, d]
        L.rg_dft_image_rows.argtypes = [vp, vp, i, d, ct.POINTER(_Vis), i, d, i, i]
        L.rg_grid_wprojection_noalloc.argtypes = [vp, i, d, ct.POINTER(_Vis), ct.POINTER(_WKern), i, vp]
        L.rg_mlp_param_count.restype = i
        L.rg_mlp_create.argtypes = [vp, i, d, d, ct.c_uint64, ct.POINTER(vp)]
        L.rg_mlp_destroy.argtypes = [vp]
        L.rg_mlp_set_params.argtypes = [vp, vp, vp]
        L.rg_mlp_get_params.argtypes = [vp, vp, vp]
        L.rg_mlp_gradient.argtypes = [vp, vp, vp, vp, i, vp, vp]
        L.rg_mlp_train.argtypes = [vp, vp, vp, vp, i64, i, i, ct.c_float, vp]
        L.rg_mlp_eval.argtypes = [vp, vp, vp, i64, vp]
        L.rg_grid_wprojection_learned.argtypes = [vp, vp, vp, i, d, ct.POINTER(_Vis), i]
        L.rg_grid_wtowers_learned.argtypes = [vp, vp, vp, i, d, ct.POINTER(_Vis), i, i, d, i]
        L.rg_read_vis_hdf5.argtypes = [ct.c_char_p, d, d, ct.POINTER(_VisData)]
        L.rg_free_vis_data.argtypes = [ct.POINTER(_VisData)]
        L.rg_free_vis_data.restype = None
        L.rg_read_wkern_hdf5.argtypes = [ct.c_char_p, d, ct.POINTER(_WKernData)]
        L.rg_free_wkern_data.argtypes = [ct.POINTER(_WKernData)]
        L.rg_free_wkern_data.restype = None
        L.rg_write_vis_hdf5.argtypes = [ct.c_char_p, i, i, i, vp, vp, vp, vp, vp, vp]
        L.rg_write_wkern_hdf5.argtypes = [ct.c_char_p, d, ct.POINTER(_WKern)]
        L.rg_write_vis_flat_hdf5.argtypes = [ct.c_char_p, i, i, vp, vp, vp, vp, vp, vp]
        L.rg_hdf5_read_f64.argtypes = [ct.c_char_p, ct.c_char_p, vp, i64, ct.POINTER(i64), ct.POINTER(i)]
        L.rg_hdf5_attr_f64.argtypes = [ct.c_char_p, ct.c_char_p, ct.c_char_p, ct.POINTER(d)]
        L.rg_selftest_wait_timeout.argtypes = [vp]
        cp = ct.c_char_p
        L.rg_wtowers_cuda_flat.argtypes = [cp, cp, vp, vp, i, d, d, d, d, i, i, d]
        L.rg_wproj_cuda_flat.argtypes = [cp, cp, vp, vp, i, d, d, d, d, i]
        L.rg_image_dft_host_flat.argtypes = [cp, vp, vp, i, d, d, d, d, i, i]
        for name in EXPORTS:
            getattr(L, name)  # raises AttributeError if a declared symbol is missing
        _lib = L
    return _lib


def _check(status):
    if status != 0:
        raise RGError(status, lib().rg_last_error().decode(errors="replace"))


def _ptr(a):
    """Address of a numpy array (must be C-contiguous) or a tensor-like."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C-contiguous")
        return a.ctypes.data
    raise TypeError(f"unsupported buffer type {type(a)}")


def _as_f64(a):
    if hasattr(a, "data_ptr"):
        return a
    return np.ascontiguousarray(a, dtype=np.float64)


def _as_c128(a):
    if hasattr(a, "data_ptr"):
        return a
    return np.ascontiguousarray(a, dtype=np.complex128)


class Visibilities:
    """Flat visibilities (struct flat_vis_data, src/common/hdf5.cuh:31-37):
    u, v, w in wavelengths (float64), vis complex128."""

    def __init__(self, u, v, w, vis):
        self.u, self.v, self.w = _as_f64(u), _as_f64(v), _as_f64(w)
        self.vis = _as_c128(vis)
        n = len(self.u) if not hasattr(self.u, "numel") else self.u.numel()
        self.n = int(n)

    def struct(self):
        return _Vis(_ptr(self.u), _ptr(self.v), _ptr(self.w), _ptr(self.vis), self.n)


def _wkern_struct(wk, data=None):
    """wk: simulate.WKernel-like (data [planes, ov, ov, size, size], w_min, w_step)."""
    arr = data if data is not None else _as_c128(wk.data)
    shape = tuple(arr.shape)
    return _WKern(_ptr(arr), int(shape[0]), int(shape[3]), int(shape[1]), float(wk.w_min),
                  float(wk.w_step)), arr


class Context:
    """A device context (streams and scratch memory), rg_context_create."""

    def __init__(self, device: int = 0):
        self._h = ct.c_void_p()
        _check(lib().rg_context_create(device, ct.byref(self._h)))

    def close(self):
        if self._h:
            lib().rg_context_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream_ptr):
        _check(lib().rg_context_set_stream(self._h, stream_ptr))

    def set_autotune(self, enabled=True):
        _check(lib().rg_context_set_autotune(self._h, int(bool(enabled))))

    def set_graphs(self, enabled=True):
        _check(lib().rg_context_set_graphs(self._h, int(bool(enabled))))

    def set_profiling(self, enabled=True):
        _check(lib().rg_context_set_profiling(self._h, 1 if enabled else 0))

    def selftest_wait_timeout(self):
        """Run the bounded tensor-core wait against an mbarrier nothing arrives
        on (rg_selftest_wait_timeout); raises RGError when the timeout path
        reports, as it should."""
        _check(lib().rg_selftest_wait_timeout(self._h))

    def last_timings(self):
        """[(stage, ms)] of the last call when profiling is enabled."""
        names = (ct.c_char_p * 64)()
        ms = (ct.c_float * 64)()
        n = lib().rg_last_timings(self._h, names, ms, 64)
        return [(names[k].decode(), float(ms[k])) for k in range(n)]

    def last_stats(self):
        out = (ct.c_int64 * 11)()
        n = lib().rg_last_stats(self._h, out, 11)
        keys = ["gridded", "active_subgrids", "towers_with_data", "floors", "dropped", "launches",
                "marked_strips", "floor_groups", "romein_points", "group_items_per_sm", "graph"]
        return {k: int(out[j]) for j, k in enumerate(keys[:n])}

    # ---- gridders (src/reference/grid.h:121-126) -------------------------
    def grid_wprojection(self, uvgrid, grid_size, theta, vis: Visibilities, wkern,
                         flags=RG_GRID_ACCUMULATE, wkern_data=None):
        s, keep = _wkern_struct(wkern, wkern_data)
        vs = vis.struct()
        _check(lib().rg_grid_wprojection(self._h, _ptr(uvgrid), int(grid_size), float(theta),
                                         ct.byref(vs), ct.byref(s), int(flags)))
        return uvgrid

    def grid_wtowers(self, uvgrid, grid_size, theta, vis: Visibilities, wkern, subgrid_size,
                     subgrid_margin, wincrement, flags=RG_GRID_ACCUMULATE, wkern_data=None):
        s, keep = _wkern_struct(wkern, wkern_data)
        vs = vis.struct()
        _check(lib().rg_grid_wtowers(self._h, _ptr(uvgrid), int(grid_size), float(theta),
                                     ct.byref(vs), ct.byref(s), int(subgrid_size),
                                     int(subgrid_margin), float(wincrement), int(flags)))
        return uvgrid

    def wkern_generate(self, theta, w_planes, size=16, oversampling=8, c=0.0, screen_pixels=128, out=None):
        """rg_wkern_generate: complex128 [planes, ov, ov, size, size] table
        (a numpy array, or `out`, which may be a device tensor)."""
        wp = np.ascontiguousarray(w_planes, np.float64)
        if out is None:
            out = np.empty((wp.size, oversampling, oversampling, size, size), np.complex128)
        _check(lib().rg_wkern_generate(self._h, float(theta), _ptr(wp), int(wp.size), int(size), int(oversampling),
                                       float(c), int(screen_pixels), _ptr(out)))
        return out

    def wstack_predict(self, theta, lam, points, u, v, w, du, dw, x0, conv_uv, conv_w, corr_lm, corr_n,
                       out=None):
        """rg_wstack_predict: complex128 visibilities of unit point sources
        (points [npts, 2] l, m) at (u, v, w).  Each table is a 2-D float64
        array [oversampling, size]."""
        pts = np.ascontiguousarray(points, np.float64).reshape(-1, 2)
        tabs = [np.ascontiguousarray(t, np.float64) for t in (conv_uv, conv_w, corr_lm, corr_n)]
        ks = [_SepKern(_ptr(t), t.shape[1], t.shape[0]) for t in tabs]
        n = int(u.shape[0]) if hasattr(u, "shape") else len(u)
        if out is None:
            out = np.zeros(n, np.complex128)
        _check(lib().rg_wstack_predict(self._h, float(theta), float(lam), _ptr(pts), int(pts.shape[0]), _ptr(u),
                                       _ptr(v), _ptr(w), n, float(du), float(dw), float(x0), ct.byref(ks[0]),
                                       ct.byref(ks[1]), ct.byref(ks[2]), ct.byref(ks[3]), _ptr(out)))
        return out

    def grid_awprojection(self, uvgrid, grid_size, theta, hv: "HierVis", wkern, akern: "AKernels", bl_min=0,
                          bl_max=None, flags=RG_GRID_ACCUMULATE):
        """rg_grid_awprojection (grid_awprojection, src/reference/grid.c:595-637)."""
        s, keep = _wkern_struct(wkern, None)
        vb, ak = hv.struct(), akern.struct()
        nbl = hv.uvw.shape[0]
        _check(lib().rg_grid_awprojection(self._h, _ptr(uvgrid), int(grid_size), float(theta), ct.byref(vb),
                                          ct.byref(s), ct.byref(ak), int(bl_min), int(nbl if bl_max is None else bl_max),
                                          int(flags)))
        return uvgrid

    # ---- one observation's towers over several GPUs ----
    def tower_loads(self, grid_size, theta, vis: Visibilities, subgrid_size, subgrid_margin, wincrement):
        """rg_wtowers_tower_loads: (visibilities, active w-floors) per tower."""
        nt = tower_count(grid_size, subgrid_size, subgrid_margin)
        nv = np.zeros(nt, np.int64)
        nf = np.zeros(nt, np.int32)
        vs = vis.struct()
        _check(lib().rg_wtowers_tower_loads(self._h, int(grid_size), float(theta), ct.byref(vs), int(subgrid_size),
                                            int(subgrid_margin), float(wincrement), _ptr(nv), _ptr(nf), nt))
        return nv, nf

    def grid_wtowers_part(self, uvgrid, grid_size, theta, vis: Visibilities, wkern, subgrid_size, subgrid_margin,
                          wincrement, part_of_tower, part, flags=RG_GRID_ACCUMULATE, wkern_data=None):
        """rg_grid_wtowers_part: the towers t with part_of_tower[t] == part."""
        s, keep = _wkern_struct(wkern, wkern_data)
        vs = vis.struct()
        pt = np.ascontiguousarray(part_of_tower, np.int32)
        if pt.size != tower_count(grid_size, subgrid_size, subgrid_margin):
            raise ValueError("part_of_tower needs one entry per tower")
        _check(lib().rg_grid_wtowers_part(self._h, _ptr(uvgrid), int(grid_size), float(theta), ct.byref(vs),
                                          ct.byref(s), int(subgrid_size), int(subgrid_margin), float(wincrement),
                                          int(flags), _ptr(pt), int(part)))
        return uvgrid

    def grid_wtowers_batch(self, uvgrids, grid_size, theta, vis_list, wkern, subgrid_size, subgrid_margin,
                           wincrement, flags=RG_GRID_ACCUMULATE, wkern_data=None):
        """rg_grid_wtowers_batch: one grid per Visibilities of vis_list, with
        the copies of neighbouring observations overlapping each pass."""
        s, keep = _wkern_struct(wkern, wkern_data)
        count = len(vis_list)
        vs = (_Vis * count)(*[v.struct() for v in vis_list])
        gp = (ct.c_void_p * count)(*[_ptr(g) for g in uvgrids])
        _check(lib().rg_grid_wtowers_batch(self._h, count, gp, int(grid_size), float(theta), vs, ct.byref(s),
                                           int(subgrid_size), int(subgrid_margin), float(wincrement), int(flags)))
        return uvgrids

    def grid_simple(self, uvgrid, grid_size, theta, vis: Visibilities, flags=RG_GRID_ACCUMULATE):
        """rg_grid_simple (grid_simple, src/reference/grid.c:83-99)."""
        vs = vis.struct()
        _check(lib().rg_grid_simple(self._h, _ptr(uvgrid), int(grid_size), float(theta), ct.byref(vs), int(flags)))
        return uvgrid

    def weight(self, grid_size, theta, vis: Visibilities, out=None):
        if out is None:
            out = np.empty(vis.n, np.complex128)
        vs = vis.struct()
        _check(lib().rg_weight(self._h, int(grid_size), float(theta), ct.byref(vs), _ptr(out)))
        return out

    # ---- image formation (src/reference/grid.c:639-680, main.c:258-294) ----
    def make_hermitian(self, uvgrid):
        _check(lib().rg_make_hermitian(self._h, _ptr(uvgrid), int(uvgrid.shape[0])))
        return uvgrid

    def fft_shift(self, uvgrid):
        _check(lib().rg_fft_shift(self._h, _ptr(uvgrid), int(uvgrid.shape[0])))
        return uvgrid

    def image_from_grid(self, uvgrid, image=None, taper_1d=None):
        n = int(uvgrid.shape[0])
        if image is None:
            image = np.empty((n, n), np.float64)
        t = None if taper_1d is None else np.ascontiguousarray(taper_1d, np.float64)
        _check(lib().rg_image_from_grid(self._h, _ptr(uvgrid), n, _ptr(image), _ptr(t)))
        return image

    def fft2d(self, data, sign):
        """Batched 2-D FFT in place on [batch, ny, nx] complex64/complex128."""
        shape = data.shape
        batch = int(np.prod(shape[:-2])) if len(shape) > 2 else 1
        cb = 8 if str(data.dtype).endswith("complex64") else 16
        _check(lib().rg_fft2d(self._h, _ptr(data), batch, int(shape[-2]), int(shape[-1]),
                              int(sign), cb))
        return data

    # ---- direct DFT (src/dft/dft_cuda.cu) ----------------------------------
    def dft_image(self, grid_size, theta, vis: Visibilities, precision=RG_DFT_FP64_REDUCED,
                  factor=2.0, image=None):
        if image is None:
            image = np.empty((grid_size, grid_size), np.float64)
        vs = vis.struct()
        _check(lib().rg_dft_image(self._h, _ptr(image), int(grid_size), float(theta),
                                  ct.byref(vs), int(precision), float(factor)))
        return image

    def dft_image_rows(self, grid_size, theta, vis: Visibilities, row0, nrows,
                       precision=RG_DFT_FP64_REDUCED, factor=2.0, image=None):
        """Rows [row0, row0 + nrows) of dft_image (one rank's share)."""
        if image is None:
            image = np.empty((nrows, grid_size), np.float64)
        vs = vis.struct()
        _check(lib().rg_dft_image_rows(self._h, _ptr(image), int(grid_size), float(theta),
                                       ct.byref(vs), int(precision), float(factor), int(row0), int(nrows)))
        return image


class LearnedKernel:
    """The learned w-kernel network (rg_mlp_*): tap(w, du, dv, tx, ty)."""

    def __init__(self, ctx: "Context", ksize=16, wmax=2000.0, out_scale=0.05, seed=0):
        self.ctx = ctx
        self.ksize, self.wmax, self.out_scale = ksize, wmax, out_scale
        self._h = ct.c_void_p()
        _check(lib().rg_mlp_create(ctx.handle, ksize, float(wmax), float(out_scale), int(seed),
                                   ct.byref(self._h)))

    def close(self):
        if self._h:
            lib().rg_mlp_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    @staticmethod
    def samples(w, du, dv, tx, ty):
        return np.ascontiguousarray(np.stack([w, du, dv, tx, ty]).astype(np.float32))

    @staticmethod
    def targets(taps):
        t = np.asarray(taps, np.complex128)
        return np.ascontiguousarray(np.stack([t.real, t.imag], axis=-1).astype(np.float32))

    def get_params(self):
        out = np.empty(lib().rg_mlp_param_count(), np.float32)
        _check(lib().rg_mlp_get_params(self.ctx.handle, self._h, _ptr(out)))
        return out

    def set_params(self, params):
        p = np.ascontiguousarray(params, np.float32)
        _check(lib().rg_mlp_set_params(self.ctx.handle, self._h, _ptr(p)))

    def gradient(self, samples, targets):
        n = samples.shape[1]
        g = np.empty(lib().rg_mlp_param_count(), np.float32)
        loss = np.zeros(1, np.float32)
        _check(lib().rg_mlp_gradient(self.ctx.handle, self._h, _ptr(samples), _ptr(targets), int(n),
                                     _ptr(g), _ptr(loss)))
        return float(loss[0]), g

    def train(self, samples, targets, batch=16384, steps=100, lr=1e-3):
        n = samples.shape[1] if not hasattr(samples, "data_ptr") else samples.shape[1]
        loss = np.zeros(1, np.float32)
        _check(lib().rg_mlp_train(self.ctx.handle, self._h, _ptr(samples), _ptr(targets), int(n),
                                  int(batch), int(steps), ct.c_float(lr), _ptr(loss)))
        return float(loss[0])

    def eval(self, samples):
        n = samples.shape[1]
        out = np.empty((n, 2), np.float32)
        _check(lib().rg_mlp_eval(self.ctx.handle, self._h, _ptr(samples), int(n), _ptr(out)))
        return out[:, 0].astype(np.complex128) + 1j * out[:, 1]


def grid_wprojection_learned(ctx, mlp, uvgrid, grid_size, theta, vis, flags=RG_GRID_ACCUMULATE):
    vs = vis.struct()
    _check(lib().rg_grid_wprojection_learned(ctx.handle, mlp.handle, _ptr(uvgrid), int(grid_size),
                                             float(theta), ct.byref(vs), int(flags)))
    return uvgrid


def grid_wtowers_learned(ctx, mlp, uvgrid, grid_size, theta, vis, subgrid_size, subgrid_margin, wincrement,
                         flags=RG_GRID_ACCUMULATE):
    """W-towers with the learned kernel (rg_grid_wtowers_learned)."""
    vs = vis.struct()
    _check(lib().rg_grid_wtowers_learned(ctx.handle, mlp.handle, _ptr(uvgrid), int(grid_size), float(theta),
                                         ct.byref(vs), int(subgrid_size), int(subgrid_margin), float(wincrement),
                                         int(flags)))
    return uvgrid


_default = None


def default_context() -> Context:
    global _default
    if _default is None:
        _default = Context(0)
    return _default


# Module-level mirror of the reference's function names ----------------------

def grid_wprojection(uvgrid, grid_size, theta, vis, wkern):
    return default_context().grid_wprojection(uvgrid, grid_size, theta, vis, wkern)


def grid_wtowers(uvgrid, grid_size, theta, vis, wkern, subgrid_size, subgrid_margin, wincrement):
    return default_context().grid_wtowers(uvgrid, grid_size, theta, vis, wkern, subgrid_size,
                                          subgrid_margin, wincrement)


def pswf0(c, x):
    """rg_pswf0 (host only): psi_0(c, x) / psi_0(c, 0) for x in [-1, 1]."""
    xa = np.ascontiguousarray(x, np.float64)
    out = np.empty_like(xa)
    _check(lib().rg_pswf0(float(c), _ptr(xa), int(xa.size), _ptr(out)))
    return out


def tower_count(grid_size, subgrid_size, subgrid_margin):
    """rg_wtowers_tower_count: towers of a W-towers shape (row-major)."""
    return int(lib().rg_wtowers_tower_count(int(grid_size), int(subgrid_size), int(subgrid_margin)))


def partition_towers(vis_per_tower, floors_per_tower, nparts, vis_per_floor=0.0):
    """rg_wtowers_partition (host only): part index per tower, balanced by
    visibilities + vis_per_floor * active floors, largest first."""
    nv = np.ascontiguousarray(vis_per_tower, np.int64)
    nf = np.ascontiguousarray(floors_per_tower, np.int32)
    out = np.zeros(nv.size, np.int32)
    _check(lib().rg_wtowers_partition(_ptr(nv), _ptr(nf), int(nv.size), int(nparts), float(vis_per_floor),
                                      _ptr(out)))
    return out


def weight(grid_size, theta, vis):
    return default_context().weight(grid_size, theta, vis)


def make_hermitian(uvgrid):
    return default_context().make_hermitian(uvgrid)


def fft_shift(uvgrid):
    return default_context().fft_shift(uvgrid)


def image_from_grid(uvgrid, taper_1d=None):
    return default_context().image_from_grid(uvgrid, taper_1d=taper_1d)


def dft_image(grid_size, theta, vis, precision=RG_DFT_FP64_REDUCED, factor=2.0):
    return default_context().dft_image(grid_size, theta, vis, precision, factor)


# Crocodile HDF5 files (host only: no device is touched) ----------------------

class FileWKernel:
    """An oversampled w-kernel table read from a file: data complex128
    [planes, ov, ov, size, size], planes at w_min + i*w_step."""

    def __init__(self, data, w_min, w_step):
        self.data, self.w_min, self.w_step = data, w_min, w_step

    @property
    def plane_count(self):
        return int(self.data.shape[0])

    @property
    def oversampling(self):
        return int(self.data.shape[1])

    @property
    def size(self):
        return int(self.data.shape[3])

    @property
    def w_max(self):
        return self.w_min + (self.plane_count - 1) * self.w_step


def read_vis_hdf5(path, bl_min=0.0, bl_max=float("inf")):
    """Flat visibilities of a crocodile visibility file (load_vis +
    flatten_visibilities_CUDA, src/reference/hdf5.c:173-318,
    src/common/hdf5.c:827-872).  Returns (Visibilities, baseline count)."""
    L, d = lib(), _VisData()
    _check(L.rg_read_vis_hdf5(os.fsencode(path), float(bl_min), float(min(bl_max, 1.7976931348623157e308)),
                              ct.byref(d)))
    try:
        n = int(d.n)
        take = (lambda p, k: np.ctypeslib.as_array(p, shape=(k,)).copy()) if n else (lambda p, k: np.zeros(k))
        vis = Visibilities(take(d.u, n), take(d.v, n), take(d.w, n), take(d.vis, 2 * n).view(np.complex128))
        return vis, int(d.bl_count)
    finally:
        L.rg_free_vis_data(ct.byref(d))


def read_wkern_hdf5(path, theta):
    """The w-kernel table of a crocodile kernel file (load_wkern,
    src/reference/hdf5.c:321-413)."""
    L, d = lib(), _WKernData()
    _check(L.rg_read_wkern_hdf5(os.fsencode(path), float(theta), ct.byref(d)))
    try:
        shape = (d.plane_count, d.oversampling, d.oversampling, d.size, d.size)
        flat = np.ctypeslib.as_array(d.data, shape=(2 * int(np.prod(shape)),)).copy()
        return FileWKernel(flat.view(np.complex128).reshape(shape), float(d.w_min), float(d.w_step))
    finally:
        L.rg_free_wkern_data(ct.byref(d))


def write_vis_hdf5(path, ant1, ant2, time, freq, uvw, vis):
    """Hierarchical visibility file: uvw [bl, time, 3] metres, freq [bl, nf] Hz,
    vis [bl, time, nf] complex, time [bl, time]."""
    uvw = np.ascontiguousarray(uvw, np.float64)
    n_bl, n_time = uvw.shape[:2]
    freq = np.ascontiguousarray(freq, np.float64).reshape(n_bl, -1)
    vis = np.ascontiguousarray(vis, np.complex128).reshape(n_bl, n_time, freq.shape[1])
    a1 = np.ascontiguousarray(ant1, np.int32)
    a2 = np.ascontiguousarray(ant2, np.int32)
    t = np.ascontiguousarray(time, np.float64).reshape(n_bl, n_time)
    _check(lib().rg_write_vis_hdf5(os.fsencode(path), n_bl, n_time, freq.shape[1], _ptr(a1), _ptr(a2),
                                   _ptr(t), _ptr(freq), _ptr(uvw), _ptr(vis)))


def write_vis_flat_hdf5(path, ant1, ant2, time, freq, uvw, vis):
    """Legacy flat visibility file: one row per time sample, uvw [rows, 3]
    metres, a shared frequency axis freq [nf] Hz, vis [rows, nf] complex."""
    uvw = np.ascontiguousarray(uvw, np.float64).reshape(-1, 3)
    rows = uvw.shape[0]
    freq = np.ascontiguousarray(freq, np.float64).ravel()
    vis = np.ascontiguousarray(vis, np.complex128).reshape(rows, freq.size)
    a1 = np.ascontiguousarray(ant1, np.int32)
    a2 = np.ascontiguousarray(ant2, np.int32)
    t = np.ascontiguousarray(time, np.float64).ravel()
    _check(lib().rg_write_vis_flat_hdf5(os.fsencode(path), rows, freq.size, _ptr(a1), _ptr(a2), _ptr(t), _ptr(freq),
                                        _ptr(uvw), _ptr(vis)))


def write_wkern_hdf5(path, theta, wkern):
    st, keep = _wkern_struct(wkern)
    _check(lib().rg_write_wkern_hdf5(os.fsencode(path), float(theta), ct.byref(st)))
    del keep


def read_vis_bl_hdf5(path, bl_min=0.0, bl_max=float("inf")):
    """Hierarchical visibilities of a crocodile file (rg_read_vis_bl_hdf5)."""
    L, d = lib(), _VisBL()
    _check(L.rg_read_vis_bl_hdf5(os.fsencode(path), float(bl_min), float(min(bl_max, 1.7976931348623157e308)),
                                 ct.byref(d)))
    try:
        nb, nt, nf = int(d.bl_count), int(d.time_count), int(d.freq_count)

        def take(p, k, dt=np.float64):
            return np.ctypeslib.as_array(p, shape=(k,)).copy() if k else np.zeros(0, dt)
        return HierVis(take(d.antenna1, nb, np.int32), take(d.antenna2, nb, np.int32),
                       take(d.time, nb * nt).reshape(nb, nt), take(d.freq, nb * nf).reshape(nb, nf),
                       take(d.uvw, nb * nt * 3).reshape(nb, nt, 3),
                       take(d.vis, 2 * nb * nt * nf).view(np.complex128).reshape(nb, nt, nf))
    finally:
        L.rg_free_vis_bl_data(ct.byref(d))


def read_akern_hdf5(path, theta):
    """The A-kernel table of a crocodile A-kernel file (rg_read_akern_hdf5)."""
    L, d = lib(), _AKern()
    _check(L.rg_read_akern_hdf5(os.fsencode(path), float(theta), ct.byref(d)))
    try:
        a, t, f, sy, sx = d.antenna_count, d.time_count, d.freq_count, d.size_y, d.size_x
        k = a * t * f
        data = np.ctypeslib.as_array(d.data, shape=(2 * k * sy * sx,)).copy().view(np.complex128)
        return AKernels(np.ctypeslib.as_array(d.freq, shape=(k,)).copy().reshape(a, t, f),
                        np.ctypeslib.as_array(d.time, shape=(k,)).copy().reshape(a, t, f),
                        data.reshape(a, t, f, sy, sx), d.t_min, d.t_step, d.f_min, d.f_step)
    finally:
        L.rg_free_akern_data(ct.byref(d))


def write_akern_hdf5(path, theta, akern: AKernels):
    st = akern.struct()
    _check(lib().rg_write_akern_hdf5(os.fsencode(path), float(theta), ct.byref(st)))


def hdf5_read(path, dataset):
    """A float64 / int64 / {r, i} dataset of any crocodile file as float64
    (complex compounds come back with a trailing axis of 2)."""
    L = lib()
    dims, nd = (ct.c_int64 * 8)(), ct.c_int(8)
    _check(L.rg_hdf5_read_f64(os.fsencode(path), dataset.encode(), None, 0, dims, ct.byref(nd)))
    shape = tuple(dims[k] for k in range(nd.value))
    out = np.empty(int(np.prod(shape)) if shape else 1, np.float64)
    _check(L.rg_hdf5_read_f64(os.fsencode(path), dataset.encode(), _ptr(out), out.size, dims, ct.byref(nd)))
    shape = tuple(dims[k] for k in range(nd.value))
    return out.reshape(shape)


def hdf5_attr(path, obj, name):
    v = ct.c_double()
    _check(lib().rg_hdf5_attr_f64(os.fsencode(path), obj.encode(), name.encode(), ct.byref(v)))
    return v.value
