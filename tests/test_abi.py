"""The C-ABI library loads and exports every symbol include/radio_gridders.h
declares (no compute calls: this runs without a GPU)."""
import ctypes as ct
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = []
    for fn in os.listdir(os.path.join(REPO, "include")):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(REPO, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"\b(rg_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = header_functions()
    for need in ("rg_grid_wprojection", "rg_grid_wtowers", "rg_dft_image", "rg_image_from_grid",
                 "rg_weight", "rg_make_hermitian", "rg_fft_shift"):
        assert need in names


def test_library_exports_every_declared_symbol(rg):
    lib = ct.CDLL(rg.LIB_PATH)
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_python_mirror_binds_every_symbol(rg):
    assert set(header_functions()) <= set(rg.EXPORTS)


def test_no_device_is_reported_not_faked(rg):
    """Without a GPU the library reports it; there is no CPU fallback."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(rg.RGError) as e:
        rg.Context(0)
    assert e.value.status == 6


def test_reference_wrapper_entries_reject_null_arguments():
    """The file-level entries with the reference wrappers' argument lists
    check their pointers before touching CUDA or the files, and report
    RG_ERR_INVALID_ARGUMENT instead of exiting."""
    import importlib
    rg = importlib.import_module("radio-gridders_b200")
    L = rg.lib()
    assert L.rg_wtowers_cuda_flat(None, b"wk.h5", None, None, 64, 0.1, 640.0, 0.0, 1e30, 32, 8, 10.0) == 1
    assert L.rg_wproj_cuda_flat(b"vis.h5", None, ct.c_void_p(1), None, 64, 0.1, 640.0, 0.0, 1e30, 256) == 1
    assert L.rg_image_dft_host_flat(b"vis.h5", None, None, 64, 0.1, 640.0, 0.0, 1e30, 1, 1) == 1
    assert b"NULL" in L.rg_last_error() or b"buffer" in L.rg_last_error()
