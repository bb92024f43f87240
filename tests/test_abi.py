"""The C-ABI library builds for sm_100a, loads without a GPU, and exports every
entry point include/gascoigne_b200.h declares (no compute calls here)."""
import ctypes
import os

import pytest

from gascoignelib_b200 import native
from gascoignelib_b200.build import build_library


@pytest.fixture(scope="module")
def so_path():
    return build_library()


def test_library_exports_every_declared_symbol(so_path):
    L = ctypes.CDLL(so_path)
    names = native.declared_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_header():
    names = set(native.declared_symbols())
    bound = set(native._SIGS) | {"gb_last_error_string"}
    assert names == bound, names ^ bound


def test_library_is_built_for_sm100a():
    from gascoignelib_b200.build import NVCC_FLAGS
    assert "arch=compute_100a,code=sm_100a" in NVCC_FLAGS
    assert not any("compute_" in f and "100a" not in f for f in NVCC_FLAGS)


@pytest.mark.gpu
def test_kernels_run_as_sm100(so_path):
    """The kernels the device loads carry compute capability 10.0 (sm_100a),
    read at run time from a kernel's attributes."""
    L = ctypes.CDLL(so_path)
    bv, pv = ctypes.c_int(0), ctypes.c_int(0)
    assert L.gb_kernel_arch(ctypes.byref(bv), ctypes.byref(pv)) == 0
    assert bv.value == 100, bv.value


def test_structs_match_header():
    txt = open(native.HEADER).read()
    for f, _ in native.GbParams._fields_:
        assert f in txt
    for f, _ in native.GbSolveInfo._fields_:
        assert f in txt


def test_context_create_fails_cleanly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(native.GBError):
        native.Context(0)
