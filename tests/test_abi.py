"""The C-ABI library loads and exports every function include/hkb.h declares.
No compute call here: this file runs without a GPU."""
import ctypes
import os

import pytest

import hkb


def test_library_exports_every_declared_symbol():
    names = hkb.header_functions()
    assert len(names) >= 20
    L = ctypes.CDLL(hkb.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_library_is_sm100a_build():
    # the fatbin is built for sm_100a only (Makefile ARCH); the version
    # string names the target
    assert b"sm_100a" in hkb.lib().hk_version()


def test_create_without_device_reports_cuda_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(hkb.HkError) as ei:
        hkb.Context(0)
    assert ei.value.status in (-5, -1)


def test_null_context_is_rejected():
    L = hkb.lib()
    assert L.hk_set_grid(None, 0.0, 1.0, 0.1, 1, 0, 1.0, 0.0) == -1
    assert L.hk_num_lines(None) == 0
    assert L.hk_last_error(None) == b"null context"
