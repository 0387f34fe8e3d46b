"""The C ABI library (CPU-only checks: no compute without a GPU).

* libxsec_b200.so loads and exports every function include/xsec_b200.h
  declares;
* without a usable sm_100 device the product fails loudly -- there is no CPU
  fallback -- and argument errors are reported as status codes.
"""
import ctypes
import os

import pytest

from gpu_cross_b200 import build, capi


def test_library_is_built_in_tree(built_libs):
    assert os.path.exists(capi.library_path())
    assert capi.library_path().startswith(os.path.dirname(build.__file__))


def test_every_declared_symbol_is_exported(built_libs):
    names = capi.declared_functions()
    assert len(names) >= 30
    lib = ctypes.CDLL(capi.library_path())
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes binding covers all of them
    assert set(names) <= set(capi._SIGS), set(names) - set(capi._SIGS)


def test_version(built_libs):
    assert b"sm_100a" in capi.lib().xs_version()


def _no_gpu():
    try:
        import torch

        return not torch.cuda.is_available()
    except Exception:
        return True


@pytest.mark.skipif(not _no_gpu(), reason="checks the behaviour on a machine without a GPU")
def test_no_cpu_fallback_without_device(built_libs):
    assert capi.device_available() is False
    with pytest.raises(capi.XsError) as ei:
        capi.Engine(0)
    assert ei.value.code == capi.XS_ERR_NODEVICE
    with pytest.raises(capi.XsError) as ei:
        capi.Manager(0, capi.VOIGT)
    assert ei.value.code == capi.XS_ERR_NODEVICE


def test_null_arguments_are_status_codes(built_libs):
    lib = capi.lib()
    assert lib.xs_engine_execute(None, None, None, 0, None, None, None, 0) == capi.XS_ERR_INVALID
    assert lib.xs_engine_create(0, None) == capi.XS_ERR_INVALID
    assert lib.xs_manager_create(0, capi.VOIGT, 0, 1, 0, None) == capi.XS_ERR_INVALID
    assert lib.xs_copy_intensity_info(None) == capi.XS_ERR_INVALID
    assert lib.xs_graph_launch(None, None) == capi.XS_ERR_INVALID
    assert b"NULL" in lib.xs_last_error()


def test_unsupported_profiles_rejected_before_device_work(built_libs):
    lib = capi.lib()
    h = ctypes.c_void_p()
    # PSUEDO_VOIGT is not implemented (nor in the reference, OpenMPManager.cpp:110-112)
    assert lib.xs_manager_create(0, capi.PSUEDO_VOIGT, 0, 1, 0, ctypes.byref(h)) == \
        capi.XS_ERR_UNSUPPORTED
    # the reference CPU backend has no GAUSSIAN
    assert lib.xs_manager_create(1, capi.GAUSSIAN, 0, 1, 0, ctypes.byref(h)) == \
        capi.XS_ERR_UNSUPPORTED


def test_scratch_bytes_needed_scales_with_lines_and_conditions(built_libs):
    o = capi.make_options(capi.VOIGT, 0.01, 17.0, precision=capi.MIXED)
    a = capi.lib().xs_scratch_bytes_needed(ctypes.byref(o), 1, 1_000_000)
    b = capi.lib().xs_scratch_bytes_needed(ctypes.byref(o), 4, 1_000_000)
    c = capi.lib().xs_scratch_bytes_needed(ctypes.byref(o), 1, 2_000_000)
    # per line and condition: a 64-byte record and a window (8 bytes); per
    # line: its nearest grid index (4 bytes)
    assert abs(a - 76 * 1_000_000) < 4096
    assert abs(b - (4 * 72 + 4) * 1_000_000) < 4096 and abs(c - 2 * a) < 4096
