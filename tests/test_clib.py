"""libwap.so loads without a GPU, exports every symbol of include/wap.h, and
rejects bad arguments before touching the device."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "wap.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(wap_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from wideanglepropagation_b200 import build, _lib
    build.build()
    return _lib.lib()


def test_header_declares_entry_points():
    names = header_functions()
    for want in ("wap_plan_create", "wap_multislice_fwd", "wap_wpm_fwd", "wap_multislice_bwd",
                 "wap_transfer_function", "wap_last_error"):
        assert want in names


def test_every_declared_symbol_is_exported(lib):
    for name in header_functions():
        assert hasattr(lib, name), name


def test_python_binding_covers_header():
    from wideanglepropagation_b200 import _lib
    assert set(header_functions()) <= set(_lib.SIGNATURES)


def test_version_and_no_error(lib):
    assert b"sm_100a" in lib.wap_version()
    assert lib.wap_last_error() == b""


@pytest.mark.parametrize("ny,nx", [(16, 64), (4096, 64), (0, 64), (1025, 128), (128, 2000), (64, 12)])
def test_unsupported_grid(lib, ny, nx):
    from wideanglepropagation_b200 import _lib
    h = ctypes.c_void_p()
    rc = lib.wap_plan_create(ctypes.byref(h), ny, nx, 1, 0, 0)
    assert rc == _lib.WAP_ERR_UNSUPPORTED
    assert b"unsupported grid" in lib.wap_last_error()
    assert not h.value


@pytest.mark.parametrize("ny,nx", [(100, 128), (128, 96), (17, 1024), (1000, 2048)])
def test_generic_grids_pass_the_size_check(lib, ny, nx):
    """Sides that are not powers of two (17 .. 1024) take the Bluestein path:
    the size check accepts them (without a device the plan then fails on its
    first CUDA call, never as an unsupported size)."""
    from wideanglepropagation_b200 import _lib
    h = ctypes.c_void_p()
    rc = lib.wap_plan_create(ctypes.byref(h), ny, nx, 1, 0, 0)
    assert rc != _lib.WAP_ERR_UNSUPPORTED
    if rc == _lib.WAP_OK:
        lib.wap_plan_destroy(h)


def test_bad_arguments(lib):
    from wideanglepropagation_b200 import _lib
    assert lib.wap_plan_create(None, 64, 64, 1, 0, 0) == _lib.WAP_ERR_ARG
    h = ctypes.c_void_p()
    assert lib.wap_plan_create(ctypes.byref(h), 64, 64, 0, 0, 0) == _lib.WAP_ERR_ARG
    assert lib.wap_plan_create(ctypes.byref(h), 64, 64, 1, 7, 0) == _lib.WAP_ERR_ARG
    assert lib.wap_plan_create(ctypes.byref(h), 64, 64, 1, 1, 1) == _lib.WAP_ERR_ARG   # WPM needs >= 2 bins
    assert lib.wap_transfer_function(5, 8, 8, 0.1, 0.1, 1.0, 2e5, None, 0, None, None) == _lib.WAP_ERR_ARG
    assert lib.wap_multislice_fwd(None, None, 1, 1, None, None, 1, 0, None, None, None, 1.0, 2e5,
                                  None, None, None, None) == _lib.WAP_ERR_ARG
    assert b"plan is NULL" in lib.wap_last_error()
    n = ctypes.c_longlong()
    assert lib.wap_profile_read(0, None, None, None) == _lib.WAP_ERR_ARG
    assert lib.wap_plan_destroy(None) == 0


def test_check_maps_codes_to_exceptions(lib):
    from wideanglepropagation_b200 import _lib
    h = ctypes.c_void_p()
    with pytest.raises(ValueError, match="unsupported grid"):
        _lib.check(lib.wap_plan_create(ctypes.byref(h), 100, 2000, 1, 0, 0))


def test_launch_counter_starts_at_zero(lib):
    assert lib.wap_launch_count() >= 0
