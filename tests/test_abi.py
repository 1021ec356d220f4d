"""The C-ABI library loads and exports every entry point include/coqui_b200.h declares
(no compute calls; the library is built by the driver's build step / conftest)."""
import ctypes
import os
import re

import pytest

from coqui_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_symbols():
    txt = open(os.path.join(ROOT, "include", "coqui_b200.h")).read()
    return sorted(set(re.findall(r"\b(coqui_b200_[a-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(capi.LIB_PATH):
        from coqui_b200 import build
        build.build(verbose=False)
    return capi.load()


def test_header_and_binding_agree():
    assert _header_symbols() == sorted(capi.SYMBOLS)


def test_library_exports_every_header_symbol(lib):
    for name in _header_symbols():
        assert hasattr(lib, name), name


def test_version(lib):
    assert "sm_100a" in capi.version()


def test_bad_dims_rejected_without_device(lib):
    d = capi.Dims(ns=2, nk=8, nb=4, Np=4, nt_f=10, nw_b=11,
                  kp_grid=(ctypes.c_int64 * 3)(2, 2, 2), precision_mode=1, device=0)
    h = ctypes.c_void_p()
    assert lib.coqui_b200_create(ctypes.byref(h), ctypes.byref(d)) == -1  # ns != 1
    d.ns = 1
    d.kp_grid = (ctypes.c_int64 * 3)(2, 2, 3)  # product != nk
    assert lib.coqui_b200_create(ctypes.byref(h), ctypes.byref(d)) == -1
    assert not h.value


def test_null_context_is_an_error(lib):
    assert lib.coqui_b200_set_thc(None, None, None) == -1
    assert lib.coqui_b200_kernel_launches(None) == 0


def test_tile_configuration_pinning_validates_its_argument(lib):
    n = capi.num_tile_configs()
    assert n >= 6
    with pytest.raises(ValueError):
        capi.set_tile_config(n)
    with pytest.raises(ValueError):
        capi.set_tile_config(-2)
    capi.set_tile_config(n - 1)
    capi.set_tile_config(-1)


def test_noalloc_rejects_wrapping_shapes_before_any_device_work(lib):
    """Dimensions whose byte counts would wrap around a 64-bit size are rejected by the
    argument check (EINVAL), which runs before the library touches the device."""
    for nk, Np, nb in ((1, 1 << 61, 1), (1 << 40, 1 << 40, 1), (1, 1, 1 << 62), (3, 1 << 62, 5)):
        with pytest.raises(capi.CoquiB200Error) as e:
            capi.primary_to_aux_noalloc(1, 1, 1, nk, Np, nb)
        assert e.value.code == -1 and "static limit" in str(e.value)
