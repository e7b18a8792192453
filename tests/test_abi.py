"""CPU tests of the C ABI boundary: the library loads, exports every function
include/ocp_flash.h declares, and validates its arguments before touching a
device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from opencaeporo_b200 import _lib
from opencaeporo_b200.fluid import spe5_fluid, synthetic_fluid

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ocp_flash.h")


def _declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ocpf_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_exports():
    assert _declared() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    for name in _declared():
        assert hasattr(L, name), name
    assert b"sm_100a" in L.ocpf_version()


def test_struct_layout_matches_header():
    # ocpf_fluid: 8 int32 + 6 doubles + 8*16 + 256 + 5 + 5 + 1 doubles
    assert C.sizeof(_lib.Fluid) == 8 * 4 + 8 * (6 + 8 * 16 + 256 + 11)
    assert C.sizeof(_lib.FimIn) == 6 * 8
    assert C.sizeof(_lib.Skip) == 5 * 8
    assert C.sizeof(_lib.FimOut) == len(_lib.OUT_FIELDS) * 8
    txt = open(HEADER).read()
    end = txt.index("} ocpf_fim_out;")
    body = txt[txt.rindex("typedef struct {", 0, end):end]
    fields = re.findall(r"\*\s*([A-Za-z_]+);", body)
    assert tuple(fields[-len(_lib.OUT_FIELDS):]) == _lib.OUT_FIELDS


@pytest.mark.parametrize("mutate", ["nc_low", "nc_high", "neg_tc", "asym_bic", "neg_maxit"])
def test_create_rejects_invalid_fluid(mutate):
    fl = _lib.make_fluid(spe5_fluid())
    if mutate == "nc_low":
        fl.nc = 1
    elif mutate == "nc_high":
        fl.nc = 17
    elif mutate == "neg_tc":
        fl.Tc[2] = -1.0
    elif mutate == "asym_bic":
        fl.BIC[1] = 0.3
    elif mutate == "neg_maxit":
        fl.rr_maxit = -1
    h = C.c_void_p()
    rc = _lib.lib().ocpf_create(C.byref(fl), 0, C.byref(h))
    assert rc == _lib.OCPF_EINVAL
    assert not h.value


def test_null_arguments_rejected():
    L = _lib.lib()
    assert L.ocpf_create(None, 0, None) == _lib.OCPF_EINVAL
    assert L.ocpf_destroy(None) == _lib.OCPF_EINVAL
    assert L.ocpf_flash_fim(None, 0, None, None, None, 0, None) == _lib.OCPF_EINVAL
    assert L.ocpf_flash_fim_host(None, 0, None, None, None, 0) == _lib.OCPF_EINVAL
    assert L.ocpf_last_kernel_ms(None, None) == _lib.OCPF_EINVAL


def test_status_strings():
    L = _lib.lib()
    for code in range(5):
        assert L.ocpf_status_string(code)
    assert L.ocpf_status_string(99) == b"unknown"


def test_unsupported_nc_reported():
    """Component counts without a compiled kernel are refused up front."""
    fl = _lib.make_fluid(synthetic_fluid(5, 1))
    h = C.c_void_p()
    assert _lib.lib().ocpf_create(C.byref(fl), 0, C.byref(h)) == _lib.OCPF_EUNSUPPORTED


def test_fluid_conversion_roundtrip():
    fl = synthetic_fluid(6, 1234)
    f = _lib.make_fluid(fl)
    assert f.nc == 6
    np.testing.assert_array_equal(np.array(f.Tc[:6]), fl.Tc)
    np.testing.assert_array_equal(np.array(f.BIC[:36]).reshape(6, 6), fl.BIC)
