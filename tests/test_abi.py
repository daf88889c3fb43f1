"""The C-ABI library loads without a GPU, exports every declared entry point, and its ctypes
mirror matches the C struct; argument errors are reported before any CUDA call."""

from __future__ import annotations

import ctypes
import re

import pytest

from ac_fdtd_b200 import _native
from tests.conftest import ROOT

HEADER = ROOT / "include" / "acfdtd_b200.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(acf_\w+)\s*\(", text, re.M)))


def test_every_declared_symbol_is_exported_and_bound():
    lib = _native.library()
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(names) == sorted(_native.EXPORTED_SYMBOLS)


def test_struct_mirror_and_version():
    lib = _native.library()
    assert lib.acf_abi_version() == 1
    assert lib.acf_struct_size() == ctypes.sizeof(_native.AcfConfig)


@pytest.mark.parametrize("field,value,needle", [
    ("nx", 0, "cell counts"),
    ("precision", 2, "precision"),
    ("n_relax", 5, "at most 4"),
])
def test_bad_configs_are_refused_with_a_message(field, value, needle):
    lib = _native.library()
    config = _native.AcfConfig()
    config.nx = config.ny = config.nz = 4
    config.precision = 8
    setattr(config, field, value)
    handle = ctypes.c_void_p()
    status = lib.acf_create(ctypes.byref(config), ctypes.byref(handle))
    assert status == 1
    assert needle in lib.acf_last_error().decode()
    with pytest.raises(_native.NativeError, match=needle):
        _native.check(status, "acf_create")


def test_null_arguments_are_refused():
    lib = _native.library()
    assert lib.acf_create(None, None) == 1
    assert lib.acf_run(None, 1, 0, None) == 1
    assert lib.acf_upload(None, 0, None, None) == 1
    assert lib.acf_launch_count(None) == -1
    assert lib.acf_set_wait_test(None, 0, -1) == 1
    assert lib.acf_batch_device_status(None, None) == 1
    assert lib.acf_device_status(None, None) == 1
    assert lib.acf_set_time_blocking(None, 2) == 1
    assert lib.acf_get_time_blocking(None) == -1
