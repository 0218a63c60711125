"""The C ABI: the library loads without a GPU and exports every symbol
include/dynb200.h declares (no compute calls here)."""
import os
import re

from dynamics_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "dynb200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(dyn_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    names = declared_symbols()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.EXPORTED)


def test_calls_without_gpu_do_not_abort():
    lib = _lib.lib()
    assert lib.dyn_version() >= 1
    assert lib.dyn_device_count() >= 0
    assert lib.dyn_sys_step(None, 1, 0.002) == _lib.DYN_ERR_INVALID
    assert b"NULL" in lib.dyn_last_error()
