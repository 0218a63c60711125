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


def _header_defines():
    src = open(os.path.join(ROOT, "include", "dynb200.h")).read()
    out = {}
    for name, val in re.findall(r"^#define\s+(DYN_[A-Z0-9_]+)\s+\(?(-?\d+)u?\)?", src, flags=re.M):
        out[name] = int(val)
    return out


def test_python_constants_match_the_header():
    defs = _header_defines()
    assert len(defs) >= 30
    for name, val in defs.items():
        if hasattr(_lib, name):
            assert getattr(_lib, name) == val, name
    for name in ("DYN_PAIR_ALCH", "DYN_SNAP_FORCES", "DYN_FLAG_RATTLE_VELOCITIES", "DYN_ERR_TIMEOUT"):
        assert hasattr(_lib, name), name


def test_struct_layouts_match_the_header(tmp_path):
    """The ctypes mirrors have the C structs' size and their fields' offsets
    (compiled with the host C compiler against the header)."""
    import ctypes as C
    import shutil
    import subprocess

    import pytest
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    pairs = [("dyn_config_t", _lib.Config), ("dyn_system_desc_t", _lib.SystemDesc),
             ("dyn_energies_t", _lib.Energies), ("dyn_frame_t", _lib.Frame)]
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "dynb200.h"', "int main(void) {"]
    for cname, py in pairs:
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        cname, field, val = line.split()
        got[(cname, field)] = int(val)
    for cname, py in pairs:
        assert got[(cname, "size")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)
