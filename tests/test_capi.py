"""The C ABI boundary without a GPU: the library loads, exports every entry
point include/ofeli_gpu.h declares, and reports failures as status codes
with a message instead of crashing."""
import ctypes
import os
import re

import pytest

from ofeli_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "ofeli_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ofg_\w+)\s*\(", src)))


def test_library_loads():
    L = capi.lib()
    assert L.ofg_version().decode().startswith("ofeli_b200")


def test_every_declared_symbol_is_exported():
    L = capi.lib()
    names = header_functions()
    assert len(names) >= 30
    for name in names:
        assert hasattr(L, name), name


def test_binding_covers_the_header():
    assert set(header_functions()) == set(capi.exported_symbols())


def test_no_fallback_when_library_missing(tmp_path, monkeypatch):
    monkeypatch.setattr(capi, "_lib", None)
    monkeypatch.setattr(capi, "LIB_PATH", str(tmp_path / "missing.so"))
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        capi.lib()


def test_null_arguments_are_rejected_with_status():
    L = capi.lib()
    assert L.ofg_matrix_create(4, 0, None, None, None) == -1
    assert b"null" in L.ofg_last_error()
    assert L.ofg_spmv(None, None, None) == -1
    assert L.ofg_prec_create(None, 1, None) == -1
    assert L.ofg_mesh_info(None, None, None, None, None) == -1


def test_profile_family_names():
    L = capi.lib()
    n = ctypes.c_int64()
    assert L.ofg_profile_read(b"no_such_family", ctypes.byref(n), None, None) == -1
    assert L.ofg_profile_read(b"spmv64", ctypes.byref(n), None, None) == 0
