"""The C ABI library loads and exports every entry point include/vlsg.h
declares (no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "vlsg.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:int|void|const char \*)\s*\**\s*(vlsg_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_lists_entry_points():
    names = declared_functions()
    assert "vlsg_advect" in names and "vlsg_upload_levelset" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol():
    from viennals_b200 import _lib

    L = _lib.load()
    for name in declared_functions():
        assert hasattr(L, name), name
    assert set(_lib.EXPORTED) >= set(declared_functions())


def test_errors_without_device_are_reported():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from viennals_b200 import _lib

    L = _lib.load()
    h = ctypes.c_void_p()
    rc = L.vlsg_create(ctypes.byref(h), 0, 0)
    assert rc != 0
    assert b"device" in L.vlsg_last_error(None)


def test_default_params_match_reference():
    from viennals_b200 import _lib
    from viennals_b200._abi import AdvectParams

    L = _lib.load()
    p = AdvectParams()
    L.vlsg_default_params(ctypes.byref(p))
    q = AdvectParams.defaults()
    for f, _ in AdvectParams._fields_:
        assert getattr(p, f) == getattr(q, f), f
