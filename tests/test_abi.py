"""The C-ABI library loads without a GPU and exports every entry point that
``include/xlbb.h`` declares (no compute calls here)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(xlbb_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from xlb_biot_b200 import build
    path = build.build()
    lib = ctypes.CDLL(path)
    names = declared("xlbb.h")
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    lib.xlbb_version.restype = ctypes.c_int
    assert lib.xlbb_version() >= 100


def test_binding_signatures_cover_the_header():
    from xlb_biot_b200 import _lib
    assert set(declared("xlbb.h")) <= set(_lib.SIGNATURES)


def test_no_cpu_fallback_without_cuda(monkeypatch):
    import torch
    from xlb_biot_b200 import _lib
    monkeypatch.setattr(torch.cuda, "is_available", lambda: False)
    with pytest.raises(_lib.XlbbError):
        _lib.require_cuda()
