"""The C-ABI library: builds, loads, exports every symbol include/*.h declares.
No compute calls (CPU only)."""

import ctypes
import glob
import os
import re

import pytest

from flatworld_b200 import _native, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names |= set(re.findall(r"\b(fw_\w+)\s*\(", text))
    return names


def test_library_builds_and_loads():
    path = build.build()
    assert os.path.exists(path)
    lib = ctypes.CDLL(path)
    for name in _declared():
        assert hasattr(lib, name), name


def test_binding_covers_header():
    declared = _declared()
    assert declared, "no fw_* declarations found"
    assert declared == set(_native.exported_symbols())


def test_no_device_means_loud_failure(monkeypatch):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    with pytest.raises(RuntimeError):
        _native.NativeWorld(0)


def test_build_info():
    lib = _native.lib()
    assert b"sm_100a" in lib.fw_build_info()
