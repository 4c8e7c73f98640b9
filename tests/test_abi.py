"""CPU checks of the C boundary: the library loads and exports every symbol declared in
include/*.h, and argument validation that happens before any device work."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b(?:int|const char\*|void)\s+(rr_[a-z0-9_]+)\s*\(", txt):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    from rerdmft_b200 import _lib
    lib = _lib.lib()
    missing = [n for n in sorted(_declared()) if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"
    assert len(_declared()) >= 8


def test_version_and_error_string():
    from rerdmft_b200 import _lib
    lib = _lib.lib()
    assert lib.rr_version() >= 100
    assert isinstance(lib.rr_last_error(), bytes)


def test_argument_errors_before_device_work():
    from rerdmft_b200 import _lib
    lib = _lib.lib()
    h = ctypes.c_void_p()
    assert lib.rr_ri_create(None, 4, 0, 0, ctypes.byref(h)) == _lib.RR_ERR_ARG
    assert b"n >= 1" in lib.rr_last_error()
    assert lib.rr_ri_create(None, 4, 3, 0, ctypes.byref(h)) == _lib.RR_ERR_ARG
    assert lib.rr_ri_info(None, None, None, None) == _lib.RR_ERR_ARG
    assert lib.rr_ri_destroy(None) == _lib.RR_OK
