"""CPU checks of the C boundary: the library loads and exports every symbol declared in
include/*.h, argument validation that happens before any device work, and the C++ drop-in
(include/rr_ri.hpp) linked into the reference's own objects exports the reference's overloads."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b(?:int|int64_t|const char\*|void)\s+(rr_[a-z0-9_]+)\s*\(", txt):
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


def test_cpp_dropin_defines_the_reference_overloads():
    so = ROOT / "oracle" / "_ref" / "librrref_dropin.so"
    if not so.exists():
        pytest.skip("oracle/_ref/librrref_dropin.so not built (make -C oracle dropin needs the reference tree)")
    syms = subprocess.run(["nm", "-DC", "--defined-only", str(so)], capture_output=True, text=True, check=True).stdout
    for sig in ("rerdmft::nonRelFockMatrix(rerdmft::Matrix<double> const&, rerdmft::RiNonRelEriSource const&",
                "rerdmft::x2cFockMatrix(rerdmft::Matrix<std::complex<double> > const&, rerdmft::RiX2cEriSource const&",
                "rerdmft::rkbFockMatrix(rerdmft::Matrix<std::complex<double> > const&, rerdmft::RiDirectEriSource const&",
                "rerdmft::riFockTwoElectronDirect(", "rerdmft::buildRiNonRelSpinMoEri(", "rerdmft::buildRiMoEri(",
                "rerdmft::RiNonRelSpinMoEri::rotated(", "rerdmft::RiMoEri::rotated(", "rerdmft::RiMoEri::positiveBlock(",
                "rerdmft::hartreeExchangeFockMatrix(", "rerdmft::jkOnlyFockMatrix("):
        assert sig in syms, sig
    needed = subprocess.run(["readelf", "-d", str(so)], capture_output=True, text=True, check=True).stdout
    assert "librr_ri.so" in needed
    ctypes.CDLL(str(so))  # loads without a GPU
