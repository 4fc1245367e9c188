"""The C-ABI library builds for sm_100a, loads, and exports every entry point
the public header declares (no compute calls: this runs without a GPU)."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def header_symbols():
    syms = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = h.read_text()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        syms |= set(re.findall(r"\b(oracle_b200_\w+)\s*\(", txt))
    return syms


def test_library_exports_header_symbols():
    from oraclev8_b200 import build
    lib_path = build.build()
    lib = ctypes.CDLL(str(lib_path))
    syms = header_symbols()
    assert len(syms) >= 14
    missing = [s for s in sorted(syms) if not hasattr(lib, s)]
    assert not missing, missing
    from oraclev8_b200 import _lib
    assert set(_lib.EXPORTS) <= syms


def test_version_and_error_string_without_gpu():
    from oraclev8_b200 import _lib
    lib = _lib.load()
    assert lib.oracle_b200_version() >= 1
    # argument validation happens before any CUDA call
    g = _lib.GridDesc(7, 8, 4, 1.0, 1.0, 1.0, 0)
    c = _lib.ComponentDesc()
    h = ctypes.c_void_p()
    rc = lib.oracle_b200_plan_create(ctypes.byref(g), ctypes.byref(c), ctypes.byref(h))
    assert rc == _lib.OB_ERR_ARG
    assert b"even" in lib.oracle_b200_last_error()
    rc = lib.oracle_b200_step(None, None, None, 1.0, 0, None)
    assert rc == _lib.OB_ERR_ARG
