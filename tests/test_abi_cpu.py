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
    assert lib.oracle_b200_version() == _lib.ABI_VERSION
    # argument validation happens before any CUDA call
    g = _lib.GridDesc(7, 8, 4, 1.0, 1.0, 1.0, 0)
    c = _lib.ComponentDesc()
    h = ctypes.c_void_p()
    rc = lib.oracle_b200_plan_create(ctypes.byref(g), ctypes.byref(c), ctypes.byref(h))
    assert rc == _lib.OB_ERR_ARG
    assert b"even" in lib.oracle_b200_last_error()
    rc = lib.oracle_b200_step(None, None, None, 1.0, 0, None)
    assert rc == _lib.OB_ERR_ARG


def test_new_entry_points_validate_before_cuda():
    """The intensity cap and the diagnostics workspace reject bad arguments
    with OB_ERR_ARG and a message, before any CUDA call."""
    from oraclev8_b200 import _lib
    lib = _lib.load()
    vp = ctypes.c_void_p
    one = vp(1)
    rc = lib.oracle_b200_intensity_cap(None, one, _lib.OB_PREC_F64, 10, 70.0, 300.0, 0.0, 0.0,
                                       one, one, None)
    assert rc == _lib.OB_ERR_ARG and b"NULL" in lib.oracle_b200_last_error()
    rc = lib.oracle_b200_intensity_cap(one, one, _lib.OB_PREC_F64, 10, 70.0, 0.0, 0.0, 0.0,
                                       one, one, None)
    assert rc == _lib.OB_ERR_ARG and b"tau" in lib.oracle_b200_last_error()
    rc = lib.oracle_b200_intensity_cap(one, one, 7, 10, 70.0, 300.0, 0.0, 0.0, one, one, None)
    assert rc == _lib.OB_ERR_ARG and b"precision" in lib.oracle_b200_last_error()
    assert lib.oracle_b200_intensity_cap(one, one, _lib.OB_PREC_F32, 0, 70.0, 300.0, 0.0, 0.0,
                                         one, one, None) == _lib.OB_OK  # nothing to do
    h = vp()
    assert lib.oracle_b200_vdiag_create(2, 8, 4, ctypes.byref(h)) == _lib.OB_ERR_ARG
    assert not h.value
    assert lib.oracle_b200_vdiag_create(8, 8, 4, None) == _lib.OB_ERR_ARG
    out = _lib.VdMax()
    lev = (ctypes.c_int * 1)(0)
    rc = lib.oracle_b200_vdiag_speed_max(None, one, one, _lib.OB_PREC_F64, lev, 1, 0.0, 0.0,
                                         ctypes.byref(out), None)
    assert rc == _lib.OB_ERR_ARG and b"workspace" in lib.oracle_b200_last_error()
    assert lib.oracle_b200_vdiag_centroid(None, 0, 1, 0, 1, None, None) == _lib.OB_ERR_ARG
    assert lib.oracle_b200_vdiag_destroy(None) == _lib.OB_OK


def header_defines():
    """Integer #defines of the public header, by name."""
    out = {}
    for h in (ROOT / "include").glob("*.h"):
        for name, val in re.findall(r"^#define\s+(OB_\w+)\s+(-?\d+)", h.read_text(), flags=re.M):
            out[name] = int(val)
    return out


def test_bindings_agree_with_the_header_constants():
    """The Python tables that index the library's arrays (kernel variants,
    profile classes) and the constants it passes follow the header's
    numbering, so a variant or class added on one side only fails here."""
    from oraclev8_b200 import _lib
    d = header_defines()
    var = sorted((v, k[len("OB_VAR_"):].lower()) for k, v in d.items()
                 if k.startswith("OB_VAR_") and k != "OB_VAR_COUNT")
    assert [v for v, _ in var] == list(range(d["OB_VAR_COUNT"]))
    assert tuple(n for _, n in var) == _lib.VARIANTS
    prof = sorted((v, k[len("OB_PROF_"):].lower()) for k, v in d.items()
                  if k.startswith("OB_PROF_") and k != "OB_PROF_CLASSES")
    assert [v for v, _ in prof] == list(range(d["OB_PROF_CLASSES"]))
    assert tuple(n for _, n in prof) == _lib.PROF_CLASSES
    assert d["OB_ABI_VERSION"] == _lib.ABI_VERSION
    for name in ("OB_OK", "OB_ERR_ARG", "OB_ERR_CUDA", "OB_ERR_NONFINITE", "OB_ERR_UNSUPPORTED",
                 "OB_PREC_F64", "OB_PREC_F32", "OB_ADV_CENTERED2", "OB_ADV_UPWIND5H",
                 "OB_TEND_ADVECTION", "OB_TEND_CORIOLIS", "OB_TEND_DAMPING", "OB_TEND_HEATING",
                 "OB_TEND_DRAG", "OB_TEND_SPONGE", "OB_TEND_DIFFUSION", "OB_TEND_COOLING"):
        assert getattr(_lib, name) == d[name], name
