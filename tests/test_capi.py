"""C-ABI library: loads, exports every declared symbol (CPU, no compute)."""
import ctypes

from semtex_b200 import _lib


def test_library_exports_header_symbols():
    L = ctypes.CDLL(_lib.LIB_PATH)
    declared = _lib.header_symbols()
    assert "stx_field_solve" in declared and "stx_context_create" in declared
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing


def test_python_signatures_cover_header():
    assert set(_lib.header_symbols()) <= set(_lib.SIGNATURES)


def test_error_path_without_session():
    L = _lib.lib()
    h = ctypes.c_void_p()
    rc = L.stx_context_create(b"/nonexistent/session", None, 0, None, ctypes.byref(h))
    assert rc != 0
    assert b"couldn't open" in L.stx_last_error()
