"""The C ABI library loads and exports every symbol include/se.h declares; host-side argument
checks answer without touching a GPU."""
import ctypes
import re

from conftest import ROOT


def declared_symbols():
    text = (ROOT / "include" / "se.h").read_text()
    return sorted(set(re.findall(r"SE_API\s+[\w\s\*]*?\b(se_\w+)\s*\(", text)))


def test_header_declares_the_entry_points():
    names = declared_symbols()
    for must in ("se_closure", "se_tally", "se_rank", "se_last_error", "se_device_info"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from scalingelections_b200 import _lib

    L = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, missing
    assert set(declared_symbols()) <= set(_lib.SIGNATURES), "ctypes signature table is incomplete"


def test_workspace_queries():
    from scalingelections_b200 import api

    assert api.closure_workspace_bytes(1, 16) > 0
    w16 = api.closure_workspace_bytes(16384, 16)
    w32 = api.closure_workspace_bytes(16384, 32)
    assert w16 >= 16384 * 16384 * 2 and w32 >= 16384 * 16384 * 4
    assert api.closure_workspace_bytes(16384, 0) == w32  # auto may fall back to 32-bit lanes
    assert api.tally_workspace_bytes(4096, 16384) >= 4096 * 16384 * 4


def test_closure_argument_errors_need_no_gpu():
    from scalingelections_b200 import _lib

    L = _lib.lib()
    buf = ctypes.create_string_buffer(1024)
    p = ctypes.cast(buf, ctypes.c_void_p)
    assert L.se_closure(p, 4, 0, p, 4, 16, 0, p, 1024, None) == _lib.SE_ERR_INVALID
    assert L.se_closure(p, 4, 4, p, 4, 16, 64, p, 1024, None) == _lib.SE_ERR_UNSUPPORTED
    assert _lib.last_error() == "Unsupported tile size"
    assert L.se_closure(p, 4, 4, p, 4, 7, 0, p, 1024, None) == _lib.SE_ERR_INVALID
    assert L.se_closure(p, 4, 4, p, 4, 16, 0, p, 16, None) == _lib.SE_ERR_WORKSPACE
    assert L.se_tally(None, None, 5, 4, p, 4, p, 1 << 20, None) == _lib.SE_ERR_INVALID
    assert L.se_rank(p, 2, 4, p, p, None) == _lib.SE_ERR_INVALID
