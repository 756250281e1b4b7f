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


def test_closure_schedule_settings_need_no_gpu():
    from scalingelections_b200 import _lib

    L = _lib.lib()
    n = 2
    max_c = (ctypes.c_int * n)(2048, 4096)
    ok = (ctypes.c_int * n)(4, 3)
    bad = (ctypes.c_int * n)(4, 2)  # the dataflow form is not a table variant
    assert L.se_closure_set_variant_table(max_c, bad, n) == _lib.SE_ERR_INVALID
    assert L.se_closure_set_variant_table(max_c, ok, 9) == _lib.SE_ERR_INVALID
    assert L.se_closure_set_variant_table(max_c, ok, n) == _lib.SE_OK
    assert L.se_closure_set_variant_table(None, None, 0) == _lib.SE_OK
    assert L.se_closure_set_mode(9) == _lib.SE_ERR_INVALID
    for mode in (4, 0):
        assert L.se_closure_set_mode(mode) == _lib.SE_OK
    from scalingelections_b200 import api

    table = api.BUILTIN_CLOSURE_VARIANTS  # put the built-in table back
    max_c = (ctypes.c_int * len(table))(*[c for c, _ in table])
    modes = (ctypes.c_int * len(table))(*[m for _, m in table])
    assert L.se_closure_set_variant_table(max_c, modes, len(table)) == _lib.SE_OK


def test_closure_schedule_query_needs_no_gpu():
    """Which schedule the automatic choice gives each size, with and without the workspace the
    one-launch-per-round schedule needs, and in 32-bit lanes (no wide micro-tile there)."""
    from scalingelections_b200 import LANES_U16, LANES_U32, api

    api.set_closure_mode(0)
    flow = lambda C: api.closure_workspace_bytes(C, LANES_U16, dataflow=True)  # noqa: E731
    plain = lambda C: api.closure_workspace_bytes(C, LANES_U16)  # noqa: E731
    assert api.closure_schedule(1000, LANES_U16, flow(1000)) == 7
    flow32 = lambda C: api.closure_workspace_bytes(C, LANES_U32, dataflow=True)  # noqa: E731
    assert api.closure_schedule(1000, LANES_U32, flow32(1000)) == 1  # no wide micro-tile in 32-bit lanes
    assert api.closure_schedule(2048, LANES_U32, flow32(2048)) == 6  # mode 8 on the default micro-tile
    assert api.closure_schedule(3000, LANES_U16, flow(3000)) == 8
    assert api.closure_schedule(4096, LANES_U16, flow(4096)) == 8
    assert api.closure_schedule(4096, LANES_U32, flow32(4096)) == 6
    assert api.closure_schedule(4096, LANES_U16, plain(4096)) == 1  # too little workspace for 8
    assert api.closure_schedule(16384, LANES_U16, flow(16384)) == 6
    assert api.closure_schedule(16384, LANES_U16, plain(16384)) == 1  # too little workspace for 6
    assert api.closure_schedule(0) == -1


HOST_ALLOC_FAILURE = r"""
import ctypes, resource, sys

L = ctypes.CDLL(sys.argv[1])
L.se_batch_workspace_bytes.restype = ctypes.c_int64
L.se_last_error.restype = ctypes.c_char_p
el = ctypes.create_string_buffer(64)  # one se_election_t, C = 0
vm = next(int(l.split()[1]) for l in open("/proc/self/status") if l.startswith("VmSize:")) * 1024
resource.setrlimit(resource.RLIMIT_AS, (vm + (32 << 20), resource.getrlimit(resource.RLIMIT_AS)[1]))
n = (1 << 24) - 1  # size_batch's first host vector alone takes 134 MB
print(L.se_batch_workspace_bytes(n, el), L.se_last_error().decode())
"""


def test_a_host_allocation_failure_is_a_status_not_an_abort():
    """A std::bad_alloc inside an entry point comes back through the C ABI as an error (here
    se_batch_workspace_bytes's -1 with its message), not as std::terminate. The process caps
    its own address space so that the batch sizer's host vectors cannot be allocated; the
    sizer throws before it reads an election, and the one election it is given would fail its
    candidate-count check if the cap did not take effect."""
    import subprocess
    import sys

    from scalingelections_b200 import _lib

    r = subprocess.run([sys.executable, "-c", HOST_ALLOC_FAILURE, str(_lib.LIB_PATH)], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    total, _, message = r.stdout.strip().partition(" ")
    assert total == "-1"
    assert message.startswith("host-side failure"), message
