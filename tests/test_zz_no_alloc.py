"""se_closure_noalloc: the closure for callers that cannot allocate device memory (plugins
whose host application owns the GPU memory budget; latency-critical code that cannot afford
cudaMalloc/cudaFree, the latter synchronising the whole device). Its scratch space is a
static device array inside libse.so, so it takes no workspace argument and allocates
nothing; it is limited to 2048 candidates.

The test calls it through the C ABI and compares its output with se_closure (which takes a
caller-provided workspace) bit for bit, on two calls in a row: the static array keeps the
previous call's contents, and the second call must not be affected by them. This file is
collected last so that a run stopping at its first failure has run every other test."""

import numpy as np
import pytest
import torch

from scalingelections_b200 import LANES_AUTO, LANES_U16, LANES_U32, _lib, api

pytestmark = pytest.mark.gpu

MAX_C = 2048


def noalloc(d: torch.Tensor, lanes: int) -> torch.Tensor:
    C = d.shape[0]
    out = torch.full((C, C), -1, dtype=torch.int32, device=d.device).view(torch.uint32)
    st = _lib.lib().se_closure_noalloc(d.data_ptr(), d.stride(0), C, out.data_ptr(), out.stride(0), lanes,
                                       torch.cuda.current_stream().cuda_stream)
    _lib.check(st)
    return out


def random_prefs(C: int, high: int, seed: int) -> torch.Tensor:
    rng = np.random.default_rng(seed)
    P = rng.integers(0, high, size=(C, C), dtype=np.uint64).astype(np.uint32)
    return api._to_device_u32(P, "cuda")


def same(a: torch.Tensor, b: torch.Tensor) -> bool:
    return torch.equal(a.view(torch.int32), b.view(torch.int32))


def test_noalloc_matches_workspace_closure_on_consecutive_calls():
    torch.cuda.set_device(0)
    # First call: the largest size, 32-bit lanes, values beyond 16 bits (fills the array).
    d1 = random_prefs(MAX_C, 2**32 - 1, seed=1)
    r1 = noalloc(d1, LANES_U32)
    assert same(r1, api.strongest_paths_device(d1, lanes=LANES_U32))
    # Second call right after: a smaller, odd size in 16-bit lanes over the stale contents.
    d2 = random_prefs(300, 4000, seed=2)
    r2 = noalloc(d2, LANES_U16)
    assert same(r2, api.strongest_paths_device(d2, lanes=LANES_U16))
    # And once more at the first input, so both lane layouts have overwritten each other.
    assert same(noalloc(d1, LANES_U32), r1)
    # Automatic lanes over the stale contents (the range probe also lives in the array): a
    # shifted 16-bit window, then plain 16-bit values, then a range only 32 bits can hold.
    d3 = api._to_device_u32(np.random.default_rng(4).integers(70000, 130000, size=(MAX_C, MAX_C))
                            .astype(np.uint32), "cuda")
    for d in (d3, d2, d1):
        want = api._to_device_u32(orc_closure(d), "cuda")
        assert same(noalloc(d, LANES_AUTO), want)
        assert same(noalloc(d, LANES_AUTO), want)


def orc_closure(d: torch.Tensor) -> np.ndarray:
    from oracle import oracle

    return oracle.strongest_paths(api._to_host_u32(d), "blocked", tile=16)


def test_noalloc_runs_round_by_round_whatever_the_closure_mode():
    """The dataflow form needs more scratch than the static array holds at C = 2048 in 32-bit
    lanes; se_closure_noalloc runs round by round whatever se_closure_set_mode chose."""
    d = random_prefs(MAX_C, 2**32 - 1, seed=5)
    want = api.strongest_paths_device(d, lanes=LANES_U32)
    api.set_closure_mode(2)
    try:
        assert same(noalloc(d, LANES_U32), want)
        assert same(noalloc(d, LANES_AUTO), want)
    finally:
        api.set_closure_mode(1)


def test_noalloc_rejects_sizes_beyond_its_static_array():
    d = random_prefs(MAX_C + 1, 10, seed=3)
    out = torch.empty_like(d)
    st = _lib.lib().se_closure_noalloc(d.data_ptr(), d.stride(0), MAX_C + 1, out.data_ptr(), out.stride(0),
                                       LANES_U16, torch.cuda.current_stream().cuda_stream)
    assert st == _lib.SE_ERR_INVALID
    assert "2048" in _lib.last_error()


def test_noalloc_on_a_long_chain():
    """Strongest paths of up to 2047 hops (a chain of strong defeats against the pivot order)
    through the static array, in every lane mode."""
    from conftest import chain_forward_ok, chain_matrix

    P, perm, w = chain_matrix(MAX_C, seed=7, order="descending")
    d = api._to_device_u32(P, "cuda")
    want = orc_closure(d)
    assert chain_forward_ok(want, perm, w)
    want_dev = api._to_device_u32(want, "cuda")
    for lanes in (LANES_U16, LANES_U32, LANES_AUTO):
        assert same(noalloc(d, lanes), want_dev), lanes
