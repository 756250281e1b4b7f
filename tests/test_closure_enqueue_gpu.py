"""The stream-ordered closure (se_closure_enqueue + se_closure_check) and the pipelined host
API built on it (api.ClosureStream), against the CPU oracle: several closures queued back to
back on one stream without a synchronisation between them, 16-bit lanes with and without a
value shift, 32-bit lanes, and the overflow report of a count outside the 16-bit window."""
import numpy as np
import pytest
import torch

from scalingelections_b200 import LANES_U16, LANES_U32, _lib, api

pytestmark = pytest.mark.gpu


def host_matrix(C, lo, hi, seed):
    rng = np.random.default_rng(seed)
    return rng.integers(lo, hi, size=(C, C), dtype=np.uint64).astype(np.uint32)


def enqueue(L, d, out, lanes, offset, work, stream):
    C = d.shape[0]
    return L.se_closure_enqueue(d.data_ptr(), d.stride(0), C, out.data_ptr(), out.stride(0), lanes, offset,
                                work.data_ptr(), work.numel(), stream)


def test_enqueued_closures_back_to_back(orc):
    """Six closures of different sizes and lane modes queued on one stream, then checked."""
    L = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    cases = [(300, 0, 60000, LANES_U16, 0), (129, 0, 2**32 - 1, LANES_U32, 0), (1000, 70000, 130000, LANES_U16, 69999),
             (1, 0, 5, LANES_U16, 0), (257, 0, 9, LANES_U32, 0), (640, 0, 65535, LANES_U16, 0)]
    jobs = []
    for n, (C, lo, hi, lanes, off) in enumerate(cases):
        P = host_matrix(C, lo, hi, seed=n)
        d = api._to_device_u32(P, "cuda")
        out = torch.full((C, C), -1, dtype=torch.int32, device="cuda").view(torch.uint32)
        work = torch.empty(api.closure_workspace_bytes(C, lanes), dtype=torch.uint8, device="cuda")
        _lib.check(enqueue(L, d, out, lanes, off, work, stream))
        jobs.append((P, out, work))
    for P, out, work in jobs:
        _lib.check(L.se_closure_check(work.data_ptr(), stream))
        assert np.array_equal(api._to_host_u32(out), orc.strongest_paths(P, "blocked", tile=16))


def test_enqueue_reports_overflow_at_check():
    L = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    P = host_matrix(200, 0, 200000, seed=9)  # kept counts above 65535, unshifted 16-bit lanes
    d = api._to_device_u32(P, "cuda")
    out = torch.empty_like(d)
    work = torch.empty(api.closure_workspace_bytes(200, LANES_U16), dtype=torch.uint8, device="cuda")
    _lib.check(enqueue(L, d, out, LANES_U16, 0, work, stream))  # nothing is known yet
    assert L.se_closure_check(work.data_ptr(), stream) == _lib.SE_ERR_OVERFLOW


def test_enqueue_rejects_automatic_lanes_and_offsets_on_32_bit_lanes():
    L = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    d = api._to_device_u32(host_matrix(64, 0, 9, seed=1), "cuda")
    out = torch.empty_like(d)
    work = torch.empty(api.closure_workspace_bytes(64, 0), dtype=torch.uint8, device="cuda")
    assert enqueue(L, d, out, 0, 0, work, stream) == _lib.SE_ERR_INVALID
    assert enqueue(L, d, out, LANES_U32, 5, work, stream) == _lib.SE_ERR_INVALID


@pytest.mark.parametrize("lanes,lo,hi,offset", [(LANES_U16, 0, 30000, 0), (LANES_U32, 0, 2**32 - 1, 0),
                                                 (LANES_U16, 70000, 130000, 69999)])
def test_closure_stream_matches_oracle(orc, lanes, lo, hi, offset):
    C = 385
    mats = [host_matrix(C, lo, hi, seed=s) for s in range(5)]
    pinned = torch.empty((C, C), dtype=torch.int32, pin_memory=True)
    pinned.copy_(torch.from_numpy(mats[1].view(np.int32)))
    inputs = [mats[0], pinned, mats[2], mats[3].astype(np.int64), mats[4]]  # pageable, pinned, other dtypes
    cs = api.ClosureStream(C, lanes=lanes, value_offset=offset)
    results = list(cs.map(inputs))
    assert len(results) == 5
    for P, S in zip(mats, results):
        assert np.array_equal(S, orc.strongest_paths(P, "blocked", tile=16))


def test_closure_stream_raises_on_overflow_in_order():
    C = 130
    ok = host_matrix(C, 0, 100, seed=1)
    bad = host_matrix(C, 0, 200000, seed=2)
    it = api.ClosureStream(C, lanes=LANES_U16).map([ok, bad, ok])
    first = next(it)
    assert first.shape == (C, C)
    with pytest.raises(api.SchulzeError):
        next(it)


def test_python_enqueue_and_check_equal_the_synchronous_call(orc):
    """api.strongest_paths_enqueue queues closures back to back without waiting, each with its
    own workspace; api.closure_check then reads each call's error word. The results equal
    strongest_paths_device's and the oracle's; a 16-bit overflow surfaces at the check."""
    import numpy as np
    import torch

    from scalingelections_b200 import LANES_U16, LANES_U32, api

    rng = np.random.default_rng(31)
    mats = [rng.integers(0, 3000, size=(C, C), dtype=np.uint64).astype(np.uint32) for C in (130, 700, 1000)]
    outs, works = [], []
    for P in mats:
        d = api._to_device_u32(P, "cuda")
        C = P.shape[0]
        w = torch.empty(api.closure_workspace_bytes(C, LANES_U16, dataflow=True), dtype=torch.uint8, device="cuda")
        outs.append((P, api.strongest_paths_enqueue(d, lanes=LANES_U16, workspace=w), d))
        works.append(w)
    for w in works:
        api.closure_check(w)
    for P, o, d in outs:
        assert np.array_equal(api._to_host_u32(o), orc.strongest_paths(P, "blocked", tile=16))
        assert torch.equal(o.view(torch.int32), api.strongest_paths_device(d, lanes=LANES_U32).view(torch.int32))
    big = api._to_device_u32(rng.integers(70000, 90000, size=(200, 200), dtype=np.uint64).astype(np.uint32), "cuda")
    w = torch.empty(api.closure_workspace_bytes(200, LANES_U16, dataflow=True), dtype=torch.uint8, device="cuda")
    api.strongest_paths_enqueue(big, lanes=LANES_U16, workspace=w)
    with pytest.raises(api.SchulzeError, match="16-bit"):
        api.closure_check(w)


@pytest.mark.parametrize("C", [700, 3000, 5000])
def test_enqueued_closure_captures_into_a_cuda_graph(C):
    """The stream-ordered closure captured into a CUDA graph (after a first call outside the
    capture) replays to the synchronous call's result: schedules 7, 8 and 6 at these sizes,
    with their split tiles and programmatic dependent launches."""
    rng = np.random.default_rng(C)
    P = rng.integers(0, 3000, size=(C, C), dtype=np.uint64).astype(np.uint32)
    d = api._to_device_u32(P, "cuda")
    ref = api.strongest_paths_device(d, lanes=LANES_U16)
    out = torch.empty_like(d)
    w = torch.empty(api.closure_workspace_bytes(C, LANES_U16, dataflow=True), dtype=torch.uint8, device="cuda")
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        api.strongest_paths_enqueue(d, lanes=LANES_U16, out=out, workspace=w)
        api.closure_check(w)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        api.strongest_paths_enqueue(d, lanes=LANES_U16, out=out, workspace=w)
    out.zero_()
    for _ in range(2):
        g.replay()
    torch.cuda.synchronize()
    api.closure_check(w)
    assert torch.equal(out.view(torch.int32), ref.view(torch.int32))
