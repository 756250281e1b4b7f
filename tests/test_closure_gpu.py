"""Closure parity on the GPU, through the C ABI: bit-exact against the reference's outputs
(golden fixtures) and against the CPU oracle on seeded inputs, in both lane modes."""
import numpy as np
import pytest
import torch

from conftest import golden_names, load_golden
from scalingelections_b200 import LANES_AUTO, LANES_U16, LANES_U32, _lib, api

pytestmark = pytest.mark.gpu


def gpu_closure(P, lanes):
    d = api._to_device_u32(np.ascontiguousarray(P, dtype=np.uint32), "cuda")
    out = api.strongest_paths_device(d, lanes=lanes)
    return api._to_host_u32(out)


def lane_modes(P):
    return [LANES_AUTO, LANES_U32] + ([LANES_U16] if P.max(initial=0) <= 0xFFFF else [])


@pytest.mark.parametrize("name", golden_names())
def test_golden_closure(name):
    case = load_golden(name)
    P = case["preferences"]
    for lanes in lane_modes(P):
        S = gpu_closure(P, lanes)
        import hashlib
        assert hashlib.sha256(S.tobytes()).hexdigest() == str(case["strongest_sha256"]), (name, lanes)


@pytest.mark.parametrize("C", [1, 2, 3, 5, 37, 127, 128, 129, 255, 256, 257, 300, 383, 1000])
def test_odd_sizes_against_oracle(orc, C):
    rng = np.random.default_rng(C)
    for hi in (2, 7, C + 1, 60000):
        P = rng.integers(0, hi, size=(C, C), dtype=np.uint64).astype(np.uint32)
        S_ref = orc.strongest_paths(P, "blocked", tile=16)
        for lanes in lane_modes(P):
            assert np.array_equal(gpu_closure(P, lanes), S_ref), (C, hi, lanes)


@pytest.mark.parametrize("C", [160, 161, 192, 193, 224, 225, 288, 353, 415])
def test_padding_skip_boundaries(orc, C):
    """The last row block holds C mod 128 real pivots and rows; tiles skip the 32-pivot chunks
    and 32-row warps wholly past C. Sizes on each side of the 32-cell steps."""
    rng = np.random.default_rng(C + 17)
    P = rng.integers(0, 3000, size=(C, C), dtype=np.uint64).astype(np.uint32)
    S_ref = orc.strongest_paths(P, "blocked", tile=16)
    for lanes in (LANES_U16, LANES_U32):
        assert np.array_equal(gpu_closure(P, lanes), S_ref), (C, lanes)


def test_u32_values_beyond_16_bits(orc):
    rng = np.random.default_rng(5)
    P = rng.integers(0, 2**32 - 1, size=(300, 300), dtype=np.uint64).astype(np.uint32)
    S_ref = orc.strongest_paths(P, "blocked", tile=16)
    assert np.array_equal(gpu_closure(P, LANES_U32), S_ref)
    assert np.array_equal(gpu_closure(P, LANES_AUTO), S_ref)
    with pytest.raises(api.SchulzeError, match="65535"):
        gpu_closure(P, LANES_U16)


def test_strided_input_and_output(orc):
    rng = np.random.default_rng(6)
    C = 200
    P = rng.integers(0, 500, size=(C, C)).astype(np.uint32)
    big = torch.zeros((C, C + 13), dtype=torch.int32, device="cuda")
    big[:, :C] = torch.from_numpy(P.view(np.int32)).cuda()
    d = big.view(torch.uint32)[:, :C]
    out_big = torch.full((C, C + 7), -1, dtype=torch.int32, device="cuda")
    out = out_big.view(torch.uint32)[:, :C]
    api.strongest_paths_device(d, lanes=LANES_U16, out=out)
    got = out_big[:, :C].cpu().numpy().view(np.uint32)
    assert np.array_equal(got, orc.strongest_paths(P, "blocked", tile=16))
    assert (out_big[:, C:] == -1).all()  # padding columns of the output untouched


def test_mallows_c2048_against_oracle(orc):
    b = orc.mallows_ballots(400, 2048, 0.8, seed=21)
    d = orc.tally(b, "positions")
    S_ref = orc.strongest_paths(d, "blocked", tile=32)
    assert np.array_equal(gpu_closure(d, LANES_U16), S_ref)


def test_uniform_c4096_against_oracle(orc):
    """Single election at C=4096, V=4096, uniform ballots: full matrix equality."""
    from scalingelections_b200.ballots import uniform_ballots

    b = uniform_ballots(4096, 4096, seed=42)
    ids = torch.from_numpy(b.reshape(-1)).cuda()
    offs = torch.arange(4097, dtype=torch.int64, device="cuda") * 4096
    d = api.tally_device(ids, offs, 4096)
    d_h = api._to_host_u32(d)
    S = api._to_host_u32(api.strongest_paths_device(d, lanes=LANES_U16))
    S_ref = orc.strongest_paths(d_h, "blocked", tile=64)
    assert np.array_equal(S, S_ref)


def test_closure_c16384_rows_by_dijkstra(orc):
    """Headline size C=16384 (Mallows phi=0.8, V=4096): whole-matrix properties on the GPU
    plus exact rows from an independent bottleneck Dijkstra on the CPU."""
    from scalingelections_b200.ballots import mallows_ballots_device

    C, V = 16384, 4096
    ids = mallows_ballots_device(V, C, 0.8, seed=7).view(-1)
    offs = torch.arange(V + 1, dtype=torch.int64, device="cuda") * C
    d = api.tally_device(ids, offs, C)
    S = api.strongest_paths_device(d, lanes=LANES_U16)
    S32 = api.strongest_paths_device(d, lanes=LANES_U32)
    assert torch.equal(S.view(torch.int32), S32.view(torch.int32))
    d_h = api._to_host_u32(d)
    S_h = api._to_host_u32(S)
    rows = [0, 1, 4095, 8191, C - 1]
    exp = orc.widest_rows(d_h, rows)
    assert np.array_equal(S_h[rows], exp)
    # Dominance: S >= the defeat matrix it started from; the diagonal is 0.
    S0 = orc.defeats(d_h)
    assert (S_h >= S0).all()
    assert not np.diagonal(S_h).any()


def test_closure_c32768_properties(orc):
    """The largest headline size, C=32768 (Mallows phi=0.8, V=4096; a 4 GiB preference
    matrix): 16-bit and 32-bit lanes agree bit for bit, two rows match the independent
    bottleneck Dijkstra exactly, S dominates its defeat matrix, the diagonal is 0, and the
    ranking from S equals the oracle's ranking rule applied to the same S."""
    from scalingelections_b200.ballots import mallows_ballots_device

    C, V = 32768, 4096
    ids = mallows_ballots_device(V, C, 0.8, seed=3).view(-1)
    offs = torch.arange(V + 1, dtype=torch.int64, device="cuda") * C
    d = api.tally_device(ids, offs, C)
    del ids
    S = api.strongest_paths_device(d, lanes=LANES_U16)
    S32 = api.strongest_paths_device(d, lanes=LANES_U32)
    assert torch.equal(S.view(torch.int32), S32.view(torch.int32))
    del S32
    wins, ranking = api.rank_device(S)
    d_h = api._to_host_u32(d)
    del d
    S_h = api._to_host_u32(S)
    rows = [5, C - 2]
    assert np.array_equal(S_h[rows], orc.widest_rows(d_h, rows))
    assert (S_h >= orc.defeats(d_h)).all()
    assert not np.diagonal(S_h).any()
    w_ref, r_ref = orc.wins_and_ranking(S_h)
    assert np.array_equal(wins.cpu().numpy(), w_ref)
    assert np.array_equal(ranking.cpu().numpy(), r_ref)


def test_shifted_16_bit_lanes_for_large_counts(orc):
    """Kept values in a window [70001, 130000] exceed 16 bits but span less than 65535: the
    automatic mode closes them in shifted 16-bit lanes, bit-identical to 32-bit lanes."""
    rng = np.random.default_rng(11)
    C = 333
    base = rng.integers(70001, 130000, size=(C, C), dtype=np.uint64).astype(np.uint32)
    P = base.copy()
    S_ref = orc.strongest_paths(P, "blocked", tile=16)
    assert orc.defeats(P).max() > 65535
    assert np.array_equal(gpu_closure(P, LANES_AUTO), S_ref)
    assert np.array_equal(gpu_closure(P, LANES_U32), S_ref)


@pytest.mark.parametrize("C", [129, 300, 640, 1000, 1700])
def test_dataflow_equals_round_by_round(orc, C):
    """The barrier-free dataflow closure and the round-by-round launches give the same
    matrix (and the oracle's), in both lane modes."""
    rng = np.random.default_rng(C + 1)
    P = rng.integers(0, 5000, size=(C, C), dtype=np.uint64).astype(np.uint32)
    S_ref = orc.strongest_paths(P, "blocked", tile=32)
    try:
        for mode in (1, 2):
            api.set_closure_mode(mode)
            for lanes in (LANES_U16, LANES_U32):
                assert np.array_equal(gpu_closure(P, lanes), S_ref), (mode, lanes)
    finally:
        api.set_closure_mode(0)


@pytest.mark.parametrize("C", [1, 127, 129, 300, 385, 512, 640, 1000, 1700, 2305, 4100])
def test_wide_micro_tile_schedules(orc, C):
    """Schedules 3 (panels on the wide micro-tile) and 4 (also a wide pivot launch per round)
    against the oracle in 16-bit lanes (shifted and not) and, where they fall back to
    schedule 1, 32-bit lanes; and the automatic schedule through an installed variant table."""
    rng = np.random.default_rng(C + 7)
    P = rng.integers(0, 9000, size=(C, C), dtype=np.uint64).astype(np.uint32)
    S_ref = orc.strongest_paths(P, "blocked", tile=16)
    Q = P + np.uint32(70000)
    Q_ref = orc.strongest_paths(Q, "blocked", tile=16)
    try:
        for mode in (3, 4, 5, 6, 7, 8):
            api.set_closure_mode(mode)
            for lanes in (LANES_U16, LANES_U32, LANES_AUTO):
                assert np.array_equal(gpu_closure(P, lanes), S_ref), (mode, lanes)
            assert np.array_equal(gpu_closure(Q, LANES_AUTO), Q_ref), mode  # shifted 16-bit lanes
        api.set_closure_mode(0)
        for table in ([(C, 3)], [(max(C - 1, 0), 1), (C, 4)], [(C, 5)], [(C, 6)], []):
            api.set_closure_variants(table)
            assert np.array_equal(gpu_closure(P, LANES_U16), S_ref), table
    finally:
        api.set_closure_variants(api.BUILTIN_CLOSURE_VARIANTS)  # the library's built-in table
        api.set_closure_mode(0)


def closure_with_workspace(P, lanes, work_bytes):
    """se_closure through the C ABI with exactly work_bytes of workspace."""
    C = P.shape[0]
    d = api._to_device_u32(np.ascontiguousarray(P, dtype=np.uint32), "cuda")
    out = torch.empty((C, C), dtype=torch.uint32, device="cuda")
    work = torch.empty(work_bytes, dtype=torch.uint8, device="cuda")
    _lib.check(_lib.lib().se_closure(d.data_ptr(), C, C, out.data_ptr(), C, int(lanes), 0, work.data_ptr(),
                                     work_bytes, torch.cuda.current_stream().cuda_stream))
    return api._to_host_u32(out)


@pytest.mark.parametrize("C", [129, 257, 700, 2305, 3584, 3585])
def test_split_panels_match_unsplit(orc, C):
    """The round-by-round schedules split each panel tile and the next pivot tile over 4 pivot
    chunks when the workspace has the split area (up to 28 row blocks, C = 3584): the same
    matrix with the full and the plain workspace (which runs the tiles whole) gives identical
    results in schedules 1, 3, 4 and 7 and both lane widths, and equals the oracle where the
    oracle is quick."""
    rng = np.random.default_rng(C + 11)
    P = rng.integers(0, 9000, size=(C, C), dtype=np.uint64).astype(np.uint32)
    S_ref = orc.strongest_paths(P, "blocked", tile=16) if C <= 2400 else None
    try:
        for mode in (1, 3, 4, 7):
            api.set_closure_mode(mode)
            for lanes in (LANES_U16, LANES_U32):
                full = api.closure_workspace_bytes(C, lanes, dataflow=True)
                plain = api.closure_workspace_bytes(C, lanes, dataflow=False)
                split = closure_with_workspace(P, lanes, full)
                whole = closure_with_workspace(P, lanes, plain)
                assert np.array_equal(split, whole), (mode, lanes)
                if S_ref is not None:
                    assert np.array_equal(split, S_ref), (mode, lanes)
    finally:
        api.set_closure_mode(0)


def test_dropin_stages_large_numpy_inputs_through_pinned_memory():
    """compute_strongest_paths with a pageable NumPy matrix of 144 MB (past the two 64 MiB
    staging chunks, with a ragged last chunk): the same result as the device-resident path,
    twice in a row (the staging buffers are reused)."""
    C = 6001
    rng = np.random.default_rng(6001)
    P = rng.integers(0, 50000, size=(C, C), dtype=np.uint64).astype(np.uint32)
    want = api._to_host_u32(api.strongest_paths_device(torch.from_numpy(P.view(np.int32)).cuda().view(torch.uint32),
                                                       lanes=LANES_AUTO))
    for _ in range(2):
        got = api.compute_strongest_paths(P, allow_gpu=True, tile_size=32)
        assert np.array_equal(got, want)
    d = api._to_device_u32(P, torch.cuda.current_device())
    assert torch.equal(d.view(torch.int32).cpu(), torch.from_numpy(P.view(np.int32)))
