"""GPU tally of streamed and packed ballots (se_tally_ex, ballot_file.tally_file) against the C
oracle's restatement of build_pairwise_preferences (scaling_elections.py:51-88)."""

import numpy as np
import pytest
import torch

from scalingelections_b200 import _lib, api
from scalingelections_b200 import ballot_file as bfm

pytestmark = pytest.mark.gpu


def ragged(V, C, seed, min_len=1):
    rng = np.random.default_rng(seed)
    return [rng.permutation(C)[:int(rng.integers(min_len, C + 1))].astype(np.int64) for _ in range(V)]


def oracle_tally(orc, B, C):
    # The oracle sizes the matrix by max id + 1; pad with a one-ballot tally when needed.
    top = max(int(b.max()) for b in B) + 1 if B else 0
    if top == C:
        return orc.tally(B)
    pad = [np.array([C - 1])]
    return orc.tally(B + pad) - orc.tally(pad)


def host_u32(t):
    return t.view(torch.int32).cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("width", [1, 2, 4])
def test_tally_ex_packed_widths_and_accumulate(orc, width):
    C = 200
    B = ragged(700, C, width)
    dtype = {1: np.uint8, 2: np.uint16, 4: np.int32}[width]
    lens = np.array([b.size for b in B])
    offs = np.zeros(len(B) + 1, dtype=np.int64)
    np.cumsum(lens, out=offs[1:])
    ids = np.concatenate(B).astype(dtype)
    tdt = {1: torch.uint8, 2: torch.int16, 4: torch.int32}[width]
    d_ids = torch.from_numpy(ids.view({1: np.uint8, 2: np.int16, 4: np.int32}[width])).cuda()
    d_offs = torch.from_numpy(offs).cuda()
    assert d_ids.dtype == tdt
    out = torch.zeros((C, C), dtype=torch.uint32, device="cuda")
    L = _lib.lib()
    need = L.se_tally_workspace_bytes(len(B), C)
    work = torch.empty(need, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    # Two calls over slices of one CSR (id_base = the slice's first offset), accumulating.
    cut = 333
    esz = d_ids.element_size()
    _lib.check(L.se_tally_ex(d_ids.data_ptr(), width, d_offs.data_ptr(), 0, cut, C, bfm.SE_TALLY_ACCUMULATE,
                             out.data_ptr(), C, work.data_ptr(), need, stream))
    _lib.check(L.se_tally_ex(d_ids.data_ptr() + int(offs[cut]) * esz, width, d_offs[cut:].data_ptr(), int(offs[cut]),
                             len(B) - cut, C, bfm.SE_TALLY_ACCUMULATE, out.data_ptr(), C, work.data_ptr(), need,
                             stream))
    assert np.array_equal(host_u32(out), oracle_tally(orc, B, C))
    # Overwrite mode equals the plain tally.
    _lib.check(L.se_tally_ex(d_ids.data_ptr(), width, d_offs.data_ptr(), 0, len(B), C, 0, out.data_ptr(), C,
                             work.data_ptr(), need, stream))
    assert np.array_equal(host_u32(out), oracle_tally(orc, B, C))


def test_tally_ex_complete_without_offsets(orc):
    rng = np.random.default_rng(9)
    C, V = 150, 900
    R = np.stack([rng.permutation(C) for _ in range(V)]).astype(np.uint8)
    d_ids = torch.from_numpy(R.reshape(-1)).cuda()
    out = torch.empty((C, C), dtype=torch.uint32, device="cuda")
    L = _lib.lib()
    need = L.se_tally_workspace_bytes(V, C)
    work = torch.empty(need, dtype=torch.uint8, device="cuda")
    _lib.check(L.se_tally_ex(d_ids.data_ptr(), 1, None, 0, V, C, 0, out.data_ptr(), C, work.data_ptr(), need,
                             torch.cuda.current_stream().cuda_stream))
    assert np.array_equal(host_u32(out), orc.tally(list(R.astype(np.int64))))


def test_tally_ex_rejects_bad_arguments():
    L = _lib.lib()
    out = torch.zeros((4, 4), dtype=torch.uint32, device="cuda")
    work = torch.empty(1 << 16, dtype=torch.uint8, device="cuda")
    ids = torch.zeros(8, dtype=torch.int16, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    assert L.se_tally_ex(ids.data_ptr(), 3, None, 0, 2, 4, 0, out.data_ptr(), 4, work.data_ptr(), 1 << 16, s) == 1
    assert L.se_tally_ex(ids.data_ptr(), 2, None, 0, 2, 4, 64, out.data_ptr(), 4, work.data_ptr(), 1 << 16, s) == 1
    assert L.se_tally_ex(ids.data_ptr() + 1, 2, None, 0, 2, 4, 0, out.data_ptr(), 4, work.data_ptr(), 1 << 16, s) == 1
    assert "aligned" in _lib.last_error()


@pytest.mark.parametrize("C,V,chunk,complete", [(40, 1000, 96, True), (300, 3001, 512, False),
                                                (129, 700, 700, False), (1000, 257, 64, False),
                                                (64, 5, 1, True)])
def test_tally_file_matches_oracle(tmp_path, orc, C, V, chunk, complete):
    if complete:
        rng = np.random.default_rng(C + V)
        B = list(np.stack([rng.permutation(C) for _ in range(V)]))
    else:
        B = ragged(V, C, C + V)
    p = tmp_path / "b.seb"
    h = bfm.write_ballots(p, B, num_candidates=C)
    assert h.complete == complete
    stats = {}
    d = bfm.tally_file(p, chunk_ballots=chunk, stats=stats)
    assert stats["chunks"] == -(-V // chunk)
    assert np.array_equal(host_u32(d), oracle_tally(orc, [np.asarray(b) for b in B], C))
    if max(int(np.max(b)) for b in B) + 1 == C:  # the in-memory GPU tally sizes C the same way
        assert np.array_equal(host_u32(d), api.build_pairwise_preferences(B))


def test_tally_file_empty(tmp_path):
    p = tmp_path / "z.seb"
    bfm.write_ballots(p, [], num_candidates=9)
    d = bfm.tally_file(p)
    assert d.shape == (9, 9) and not host_u32(d).any()


def test_tally_file_large_stream_properties(tmp_path):
    """200k incomplete ballots through many chunks: d[i][j] + d[j][i] = V off the diagonal, and
    the chunked tally equals one in-memory tally of the same ballots."""
    C, V = 96, 200_000
    rng = np.random.default_rng(77)
    lens = rng.integers(1, C + 1, size=V)
    perms = np.argsort(rng.random((V, C)), axis=1)
    B = [perms[v, :lens[v]] for v in range(V)]
    p = tmp_path / "big.seb"
    bfm.write_ballots(p, B, num_candidates=C)
    d = host_u32(bfm.tally_file(p, chunk_ballots=8192)).astype(np.int64)
    off = ~np.eye(C, dtype=bool)
    assert (d + d.T)[off].min() == V and (d + d.T)[off].max() == V and np.all(np.diag(d) == 0)
    f = bfm.BallotFile(p)
    ids, offs = f.csr()
    ref = api.tally_device(torch.from_numpy(ids).cuda(), torch.from_numpy(offs).cuda(), C)
    assert np.array_equal(d.astype(np.uint32), host_u32(ref))


@pytest.mark.parametrize("where", [5, 40 * 50 + 3])  # ballot 0 (first chunk) or ballot 40 (a later one)
def test_tally_file_reports_bad_ids(orc, tmp_path, where):
    rng = np.random.default_rng(3)
    B = [rng.permutation(50) for _ in range(100)]  # complete: ballot v's ids start at v * 50
    p = tmp_path / "bad.seb"
    h = bfm.write_ballots(p, B)
    good = p.read_bytes()
    raw = bytearray(good)
    raw[h.ids_offset + where] = 60  # an id outside [0, 50)
    p.write_bytes(bytes(raw))
    with pytest.raises(ValueError, match="outside"):
        bfm.tally_file(p, chunk_ballots=16)
    raw = bytearray(good)
    raw[h.ids_offset + where] = raw[h.ids_offset + where - 1]  # the same id twice in one ballot
    p.write_bytes(bytes(raw))
    B[where // 50][where % 50] = B[where // 50][where % 50 - 1]
    # Not an error: counted pair by pair like the reference (py:46-48), not completed (length C).
    assert np.array_equal(host_u32(bfm.tally_file(p, chunk_ballots=16)), orc.tally(B, "scatter"))


@pytest.mark.parametrize("accumulate", [False, True])
def test_tally_split_voters(orc, accumulate):
    """Few tiles, many voters: the count kernel splits the voters across CTAs and adds the
    partial counts with atomics; results stay exact, in overwrite and accumulate modes."""
    C, V = 260, 20000
    B = ragged(V, C, 123, min_len=C // 2)
    lens = np.array([b.size for b in B])
    offs = np.zeros(V + 1, dtype=np.int64)
    np.cumsum(lens, out=offs[1:])
    d_ids = torch.from_numpy(np.concatenate(B).astype(np.int16)).cuda()
    d_offs = torch.from_numpy(offs).cuda()
    L = _lib.lib()
    need = L.se_tally_workspace_bytes(V, C)
    work = torch.empty(need, dtype=torch.uint8, device="cuda")
    seed = torch.randint(0, 1000, (C, C), dtype=torch.int32, device="cuda")
    out = seed.clone().view(torch.uint32)
    flags = bfm.SE_TALLY_ACCUMULATE if accumulate else 0
    _lib.check(L.se_tally_ex(d_ids.data_ptr(), 2, d_offs.data_ptr(), 0, V, C, flags, out.data_ptr(), C,
                             work.data_ptr(), need, torch.cuda.current_stream().cuda_stream))
    expect = oracle_tally(orc, B, C).astype(np.int64)
    if accumulate:
        base = seed.cpu().numpy().astype(np.int64)
        np.fill_diagonal(expect, 0)
        expect = expect + base
    assert np.array_equal(host_u32(out).astype(np.int64), expect)


@pytest.mark.parametrize("accumulate", [False, True])
def test_tally_last_wave_split_over_voter_ranges(orc, accumulate):
    """C = 4096 and 4099 voters: 528 upper tiles, so the count's last partial wave (84 tiles) is
    split over 3 voter ranges and added with atomics, while the other tiles store whole counts.
    The ballots rotate one order (one voter per rotation: a closed-form tally), and three more
    repeat a candidate, in the first, a middle and the last voter chunk (added from the oracle's
    tally of those three alone; tallies are additive). Overwrite and accumulate modes."""
    from conftest import cyclic_ballots, cyclic_tally

    C = 4096
    ballots, perm, n = cyclic_ballots(C, seed=17, max_count=1)
    extra = [np.concatenate([perm, perm[k:k + 1]]) for k in (0, 7, 99)]  # length C + 1: one id twice
    B = list(ballots)
    B.insert(3, extra[0])
    B.insert(len(B) // 2, extra[1])
    B.append(extra[2])
    V = len(B)
    lens = np.array([b.size for b in B])
    offs = np.zeros(V + 1, dtype=np.int64)
    np.cumsum(lens, out=offs[1:])
    d_ids = torch.from_numpy(np.concatenate(B).astype(np.int16)).cuda()
    d_offs = torch.from_numpy(offs).cuda()
    L = _lib.lib()
    need = L.se_tally_workspace_bytes(V, C)
    work = torch.empty(need, dtype=torch.uint8, device="cuda")
    seed = torch.randint(0, 1000, (C, C), dtype=torch.int32, device="cuda")
    out = seed.clone().view(torch.uint32)
    flags = bfm.SE_TALLY_ACCUMULATE if accumulate else 0
    _lib.check(L.se_tally_ex(d_ids.data_ptr(), 2, d_offs.data_ptr(), 0, V, C, flags, out.data_ptr(), C,
                             work.data_ptr(), need, torch.cuda.current_stream().cuda_stream))
    expect = cyclic_tally(perm, n).astype(np.int64) + orc.tally(extra, "scatter").astype(np.int64)
    if accumulate:
        expect = expect + seed.cpu().numpy().astype(np.int64)
    assert np.array_equal(host_u32(out).astype(np.int64), expect)
