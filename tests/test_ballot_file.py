"""Ballot files on the host: format round trips, header checks and chunking. The tallies are
checked with the C oracle (the GPU tally of the same files is in test_ballot_file_gpu.py)."""
import numpy as np
import pytest

from scalingelections_b200 import ballot_file as bfm
from scalingelections_b200.api import Ballots


def ragged(V, C, seed, min_len=1):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(V):
        n = int(rng.integers(min_len, C + 1))
        out.append(rng.permutation(C)[:n].astype(np.int64))
    return out


@pytest.mark.parametrize("C,width", [(1, 1), (256, 1), (257, 2), (65536, 2), (65537, 4)])
def test_id_width(C, width):
    assert bfm.id_width(C) == width


def test_round_trip_complete(tmp_path):
    rng = np.random.default_rng(1)
    R = np.stack([rng.permutation(40) for _ in range(300)])
    h = bfm.write_ballots(tmp_path / "a.seb", R)
    assert h.complete and h.id_bytes == 1 and h.num_voters == 300 and h.num_candidates == 40
    f = bfm.BallotFile(tmp_path / "a.seb")
    assert f.offsets is None and len(f) == 300
    ids, offs = f.csr()
    assert np.array_equal(ids.reshape(300, 40), R)
    assert np.array_equal(offs, np.arange(301) * 40)
    assert np.array_equal(f.ballot(17), R[17])


def test_round_trip_ragged_and_widths(tmp_path):
    B = ragged(500, 300, 2)
    for width in (2, 4):
        h = bfm.write_ballots(tmp_path / f"r{width}.seb", B, id_bytes=width)
        assert not h.complete and h.id_bytes == width and h.num_candidates == 300
        f = bfm.BallotFile(tmp_path / f"r{width}.seb")
        for v in (0, 1, 250, 499):
            assert np.array_equal(f.ballot(v), B[v])
        ids, offs = f.csr(100, 230)
        assert offs[0] == 0 and np.array_equal(ids[offs[3]:offs[4]], B[103])
    with pytest.raises(ValueError, match="cannot hold"):
        bfm.write_ballots(tmp_path / "x.seb", B, id_bytes=1)


def test_ballots_object_and_explicit_candidates(tmp_path):
    B = ragged(50, 20, 3)
    b = Ballots.from_rankings(B)
    h = bfm.write_ballots(tmp_path / "b.seb", b, num_candidates=64)
    assert h.num_candidates == 64 and not h.complete
    with pytest.raises(ValueError, match="outside"):
        bfm.write_ballots(tmp_path / "c.seb", B, num_candidates=5)


def test_rejects_empty_ballot_and_negative_ids(tmp_path):
    with pytest.raises(ValueError, match="zero-size"):
        bfm.write_ballots(tmp_path / "e.seb", [np.array([0, 1]), np.array([], dtype=np.int64)])
    with pytest.raises(ValueError, match="non-negative"):
        bfm.write_ballots(tmp_path / "n.seb", [np.array([0, -1])])


def test_empty_file(tmp_path):
    h = bfm.write_ballots(tmp_path / "z.seb", [], num_candidates=7)
    assert h.num_voters == 0 and h.num_ids == 0
    f = bfm.BallotFile(tmp_path / "z.seb")
    assert len(f) == 0 and list(f.chunks(10)) == []


def test_corrupt_headers(tmp_path):
    B = ragged(30, 12, 4)
    p = tmp_path / "ok.seb"
    bfm.write_ballots(p, B)
    raw = bytearray(p.read_bytes())
    bad = tmp_path / "bad.seb"
    bad.write_bytes(b"NOTBALLOT" + bytes(raw[9:]))
    with pytest.raises(ValueError, match="magic"):
        bfm.BallotFile(bad)
    v = bytearray(raw)
    v[8] = 9
    bad.write_bytes(bytes(v))
    with pytest.raises(ValueError, match="version"):
        bfm.BallotFile(bad)
    bad.write_bytes(bytes(raw[:len(raw) - 16]))
    with pytest.raises(ValueError, match="truncated"):
        bfm.BallotFile(bad)
    bad.write_bytes(bytes(raw[:20]))
    with pytest.raises(ValueError, match="too short"):
        bfm.BallotFile(bad)


def test_chunks_cover_every_ballot_once(tmp_path):
    B = ragged(1001, 33, 5)
    bfm.write_ballots(tmp_path / "c.seb", B)
    f = bfm.BallotFile(tmp_path / "c.seb")
    for step in (1, 7, 128, 1000, 1001, 5000):
        spans = list(f.chunks(step))
        assert spans[0][0] == 0 and spans[-1][1] == 1001
        assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
        assert all(0 < v1 - v0 <= step for v0, v1 in spans)


def test_chunked_tally_is_additive(tmp_path, orc):
    """The property tally_file relies on: the tally of all ballots is the sum of the tallies of
    consecutive chunks (every completed ballot is a permutation), checked with the oracle."""
    B = ragged(600, 45, 6)
    bfm.write_ballots(tmp_path / "t.seb", B, num_candidates=45)
    f = bfm.BallotFile(tmp_path / "t.seb")
    whole = orc.tally(B)
    total = np.zeros_like(whole)
    for v0, v1 in f.chunks(97):
        total += orc.tally([f.ballot(v) for v in range(v0, v1)] + [np.array([44])])
        total -= orc.tally([np.array([44])])
    assert np.array_equal(total, whole)


def test_default_chunk_ballots_bounds():
    assert bfm.default_chunk_ballots(16384) * 16384 * 4 <= 1 << 30
    assert bfm.default_chunk_ballots(8) >= 32
