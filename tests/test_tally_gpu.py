"""Tally parity on the GPU against the reference's build_pairwise_preferences outputs and the
CPU oracle: complete, incomplete and repeated-id ballots, out-of-range ids, voters beyond 16
bits."""
import numpy as np
import pytest
import torch

from conftest import ballots_of, golden_names, load_golden
from scalingelections_b200 import api

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", [n for n in golden_names() if "random" not in n])
def test_golden_tally(name):
    case = load_golden(name)
    d = api.build_pairwise_preferences(ballots_of(case))
    assert np.array_equal(d, case["preferences"])


@pytest.mark.parametrize("C,V", [(1, 1), (2, 3), (127, 50), (128, 33), (129, 31), (700, 97)])
def test_random_sizes(orc, C, V):
    from scalingelections_b200.ballots import uniform_ballots

    b = uniform_ballots(V, C, seed=C * 7 + V)
    assert np.array_equal(api.build_pairwise_preferences(b), orc.tally(b, "positions"))


def test_incomplete_ballots(orc):
    rng = np.random.default_rng(3)
    ballots = []
    for _ in range(300):
        perm = rng.permutation(300)
        ballots.append(perm[: rng.integers(1, 301)])
    ballots.append(np.array([299]))
    assert np.array_equal(api.build_pairwise_preferences(ballots), orc.tally(ballots, "scatter"))


@pytest.mark.parametrize("C,complete", [(2048, True), (2500, False), (4096, False)])
def test_long_ballots_one_cta_per_ballot(orc, C, complete):
    """From 2048 candidates on, one CTA places each ballot: complete and incomplete ballots,
    and a repeated or out-of-range id in a long ballot, against the oracle."""
    rng = np.random.default_rng(C)
    V = 60
    ballots = [rng.permutation(C) if complete else rng.permutation(C)[: rng.integers(1, C + 1)] for _ in range(V)]
    ballots.append(np.array([C - 1]))
    assert np.array_equal(api.build_pairwise_preferences(ballots), orc.tally(ballots, "scatter"))
    rep = [b.copy() for b in ballots[:3]] + [np.array([C - 1])]
    rep[1][len(rep[1]) // 2] = rep[1][0]
    assert np.array_equal(api.build_pairwise_preferences(rep), orc.tally(rep, "scatter"))
    ids = torch.from_numpy(np.concatenate(ballots[:2]).astype(np.int32)).cuda()
    ids[len(ballots[0]) // 2] = C + 5
    offs = torch.tensor([0, len(ballots[0]), len(ballots[0]) + len(ballots[1])], dtype=torch.int64, device="cuda")
    with pytest.raises(api.SchulzeError, match="outside"):
        api.tally_device(ids, offs, C)


@pytest.mark.parametrize("C", [23552, 23553])
def test_place_rows_either_side_of_the_shared_memory_limit(orc, C):
    """Up to C = 23552 a ballot's place row is built in shared memory, beyond it in global
    memory: incomplete ballots on both sides, and a repeated id, against the oracle."""
    rng = np.random.default_rng(C)
    ballots = [rng.permutation(C)[: rng.integers(C // 2, C + 1)] for _ in range(5)] + [np.array([C - 1])]
    assert np.array_equal(api.build_pairwise_preferences(ballots), orc.tally(ballots, "scatter"))
    rep = [ballots[0].copy(), np.array([C - 1])]
    rep[0][-1] = rep[0][0]
    assert np.array_equal(api.build_pairwise_preferences(rep), orc.tally(rep, "scatter"))


def test_many_voters_beyond_16_bits(orc):
    """V = 70000 > 65535: counts need 32-bit lanes downstream; the tally itself is exact."""
    from scalingelections_b200.ballots import mallows_ballots

    b = mallows_ballots(70000, 24, 0.5, seed=4)
    d = api.build_pairwise_preferences(b)
    assert np.array_equal(d, orc.tally(b, "positions"))
    assert d.max() > 65535
    r = api.schulze(b, return_paths=True)
    S_ref = orc.strongest_paths(d, "serial")
    assert np.array_equal(r.strongest_paths, S_ref)


def test_repeated_ids_count_like_the_reference(orc):
    """A repeated id adds every ordered pair, diagonal included (py:46-48), and the ballot is
    completed only when its length differs from C (py:75): against the oracle's scatter form."""
    cases = [
        [np.array([0, 1, 2]), np.array([2, 2, 1])],
        [np.array([0, 0])],
        [np.array([1, 1, 1, 1, 1, 1, 1, 1]), np.array([0, 1, 2, 3, 4, 5, 6, 7])],
        [np.array([3, 2, 1, 0]), np.array([3, 3, 0, 0])],
    ]
    for ballots in cases:
        d = api.build_pairwise_preferences(ballots)
        assert np.array_equal(d, orc.tally(ballots, "scatter")), ballots
    # Eight 1s: 28 pairs on the diagonal. Its length is C = 8, so it is not completed and
    # candidate 0 gets nothing from it; the permutation adds d[0][1] = 1.
    d = api.build_pairwise_preferences(cases[2])
    assert (d[1, 1], d[1, 0], d[0, 1]) == (28, 0, 1)
    d = api.build_pairwise_preferences([np.array([1, 1, 1]), np.array([0, 1, 2, 3])])
    # Length 3 != C = 4: completed to [1, 1, 1, 0, 2, 3]: 3 diagonal pairs, 1 above 0 three times.
    assert (d[1, 1], d[1, 0], d[0, 1], d[2, 3]) == (3, 3, 1, 2)


@pytest.mark.parametrize("C,V,width", [(40, 3000, 1), (300, 777, 2), (3000, 100, 4)])
@pytest.mark.parametrize("all_length_c", [False, True])
def test_repeats_mixed_into_every_chunk(orc, tmp_path, C, V, width, all_length_c):
    """Irregular ballots spread over many 32-voter chunks beside permutations: through the
    drop-in tally, and streamed from a ballot file in chunks (accumulating, every id width,
    voter splits in the count at C = 40). With every ballot of length C the file holds no
    offsets, and no ballot is completed."""
    from scalingelections_b200 import ballot_file

    rng = np.random.default_rng(C + V + all_length_c)
    ballots = []
    for v in range(V):
        if all_length_c:
            r = rng.permutation(C)
            if v % 5 == 0:
                r[rng.integers(0, C, size=2)] = r[rng.integers(0, C)]
        elif v % 5 == 0:
            r = rng.integers(0, C, size=rng.integers(1, 2 * C))
        else:
            r = rng.permutation(C)[: rng.integers(1, C + 1)]
        ballots.append(r)
    ballots.append(np.arange(C))
    want = orc.tally(ballots, "scatter")
    assert np.array_equal(api.build_pairwise_preferences(ballots), want)
    path = tmp_path / "ballots.bin"
    h = ballot_file.write_ballots(path, ballots, C, id_bytes=width)
    assert (h.offsets_offset == 0) == all_length_c
    d = ballot_file.tally_file(path, chunk_ballots=96)
    assert np.array_equal(api._to_host_u32(d), want)


def test_out_of_range_ids_raise():
    ids = torch.tensor([0, 1, 5], dtype=torch.int32, device="cuda")
    offs = torch.tensor([0, 3], dtype=torch.int64, device="cuda")
    with pytest.raises(api.SchulzeError, match="outside"):
        api.tally_device(ids, offs, 3)


def test_zero_voters():
    ids = torch.zeros(0, dtype=torch.int32, device="cuda")
    offs = torch.zeros(1, dtype=torch.int64, device="cuda")
    d = api.tally_device(ids, offs, 5)
    assert (d.view(torch.int32) == 0).all()
