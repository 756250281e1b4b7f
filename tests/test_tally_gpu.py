"""Tally parity on the GPU against the reference's build_pairwise_preferences outputs and the
CPU oracle: complete, incomplete and malformed ballots, voters beyond 16 bits."""
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
    bad = [b.copy() for b in ballots[:3]]
    bad[1][len(bad[1]) // 2] = bad[1][0] if len(bad[1]) > 1 else C + 5
    with pytest.raises(ValueError):
        api.build_pairwise_preferences(bad + [np.array([C - 1])])


@pytest.mark.parametrize("C", [23552, 23553])
def test_place_rows_either_side_of_the_shared_memory_limit(orc, C):
    """Up to C = 23552 a ballot's place row is built in shared memory, beyond it in global
    memory: incomplete ballots on both sides, and a repeated id, against the oracle."""
    rng = np.random.default_rng(C)
    ballots = [rng.permutation(C)[: rng.integers(C // 2, C + 1)] for _ in range(5)] + [np.array([C - 1])]
    assert np.array_equal(api.build_pairwise_preferences(ballots), orc.tally(ballots, "scatter"))
    bad = [ballots[0].copy(), np.array([C - 1])]
    bad[0][-1] = bad[0][0]
    with pytest.raises(ValueError, match="twice"):
        api.build_pairwise_preferences(bad)


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


def test_repeated_or_out_of_range_ids_raise():
    with pytest.raises(ValueError, match="twice"):
        api.build_pairwise_preferences([np.array([0, 1, 2]), np.array([2, 2, 1])])
    ids = torch.tensor([0, 1, 5], dtype=torch.int32, device="cuda")
    offs = torch.tensor([0, 3], dtype=torch.int64, device="cuda")
    with pytest.raises(api.SchulzeError, match="outside"):
        api.tally_device(ids, offs, 3)


def test_zero_voters():
    ids = torch.zeros(0, dtype=torch.int32, device="cuda")
    offs = torch.zeros(1, dtype=torch.int64, device="cuda")
    d = api.tally_device(ids, offs, 5)
    assert (d.view(torch.int32) == 0).all()
