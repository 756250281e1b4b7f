"""Seeded ballot generators: shapes, determinism, and the Mallows sampler against a direct
repeated-insertion construction."""
import numpy as np

from scalingelections_b200 import ballots


def test_uniform_ballots_are_seeded_permutations():
    a = ballots.uniform_ballots(50, 17, seed=3)
    b = ballots.uniform_ballots(50, 17, seed=3)
    assert a.dtype == np.int32 and a.shape == (50, 17)
    assert np.array_equal(a, b)
    assert (np.sort(a, axis=1) == np.arange(17)).all()


def test_mallows_decode_matches_list_insertion():
    rng = np.random.default_rng(1)
    slots = ballots._insertion_positions(rng, 40, 33, 0.6)
    final = ballots._decode_insertions(slots)
    for v in range(40):
        order = []
        for i in range(33):
            order.insert(int(slots[v, i]), i)
        expect = np.empty(33, dtype=np.int64)
        expect[order] = np.arange(33)
        assert np.array_equal(final[v], expect)


def test_mallows_concentrates_near_reference():
    ref = np.arange(12)
    tight = ballots.mallows_ballots(400, 12, 0.2, seed=2, reference=ref)
    loose = ballots.mallows_ballots(400, 12, 1.0, seed=2, reference=ref)
    assert (np.sort(tight, axis=1) == np.arange(12)).all()

    def mean_displacement(b):
        pos = np.argsort(b, axis=1)
        return np.abs(pos - ref).mean()

    assert mean_displacement(tight) < 0.5 * mean_displacement(loose)


def test_random_preferences_match_reference_mode():
    P = ballots.random_preferences(9, seed=4)
    assert P.dtype == np.uint32 and P.shape == (9, 9) and P.max() < 9


def test_random_matrix_host_restatement():
    """Host restatement of the device generator: deterministic, in range, roughly uniform."""
    from scalingelections_b200.ballots import random_matrix_host

    a = random_matrix_host(200, 5)
    assert a.dtype == np.uint32 and a.shape == (200, 200)
    assert np.array_equal(a, random_matrix_host(200, 5)) and not np.array_equal(a, random_matrix_host(200, 6))
    assert a.max() == 199 and abs(a.mean() - 99.5) < 2
    assert random_matrix_host(50, 1, high=3).max() == 2
