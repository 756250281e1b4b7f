"""The CPU oracle pinned against the reference's own outputs (golden fixtures generated by
tests/golden/make_golden.py from the reference's Numba code) and against the reference's
compiled OpenMP closure where it was built."""
import numpy as np
import pytest

from conftest import ballots_of, golden_names, has_repeats, load_golden

NAMES = golden_names()


@pytest.mark.parametrize("name", NAMES)
def test_oracle_closure_matches_reference(orc, name):
    import hashlib

    case = load_golden(name)
    P = case["preferences"]
    if P.shape[0] > 1024:  # the serial C^3 loop would take minutes on one core
        S = orc.strongest_paths(P, "blocked", tile=16)
        assert hashlib.sha256(S.tobytes()).hexdigest() == str(case["strongest_sha256"])
        return
    S = orc.strongest_paths(P, "serial")
    if "strongest" in case:
        assert np.array_equal(S, case["strongest"])
    assert hashlib.sha256(S.tobytes()).hexdigest() == str(case["strongest_sha256"])
    Sb = orc.strongest_paths(P, "blocked", tile=16)
    assert np.array_equal(S, Sb)
    Sb7 = orc.strongest_paths(P, "blocked", tile=7)  # tail tiles
    assert np.array_equal(S, Sb7)


@pytest.mark.parametrize("name", NAMES)
def test_oracle_ranking_matches_reference(orc, name):
    case = load_golden(name)
    P = case["preferences"]
    S = orc.strongest_paths(P, "serial" if P.shape[0] <= 1024 else "blocked")
    winner, ranking = orc.winner_and_ranking(S)
    assert winner == int(case["winner"])
    assert ranking == list(case["ranking"])


@pytest.mark.parametrize("name", [n for n in NAMES if "random" not in n])
def test_oracle_tally_matches_reference(orc, name):
    case = load_golden(name)
    ballots = ballots_of(case)
    d = orc.tally(ballots, "scatter")
    assert np.array_equal(d, case["preferences"])
    if has_repeats(case):  # the positions form holds for permutations only, and says so
        with pytest.raises(ValueError):
            orc.tally(ballots, "positions")
        return
    d2 = orc.tally(ballots, "positions")
    assert np.array_equal(d2, case["preferences"])


def test_paradox_known_answer(orc):
    """validate_paradox.py:26-28: Java wins, then one more Java-first ballot makes Python win."""
    names = ["Python", "Rust", "Go", "Java"]
    before, after = load_golden("paradox_before"), load_golden("paradox_after")
    w0, _ = orc.winner_and_ranking(orc.strongest_paths(orc.tally(ballots_of(before)), "serial"))
    w1, _ = orc.winner_and_ranking(orc.strongest_paths(orc.tally(ballots_of(after)), "serial"))
    assert (names[w0], names[w1]) == ("Java", "Python")


def test_widest_rows_match_closure(orc):
    rng = np.random.default_rng(0)
    for C in (1, 2, 9, 64, 150):
        P = rng.integers(0, 6, size=(C, C)).astype(np.uint32)
        S = orc.strongest_paths(P, "serial")
        rows = orc.widest_rows(P, range(C))
        assert np.array_equal(rows, S)


def test_oracle_rejects_bad_ballots(orc):
    with pytest.raises(ValueError):
        orc.tally([np.array([0, 1, 1])], "positions")


def test_reference_openmp_agrees_at_aligned_sizes(orc):
    ref = orc.reference_cpu()
    if ref is None:
        pytest.skip("reference CPU module not built here")
    for name in ("uniform_c128_v2000", "random_c256_hi256", "random_c64_hi4"):
        case = load_golden(name)
        out = ref.compute_strongest_paths(case["preferences"], allow_gpu=False, allow_tma=False, tile_size=16)
        assert np.array_equal(out, case["strongest"])
