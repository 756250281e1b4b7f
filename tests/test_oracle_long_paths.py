"""The oracle on inputs whose strongest paths run the length of the matrix, each with a
closed-form answer:
  * a chain of strong defeats over weak noise: the serial and blocked closures agree, and every
    forward pair along the chain has the smallest chain weight on the segment;
  * ballots that rotate one order (tallied by the oracle): every strongest path runs the cycle
    in single steps.
This pins the oracle on the inputs the GPU long-path tests compare against."""
import numpy as np
import pytest

from conftest import chain_forward_ok, chain_matrix, cyclic_ballots, cyclic_strongest_paths, cyclic_tally


@pytest.mark.parametrize("C", [1, 2, 3, 17, 130, 300])
@pytest.mark.parametrize("order", ["shuffled", "ascending", "descending"])
def test_chain_closure_known_strengths(orc, C, order):
    P, perm, w = chain_matrix(C, seed=C, order=order)
    S = orc.strongest_paths(P, "serial")
    assert np.array_equal(orc.strongest_paths(P, "blocked", tile=16), S)
    assert chain_forward_ok(S, perm, w)
    assert np.all(np.diag(S) == 0)


def test_chain_closure_shifted_and_wide_values(orc):
    C = 200
    P, perm, w = chain_matrix(C, seed=3, base=70000)
    S = orc.strongest_paths(P, "serial")
    assert np.array_equal(orc.strongest_paths(P, "blocked", tile=16), S)
    assert chain_forward_ok(S, perm, w, base=70000)
    P, perm, w = chain_matrix(C, seed=4, low=2**31, high=2**32 - 1, noise=2**20)
    S = orc.strongest_paths(P, "serial")
    assert chain_forward_ok(S, perm, w)


def test_chain_check_catches_a_planted_error(orc):
    """The closed-form check is not vacuous: one weakened forward pair fails it."""
    P, perm, w = chain_matrix(64, seed=9)
    S = orc.strongest_paths(P, "serial")
    S[perm[3], perm[40]] -= 1
    assert not chain_forward_ok(S, perm, w)


@pytest.mark.parametrize("C", [11, 12, 50, 300])
def test_cyclic_ballots_known_strengths(orc, C):
    """Rotations of one order (the reference's own ballot shape, tallied by the oracle): every
    strongest path runs the cycle in single steps and has its closed-form strength."""
    ballots, perm, n = cyclic_ballots(C, seed=C)
    d = orc.tally(list(ballots), "scatter")
    assert np.array_equal(d, cyclic_tally(perm, n))
    S = orc.strongest_paths(d, "serial")
    assert np.array_equal(S, cyclic_strongest_paths(perm, n))
