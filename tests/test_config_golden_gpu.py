"""Single-election configurations against the reference's own outputs on the same ballots:
C = 4096, V = 4096 uniform permutations, the headline C = 16384, V = 4096 Mallows(0.8)
ballots, and C = 32768, V = 4096 Mallows(0.8). The outputs were produced by
tests/golden/make_golden.py from scaling_elections.py:
  * the tally of build_pairwise_preferences (py:51-88; at C = 32768 run over slices of the
    voters in parallel and summed, which the generator checks at C = 16384 against the single
    call's hash),
  * the strongest paths of compute_strongest_paths_numba_parallel, tile 16 (py:162-271); at
    C = 4096 also checked there equal to the serial Numba path (py:91-125); at C = 32768 the
    reference's OpenMP closure (scaling_elections.cu:738-849, tile 16), which the generator
    checks at C = 16384 against the Numba hash,
  * the ranking and winner of get_winner_and_ranking (py:274-296).
The fixture holds hashes and the ranking; the ballots are regenerated from their seed."""
import hashlib
import json
import os
from pathlib import Path

import numpy as np
import pytest

from scalingelections_b200 import LANES_U16, LANES_U32, api
from scalingelections_b200.ballots import uniform_ballots

GOLDEN = Path(__file__).parent / "golden"
CASE = json.loads((GOLDEN / "config_c4096_v4096.json").read_text())


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint32).tobytes()).hexdigest()


def ballots():
    return uniform_ballots(CASE["V"], CASE["C"], seed=CASE["seed"])


@pytest.mark.gpu
def test_config_c4096_matches_reference():
    d = api.build_pairwise_preferences(ballots())
    assert sha(d) == CASE["tally_sha256"]
    for lanes in (LANES_U16, LANES_U32):  # V < 65536: both lane modes are exact here
        S = api.compute_strongest_paths(d, allow_gpu=True, tile_size=32, lanes=lanes)
        assert sha(S) == CASE["strongest_sha256"], lanes
    winner, ranking = api.get_winner_and_ranking(list(range(CASE["C"])), S)
    assert winner == CASE["winner"]
    assert list(ranking) == CASE["ranking"]


@pytest.mark.skipif(not os.environ.get("SE_TEST_SLOW"), reason="about a minute on one core; set SE_TEST_SLOW=1")
def test_oracle_tally_at_config_size(orc):
    """The C oracle's tally on the same ballots gives the reference's tally (CPU)."""
    assert sha(orc.tally(list(ballots()))) == CASE["tally_sha256"]


@pytest.mark.gpu
def test_config_c16384_matches_reference(orc):
    """The headline size. The ballots come from the oracle's C decode of the package's host
    Mallows sampler (the same stream, 15x faster); the tally hash pins them."""
    path = GOLDEN / "config_c16384_v4096.json"
    if not path.exists():
        pytest.skip("fixture not generated")
    case = json.loads(path.read_text())
    B = orc.mallows_ballots(case["V"], case["C"], case["phi"], seed=case["seed"])
    d = api.build_pairwise_preferences(B)
    del B
    assert sha(d) == case["tally_sha256"]
    S = api.compute_strongest_paths(d, allow_gpu=True, tile_size=32)  # 16-bit lanes: V < 65536
    assert sha(S) == case["strongest_sha256"]
    winner, ranking = api.get_winner_and_ranking(list(range(case["C"])), S)
    assert winner == case["winner"]
    assert list(ranking) == case["ranking"]


@pytest.mark.gpu
def test_config_c32768_matches_reference(orc):
    """The larger size of the headline configuration, through the drop-in API."""
    path = GOLDEN / "config_c32768_v4096.json"
    if not path.exists():
        pytest.skip("fixture not generated")
    case = json.loads(path.read_text())
    B = orc.mallows_ballots(case["V"], case["C"], case["phi"], seed=case["seed"])
    d = api.build_pairwise_preferences(B)
    del B
    assert sha(d) == case["tally_sha256"]
    S = api.compute_strongest_paths(d, allow_gpu=True, tile_size=32)
    del d
    assert sha(S) == case["strongest_sha256"]
    winner, ranking = api.get_winner_and_ranking(list(range(case["C"])), S)
    assert winner == case["winner"]
    assert list(ranking) == case["ranking"]
