"""Strongest paths that run the length of the matrix, on the GPU.

Random and Mallows matrices give strongest paths of a few hops. A chain of strong defeats over
weak noise (conftest.chain_matrix) gives paths of up to C - 1 hops. Those carry a path through
every round, every pivot block and every consecutive pivot pair:
  * the in-register pivot closure's pair fix-ups and its publish of each group of 8 pivots;
  * the split tiles' max-folds;
  * the panels that ride in the remainder launch;
  * the batch's dependency counters;
  * the sharded look-ahead.
Each result is compared with the oracle (up to C = 2305) or with the closed-form strength of
every forward pair along the chain and with every other schedule (C = 4100)."""
import numpy as np
import pytest
import torch

from conftest import chain_forward_ok, chain_matrix
from scalingelections_b200 import LANES_AUTO, LANES_U16, LANES_U32, api
from scalingelections_b200.batch import BatchedElections
from scalingelections_b200.sharded import strongest_paths_virtual

pytestmark = pytest.mark.gpu

SCHEDULES = (0, 1, 2, 3, 4, 5, 6, 7, 8)


def closure(P, lanes):
    d = api._to_device_u32(np.ascontiguousarray(P, dtype=np.uint32), "cuda")
    return api._to_host_u32(api.strongest_paths_device(d, lanes=lanes))


def every_schedule(P, lane_list):
    """{(schedule, lanes): result} over every closure schedule."""
    out = {}
    try:
        for mode in SCHEDULES:
            api.set_closure_mode(mode)
            for lanes in lane_list:
                out[(mode, lanes)] = closure(P, lanes)
    finally:
        api.set_closure_mode(0)
    return out


@pytest.mark.parametrize("C", [129, 300, 1000, 2305])
@pytest.mark.parametrize("order", ["shuffled", "ascending", "descending"])
def test_chain_every_schedule_against_oracle(orc, C, order):
    P, perm, w = chain_matrix(C, seed=C, order=order)
    S_ref = orc.strongest_paths(P, "blocked", tile=16)
    assert chain_forward_ok(S_ref, perm, w)
    for key, S in every_schedule(P, (LANES_U16, LANES_U32, LANES_AUTO)).items():
        assert np.array_equal(S, S_ref), key


@pytest.mark.parametrize("C", [300, 2305])
def test_chain_shifted_and_wide_values(orc, C):
    """A chain in a shifted 16-bit window (counts above 65535 that span less than 16 bits),
    and one whose counts need all 32 bits."""
    P, perm, w = chain_matrix(C, seed=C + 1, base=70000)
    S_ref = orc.strongest_paths(P, "blocked", tile=16)
    assert chain_forward_ok(S_ref, perm, w, base=70000)
    for key, S in every_schedule(P, (LANES_AUTO,)).items():
        assert np.array_equal(S, S_ref), key
    P, perm, w = chain_matrix(C, seed=C + 2, low=2**31, high=2**32 - 1, noise=2**20)
    S_ref = orc.strongest_paths(P, "blocked", tile=16)
    for key, S in every_schedule(P, (LANES_U32, LANES_AUTO)).items():
        assert np.array_equal(S, S_ref), key


@pytest.mark.parametrize("order", ["shuffled", "descending"])
def test_chain_beyond_the_split_tiles(order):
    """C = 4100: 33 row blocks, past the 28 that split their panel tiles, with a partial last
    block. Every forward pair has its closed-form strength and every schedule agrees."""
    P, perm, w = chain_matrix(4100, seed=41, order=order)
    results = every_schedule(P, (LANES_U16, LANES_U32))
    first = results[(0, LANES_U16)]
    assert chain_forward_ok(first, perm, w)
    for key, S in results.items():
        assert np.array_equal(S, first), key


def test_chain_batch_against_oracle(orc):
    """Chains of mixed sizes in one batch: 16-bit lanes on both micro-tiles, shifted 16-bit
    lanes, and 32-bit lanes; strongest paths, wins and rankings equal the oracle's."""
    specs = [  # (C, order, base, lanes, micro-tile)
        (1, "shuffled", 0, (LANES_U16, 0), 8), (2, "descending", 0, (LANES_U16, 0), 8),
        (127, "shuffled", 0, (LANES_U16, 0), 8), (128, "ascending", 0, (LANES_U16, 0), 8),
        (129, "descending", 0, (LANES_U16, 0), 4), (300, "shuffled", 0, (LANES_U16, 0), 4),
        (513, "descending", 0, (LANES_U16, 0), 8), (1000, "shuffled", 0, (LANES_U16, 0), 4),
        (700, "shuffled", 70000, (LANES_U16, 70000), 8), (640, "ascending", 70000, (LANES_U16, 70000), 4),
        (450, "shuffled", 0, (LANES_U32, 0), 8), (1300, "descending", 0, (LANES_U32, 0), 8),
    ]
    host, chains = [], []
    for i, (C, order, base, _, _) in enumerate(specs):
        P, perm, w = chain_matrix(C, seed=100 + i, order=order, base=base)
        host.append(P)
        chains.append((perm, w, base))
    dev = [api._to_device_u32(P, "cuda") for P in host]
    b = BatchedElections(dev, [s[3] for s in specs], micro_tiles=[s[4] for s in specs])
    b.run()
    b.check()
    for e, P in enumerate(host):
        S_ref = orc.strongest_paths(P, "blocked", tile=16)
        assert chain_forward_ok(S_ref, *chains[e][:2], base=chains[e][2])
        assert np.array_equal(api._to_host_u32(b.outs[e]), S_ref), f"election {e} C={P.shape[0]}"
        wins_ref, rank_ref = orc.wins_and_ranking(S_ref)
        assert np.array_equal(b.wins[e].cpu().numpy(), wins_ref), f"wins {e}"
        assert np.array_equal(b.rankings[e].cpu().numpy(), rank_ref), f"ranking {e}"


@pytest.mark.parametrize("C,parts", [(1000, 3), (2049, 5), (2305, 16)])
def test_chain_virtual_shards(C, parts):
    """The sharded closure (one GPU, several shards; with and without the look-ahead
    broadcast order) on a chain equals the single closure, which has the closed-form strengths."""
    P, perm, w = chain_matrix(C, seed=C + parts, order="shuffled")
    d = api._to_device_u32(P, "cuda")
    single = api.strongest_paths_device(d, lanes=LANES_U16)
    assert chain_forward_ok(api._to_host_u32(single), perm, w)
    for lanes in (LANES_U16, LANES_U32):
        for lookahead in (True, False):
            got = strongest_paths_virtual(d, parts, lanes=lanes, lookahead=lookahead)
            assert torch.equal(got.view(torch.int32), single.view(torch.int32)), (lanes, lookahead)
