"""Serving engine: requests arriving while others run are closed in the same persistent
kernel; every result is bit-identical to the same election run alone."""
import numpy as np
import pytest
import torch

from scalingelections_b200 import api
from scalingelections_b200.ballots import mallows_ballots_device
from scalingelections_b200.serve import Server, run_arrivals

pytestmark = pytest.mark.gpu


def make_requests(seed, n):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        C = int(rng.integers(2, 700))
        V = int(rng.integers(5, 2500))
        if i % 7 == 3:
            C, V = int(rng.integers(3, 40)), int(rng.integers(66000, 90000))  # shifted 16-bit lanes
        b = mallows_ballots_device(V, C, float(rng.uniform(0.2, 1.0)), seed=seed * 1000 + i)
        reqs.append((V, C, b))
    torch.cuda.synchronize()
    return reqs


def alone(V, C, b):
    ids = b.reshape(-1)
    offs = torch.arange(V + 1, dtype=torch.int64, device=b.device) * C
    d = api.tally_device(ids, offs, C)
    S = api.strongest_paths_device(d, lanes=api.LANES_AUTO)
    wins, ranking = api.rank_device(S)
    return api._to_host_u32(S), ranking.cpu().numpy()


def test_in_mix_equals_alone():
    reqs = make_requests(1, 24)
    server = Server(budget_bytes=2 << 30, max_slots=64, idle_ms=20)
    # Arrivals in three bursts, so requests join while earlier ones are on the GPU.
    times = [0.0] * 8 + [0.002] * 8 + [0.004] * 8
    done, _ = run_arrivals(server, reqs, times, keep_paths=True)
    server.close()
    assert len(done) == len(reqs)
    for t in done:
        V, C, b = reqs[t.rid]
        assert t.status == 0, (t.rid, t.status)
        S, ranking = alone(V, C, b)
        assert np.array_equal(t.strongest_paths, S), t.rid
        assert np.array_equal(t.ranking, ranking), t.rid


def test_admission_under_a_tight_budget(orc):
    """A budget too small for all requests at once: they queue on the host and are admitted
    as memory frees up; results stay exact."""
    reqs = make_requests(2, 10)
    with Server(budget_bytes=64 << 20, max_slots=8, idle_ms=5) as server:
        done, _ = run_arrivals(server, reqs, [0.0] * len(reqs), keep_paths=True)
    assert len(done) == len(reqs)
    for t in done:
        V, C, b = reqs[t.rid]
        d = orc.tally(b.cpu().numpy(), "positions")
        S_ref = orc.strongest_paths(d, "blocked", tile=32)
        assert np.array_equal(t.strongest_paths, S_ref), t.rid
        _, rank_ref = orc.wins_and_ranking(S_ref)
        assert np.array_equal(t.ranking, rank_ref), t.rid


def test_large_candidate_counts_beside_small_ones():
    """POS tasks build each ballot's places in a 16-bit shared-memory row per warp while four
    rows fit (C up to 12288), and in global memory beyond that: one request on each side of the
    limit, served together with small ones, each equal to the same election run alone."""
    reqs = []
    for i, (C, V) in enumerate([(12288, 150), (12400, 130), (300, 500), (50, 70000)]):
        reqs.append((V, C, mallows_ballots_device(V, C, 0.7, seed=900 + i)))
    torch.cuda.synchronize()
    server = Server(budget_bytes=8 << 30, max_slots=16, idle_ms=20)
    done, _ = run_arrivals(server, reqs, [0.0, 0.0, 0.001, 0.001], keep_paths=True)
    server.close()
    assert len(done) == len(reqs)
    for t in done:
        V, C, b = reqs[t.rid]
        assert t.status == 0, (t.rid, t.status)
        S, ranking = alone(V, C, b)
        assert np.array_equal(t.strongest_paths, S), t.rid
        assert np.array_equal(t.ranking, ranking), t.rid


def test_malformed_ballots_reported_in_status():
    V, C = 10, 6
    b = torch.arange(C, dtype=torch.int32, device="cuda").repeat(V, 1)
    b[3, 2] = 0  # repeated id in ballot 3
    server = Server(budget_bytes=64 << 20, max_slots=4, idle_ms=5)
    done, _ = run_arrivals(server, [(V, C, b)], [0.0])
    server.close()
    assert done[0].status & 8 and (done[0].status & 3) == 3


def test_host_ballots_and_cancel_in_the_mix():
    """Ballots submitted from host memory (pinned tensors and NumPy arrays, copied into the
    server's block when admitted) beside device-resident ones, under a budget that makes them
    queue; one waiting request and one in-flight request cancelled. Every result equals the
    same election run alone, and the budget is whole again at the end."""
    reqs = make_requests(3, 14)
    mixed = []
    for i, (V, C, b) in enumerate(reqs):
        if i % 3 == 0:
            h = torch.empty((V, C), dtype=torch.int32, pin_memory=True)
            h.copy_(b)
            mixed.append((V, C, h))
        elif i % 3 == 1:
            mixed.append((V, C, b.cpu().numpy()))
        else:
            mixed.append((V, C, b))
    from scalingelections_b200.serve import Ticket

    with Server(budget_bytes=256 << 20, max_slots=8, idle_ms=5) as server:
        done, _ = run_arrivals(server, mixed, [0.0] * 7 + [0.003] * 7, keep_paths=True)
        assert len(done) == len(reqs)
        # Cancel: one request cancelled before admission never runs; one cancelled after it is
        # admitted is not returned, and its memory comes back.
        V, C, b = mixed[0]
        waiting = Ticket(rid=0, V=V, C=C, arrival=0.0, keep_paths=True)
        assert server.cancel(waiting)
        pending = [waiting]
        assert server.admit(pending, lambda t: b, now=0.0) == 0 and pending == []
        flying = Ticket(rid=1, V=V, C=C, arrival=0.0)
        assert server.try_submit(flying, b)
        assert not server.cancel(flying)
        import time
        t0 = time.perf_counter()
        while server.in_flight and time.perf_counter() - t0 < 30:
            assert server.poll() == []
        assert server.in_flight == 0 and server.arena.used == 0
    for t in done:
        V, C, b = reqs[t.rid]
        assert t.status == 0, (t.rid, t.status)
        S, ranking = alone(V, C, b)
        assert np.array_equal(t.strongest_paths, S), t.rid
        assert np.array_equal(t.ranking, ranking), t.rid


def test_cyclic_ballots_in_the_mix():
    """Ballots that rotate one order, whose strongest paths run around a cycle in single steps
    (conftest.cyclic_ballots), served in bursts beside Mallows requests: each has its
    closed-form strongest paths and equals the election run alone."""
    from conftest import cyclic_ballots, cyclic_strongest_paths

    reqs, want = [], {}
    for i, C in enumerate([12, 40, 129, 300, 513, 900]):
        ballots, perm, n = cyclic_ballots(C, seed=100 + i)
        want[len(reqs)] = cyclic_strongest_paths(perm, n)
        reqs.append((len(ballots), C, torch.from_numpy(ballots).cuda()))
    reqs += make_requests(5, 6)
    with Server(budget_bytes=2 << 30, max_slots=64, idle_ms=20) as server:
        times = [0.0, 0.0, 0.002, 0.002, 0.004, 0.004] * 2
        done, _ = run_arrivals(server, reqs, times, keep_paths=True)
    assert len(done) == len(reqs)
    for t in done:
        assert t.status == 0, (t.rid, t.status)
        V, C, b = reqs[t.rid]
        S, ranking = alone(V, C, b)
        assert np.array_equal(t.strongest_paths, S), t.rid
        assert np.array_equal(t.ranking, ranking), t.rid
        if t.rid in want:
            assert np.array_equal(S, want[t.rid]), t.rid
