"""Batched persistent closure: every election's strongest paths, wins and ranking are
bit-identical to the CPU oracle (and hence to the reference) whether closed alone or inside
a mixed batch; graph replay; lane modes; error reporting."""
import numpy as np
import pytest
import torch

from scalingelections_b200 import LANES_U16, LANES_U32, api
from scalingelections_b200.batch import BatchedElections

pytestmark = pytest.mark.gpu


def make_batch(seed, sizes, highs):
    rng = np.random.default_rng(seed)
    host = []
    for C, hi in zip(sizes, highs):
        host.append(rng.integers(0, hi, size=(C, C), dtype=np.uint64).astype(np.uint32))
    dev = [api._to_device_u32(P, "cuda") for P in host]
    return host, dev


def check_against_oracle(orc, host, batch):
    for e, P in enumerate(host):
        S_ref = orc.strongest_paths(P, "blocked", tile=32)
        got = api._to_host_u32(batch.outs[e])
        assert np.array_equal(got, S_ref), f"election {e} C={P.shape[0]}"
        wins_ref, rank_ref = orc.wins_and_ranking(S_ref)
        assert np.array_equal(batch.wins[e].cpu().numpy(), wins_ref), f"wins {e}"
        assert np.array_equal(batch.rankings[e].cpu().numpy(), rank_ref), f"ranking {e}"


def test_mixed_batch_matches_oracle(orc):
    rng = np.random.default_rng(1)
    sizes = [1, 2, 3, 8, 31, 64, 100, 127, 128, 129, 200, 255, 256, 257, 300, 384, 450, 513, 640]
    sizes += list(rng.integers(1, 700, size=25))
    highs = [int(rng.choice([3, 50, 4000, 60000, 2**32 - 1])) for _ in sizes]
    host, dev = make_batch(2, sizes, highs)
    b = BatchedElections(dev)  # lanes chosen from each matrix's maximum
    assert set(b.lanes) == {LANES_U16, LANES_U32}
    b.run()
    b.check()
    check_against_oracle(orc, host, b)


def test_wide_micro_tile_queue_matches_oracle(orc):
    """Elections given the wide micro-tile run in a third persistent launch of 256-thread CTAs:
    the same results as the oracle, beside default-micro-tile and 32-bit elections in one batch;
    a small election (C <= 128) asked to be wide runs on the default, and the wide micro-tile
    in 32-bit lanes is refused."""
    sizes = [60, 129, 200, 257, 300, 384, 513, 700, 130, 450, 90]
    highs = [4000] * 8 + [2**32 - 1, 2**32 - 1, 60000]
    host, dev = make_batch(11, sizes, highs)
    lanes = [LANES_U16] * 8 + [LANES_U32, LANES_U32, LANES_U16]
    micro = [4, 4, 8, 4, 8, 4, 4, 4, 8, 8, 4]
    b = BatchedElections(dev, lanes, micro_tiles=micro)
    counts = b.task_counts()
    assert counts[2] > 0 and counts[0] > 0 and counts[1] > 0
    b.run()
    b.check()
    check_against_oracle(orc, host, b)
    b.build_graph()
    b.launch_graph()
    b.check()
    check_against_oracle(orc, host, b)
    with pytest.raises(api.SchulzeError, match="micro_tile"):
        BatchedElections(dev[8:9], [LANES_U32], micro_tiles=[4])


def test_alone_equals_in_batch():
    sizes = [40, 130, 300, 520]
    host, dev = make_batch(3, sizes, [1000] * 4)
    b = BatchedElections(dev, [LANES_U16] * 4)
    b.run()
    b.check()
    for e, d in enumerate(dev):
        alone = api.strongest_paths_device(d, lanes=LANES_U16)
        assert torch.equal(alone.view(torch.int32), b.outs[e].view(torch.int32))
        w, r = api.rank_device(alone)
        assert torch.equal(w, b.wins[e]) and torch.equal(r, b.rankings[e])


def test_graph_replay_and_order(orc):
    sizes = [5, 77, 128, 260, 390]
    host, dev = make_batch(4, sizes, [300] * 5)
    b0 = BatchedElections(dev, [LANES_U16] * 5, order=0)
    b1 = BatchedElections(dev, [LANES_U32] * 5, order=1)
    b0.launch_graph()
    b1.launch_graph()
    b0.check()
    b1.check()
    for e in range(5):
        assert torch.equal(b0.outs[e].view(torch.int32), b1.outs[e].view(torch.int32))
    check_against_oracle(orc, host, b0)
    # New inputs written in place, same graph: fresh results.
    host2, dev2 = make_batch(5, sizes, [300] * 5)
    for d, d2 in zip(dev, dev2):
        d.copy_(d2)
    b0.launch_graph()
    b0.check()
    check_against_oracle(orc, host2, b0)
    b0.close()
    b1.close()


def test_u16_overflow_is_reported():
    host, dev = make_batch(6, [50, 200], [70000, 70000])
    b = BatchedElections(dev, [LANES_U16, LANES_U16])
    b.run()
    with pytest.raises(api.SchulzeError, match="65535"):
        b.check()


def test_without_ranking():
    host, dev = make_batch(7, [10, 150], [9, 9])
    b = BatchedElections(dev, ranking=False)
    b.run()
    b.check()
    for e, P in enumerate(host):
        assert b.wins[e] is None


def test_shifted_lanes_for_large_electorates(orc):
    """Tallies of more than 65535 ballots in 16-bit lanes shifted by V // 2 (lanes_for_voters):
    bit-identical to the oracle, and to 32-bit lanes."""
    from scalingelections_b200.batch import lanes_for_voters

    Vs = [70000, 100000, 131070]
    host, dev, lanes = [], [], []
    for n, (V, C) in enumerate(zip(Vs, [60, 150, 290])):
        b = orc.mallows_ballots(V, C, 0.9, seed=n)
        d = orc.tally(b, "positions")
        host.append(d)
        dev.append(api._to_device_u32(d, "cuda"))
        lanes.append(lanes_for_voters(V))
    assert all(l[0] == LANES_U16 and l[1] > 0 for l in lanes)
    b16 = BatchedElections(dev, lanes)
    b16.run()
    b16.check()
    check_against_oracle(orc, host, b16)
    b32 = BatchedElections(dev, [LANES_U32] * 3)
    b32.run()
    b32.check()
    for e in range(3):
        assert torch.equal(b16.outs[e].view(torch.int32), b32.outs[e].view(torch.int32))
    # A window that does not hold the values is reported, not silently wrong.
    bad = BatchedElections(dev[:1], [(LANES_U16, 0)])
    bad.run()
    with pytest.raises(api.SchulzeError):
        bad.check()


def test_dependency_wait_that_runs_out_reports_an_error_and_the_gpu_stays_usable(orc):
    """Failure detection without a GPU fault. With the dependency-wait limit at zero, the panel
    tasks, claimed as the kernel starts, find round 0's pivot tiles (tens of microseconds of
    work) unfinished, and their waits run out: the run ends with SE_ERR_DEVICE, every CTA
    drains the queue, and the context stays usable. With the limit restored the same plan
    runs exactly, through a rebuilt graph too."""
    from scalingelections_b200 import _lib

    sizes = [1000, 900, 700, 600, 513]
    host, dev = make_batch(11, sizes, [5000] * len(sizes))
    b = BatchedElections(dev, [LANES_U16] * len(sizes))
    b.set_wait_limit(0.0)
    b.run()
    with pytest.raises(_lib.SchulzeError) as e:
        b.check()
    assert e.value.status == _lib.SE_ERR_DEVICE and "dependency" in str(e.value)
    x = torch.arange(1 << 20, device="cuda", dtype=torch.int64)
    assert int(x.sum().item()) == (1 << 20) * ((1 << 20) - 1) // 2  # the context still works
    b.set_wait_limit(5.0)
    b.run()
    b.check()
    check_against_oracle(orc, host, b)
    b.launch_graph()
    b.check()
    check_against_oracle(orc, host, b)
