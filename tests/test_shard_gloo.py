"""Multi-process sharding of independent elections, world_size 2 over gloo on CPU: every rank
derives the same work-balanced partition, closes its share (here with the CPU oracle), and
rank 0 gathers every election's ranking exactly once."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from scalingelections_b200.shard import election_cost, gather_results, partition_by_work


def test_partition_is_balanced_and_complete():
    rng = np.random.default_rng(0)
    C = np.rint(np.exp(rng.uniform(np.log(8), np.log(2048), size=500))).astype(int)
    costs = [election_cost(c) for c in C]
    for world in (1, 2, 3, 8):
        parts = partition_by_work(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs) + 1e-6
    assert partition_by_work(costs, 4) == partition_by_work(list(costs), 4)  # deterministic


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, specs, results_path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle

        costs = [election_cost(C, V, with_tally=True) for (C, V, _) in specs]
        mine = partition_by_work(costs, world)[rank]
        local = {}
        for i in mine:
            C, V, seed = specs[i]
            b = oracle.mallows_ballots(V, C, 0.7, seed)
            S = oracle.strongest_paths(oracle.tally(b, "positions"), "serial")
            local[i] = oracle.wins_and_ranking(S)[1].tolist()
        merged = gather_results(local, world)
        if rank == 0:
            np.save(results_path, np.array([merged[i] for i in range(len(specs))], dtype=object), allow_pickle=True)
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_shards_and_gathers(tmp_path):
    from oracle import oracle

    oracle.lib()
    specs = [(int(c), int(v), s) for s, (c, v) in enumerate([(5, 30), (40, 9), (17, 100), (60, 7), (3, 11), (33, 50)])]
    out = tmp_path / "merged.npy"
    mp.start_processes(_worker, args=(2, _free_port(), specs, str(out)), nprocs=2, join=True, start_method="spawn")
    merged = np.load(out, allow_pickle=True)
    for i, (C, V, seed) in enumerate(specs):
        b = oracle.mallows_ballots(V, C, 0.7, seed)
        S = oracle.strongest_paths(oracle.tally(b, "positions"), "serial")
        assert list(merged[i]) == oracle.wins_and_ranking(S)[1].tolist()
