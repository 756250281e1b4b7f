"""The sharded closure's GPU kernels (se_shard_*): several shards in one process on one GPU,
panels copied device to device, and a one-rank NCCL run of the distributed driver. Every
result must equal the single-GPU closure bit for bit (and the oracle)."""
import os
import socket

import numpy as np
import pytest
import torch

from scalingelections_b200 import LANES_U16, LANES_U32, _lib, api
from scalingelections_b200.sharded import Shard, strongest_paths_sharded, strongest_paths_virtual

pytestmark = pytest.mark.gpu


def tallied(C, V, seed, phi=0.8):
    from scalingelections_b200.ballots import mallows_ballots_device

    b = mallows_ballots_device(V, C, phi, seed=seed)
    offs = torch.arange(V + 1, dtype=torch.int64, device=b.device) * C
    return api.tally_device(b.view(-1), offs, C)


def same(a, b):
    return torch.equal(a.view(torch.int32), b.view(torch.int32))


@pytest.mark.parametrize("C,parts", [(300, 1), (300, 2), (300, 3), (1000, 2), (1000, 8), (2049, 5), (2048, 16)])
def test_virtual_shards_equal_single_closure(C, parts):
    d = tallied(C, 777, seed=C + parts)
    single = api.strongest_paths_device(d, lanes=LANES_U16)
    assert same(strongest_paths_virtual(d, parts, lanes=LANES_U16), single)
    assert same(strongest_paths_virtual(d, parts, lanes=LANES_U32), single)
    assert same(strongest_paths_virtual(d, parts, lanes=LANES_U16, lookahead=False), single)


def test_virtual_shards_against_oracle(orc):
    C = 700
    d = tallied(C, 4000, seed=5, phi=1.0)
    S_ref = orc.strongest_paths(api._to_host_u32(d), "blocked", tile=16)
    assert np.array_equal(api._to_host_u32(strongest_paths_virtual(d, 3)), S_ref)


def test_virtual_shards_shifted_16_bit_lanes(orc):
    """Counts above 16 bits in a window narrower than 65535: shifted 16-bit lanes, as the batch
    and the server use them, equal 32-bit lanes."""
    rng = np.random.default_rng(8)
    C, V = 400, 150000
    up = rng.integers(75001, 140000, size=(C, C))  # kept values in [75001, 139999]: base V // 2 fits them
    P = (np.triu(up, 1) + np.triu(V - up, 1).T).astype(np.uint32)
    d = api._to_device_u32(P, torch.device("cuda"))
    ref = strongest_paths_virtual(d, 2, lanes=LANES_U32)
    assert same(strongest_paths_virtual(d, 2, lanes=(LANES_U16, V // 2)), ref)
    assert np.array_equal(api._to_host_u32(ref), orc.strongest_paths(P, "blocked", tile=16))


def test_shard_rejects_bad_calls():
    L = _lib.lib()
    assert L.se_shard_workspace_bytes(1000, 3, 2, 16) < 0
    assert L.se_shard_workspace_bytes(1000, 0, 9, 16) < 0
    assert L.se_shard_workspace_bytes(1000, 0, 8, 24) < 0
    sh = Shard(1000, 2, 5)
    with pytest.raises(_lib.SchulzeError, match="not in this shard"):
        sh.pivot(1)
    with pytest.raises(ValueError):
        sh.panel(8)
    with pytest.raises(_lib.SchulzeError, match="part must be"):
        sh.update_part(0, 3)
    assert sh.panel(0).data_ptr() != sh.panel(1).data_ptr()  # a receive buffer per round parity
    assert sh.panel(0).data_ptr() == sh.panel(6).data_ptr()  # rounds 2-4 are this shard's own rows
    sh.close()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_one_rank_nccl_run():
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        C = 1500
        d = tallied(C, 999, seed=9)
        rows, (r0, r1) = strongest_paths_sharded(d)
        torch.cuda.synchronize()
        assert (r0, r1) == (0, C)
        assert same(rows, api.strongest_paths_device(d, lanes=LANES_U16))
    finally:
        dist.destroy_process_group()
