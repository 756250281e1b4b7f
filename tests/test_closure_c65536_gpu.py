"""C = 65536 on one GPU (a 16 GiB preference matrix, 8 GiB working matrix in 16-bit lanes): the
capacity for which multi-GPU sharding of one election was first considered. Properties
that do not depend on size: exact rows from an independent bottleneck Dijkstra, dominance over
the defeat matrix, a zero diagonal. Opt-in (it holds about 40 GB on the device and runs for
about a minute): set SE_TEST_HUGE=1."""
import os

import numpy as np
import pytest
import torch

from scalingelections_b200 import LANES_U16, api

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(os.environ.get("SE_TEST_HUGE") != "1", reason="set SE_TEST_HUGE=1")]


def test_closure_c65536_properties(orc):
    from scalingelections_b200.ballots import mallows_ballots_device

    C, V = 65536, 1024
    ids = mallows_ballots_device(V, C, 0.8, seed=65536).view(-1)
    offs = torch.arange(V + 1, dtype=torch.int64, device="cuda") * C
    d = api.tally_device(ids, offs, C)
    del ids
    torch.cuda.empty_cache()
    S = api.strongest_paths_device(d, lanes=LANES_U16)
    torch.cuda.synchronize()
    d_h = api._to_host_u32(d)
    del d
    S_h = api._to_host_u32(S)
    del S
    rows = [7, C - 3]
    assert np.array_equal(S_h[rows], orc.widest_rows(d_h, rows))
    D = orc.defeats(d_h)
    assert (S_h >= D).all()
    assert not np.diagonal(S_h).any()
