"""The batched-closure autotuner measures every candidate (lane mode per size bucket; CTAs per
SM and queue order for the whole launch) and its choices drive a batch that stays bit-exact."""
import numpy as np
import pytest
import torch

from scalingelections_b200 import api, autotune
from scalingelections_b200.batch import BatchedElections

pytestmark = pytest.mark.gpu


def test_autotune_table_and_choice(tmp_path):
    table = autotune.tune(V=70000, per_bucket=3, reps=1, path=tmp_path / "t.json")
    assert autotune.load(tmp_path / "t.json") == table
    assert set(table["buckets"]) == {str(b) for b in range(len(autotune.BUCKETS))}
    for entry in table["buckets"].values():
        assert entry["lanes"] in (16, 32)
        assert all(ms > 0 for ms in entry["ms"].values())
    assert table["ctas_per_sm"] in (1, 2) and table["order"] in (0, 1)
    assert len(table["launch_ms"]) == 4 and all(ms > 0 for ms in table["launch_ms"].values())
    Cs, Vs = [5, 100, 300, 700], [40, 2000, 70000, 90000]
    lanes, order, ctas = autotune.choose(table, Cs, Vs)
    rng = np.random.default_rng(0)
    prefs, host = [], []
    for C, V in zip(Cs, Vs):
        up = rng.integers(0, V + 1, size=(C, C))
        d = (np.triu(up, 1) + np.triu(V - up, 1).T).astype(np.uint32)
        host.append(d)
        prefs.append(api._to_device_u32(d, "cuda"))
    b = BatchedElections(prefs, lanes, order=order, ctas_per_sm=ctas)
    b.run()
    b.check()
    for e, d in enumerate(host):
        alone = api.strongest_paths_device(prefs[e], lanes=api.LANES_U32)
        assert torch.equal(alone.view(torch.int32), b.outs[e].view(torch.int32))
