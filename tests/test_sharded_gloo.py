"""The sharded closure's rounds (scalingelections_b200.sharded) over two gloo ranks on CPU.
Each rank runs the real driver, strongest_paths_sharded, with its one asynchronous broadcast
per round in look-ahead order; a numpy model of one shard stands in for the GPU kernels. The
model does the same tile steps: pivot closure, pivot-row panel, column panels, remainder, with
a receive buffer per round parity, and it checks the order (row block k+1 before the next
pivot, the rest after). The gathered rows must equal the oracle's closure exactly."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from scalingelections_b200.sharded import owner_of, row_block_bounds

T = 128


def maxmin(A, B):
    return np.max(np.minimum(A[:, :, None], B[None, :, :]), axis=1)


class ModelShard:
    """Row blocks [b0, b1) of the padded working matrix, as the GPU shard holds them."""

    def __init__(self, C, b0, b1, lanes, offset):
        self.C, self.b0, self.b1 = C, b0, b1
        self.Cp = (C + T - 1) // T * T
        self.slab = torch.zeros(((b1 - b0) * T, self.Cp), dtype=torch.int64)
        self.P = torch.zeros((2, T, self.Cp), dtype=torch.int64)  # receive buffers by round parity
        self.done = {}  # round -> local row blocks already updated in it

    def init(self, d):
        dn = d.view(torch.int32).numpy().view(np.uint32).astype(np.int64)
        S = np.where(dn > dn.T, dn, 0)
        np.fill_diagonal(S, 0)
        full = np.zeros((self.Cp, self.Cp), dtype=np.int64)
        full[:self.C, :self.C] = S
        self.slab.numpy()[:] = full[self.b0 * T:self.b1 * T]

    def _blk(self, a, r, c):
        return a[r * T:(r + 1) * T, c * T:(c + 1) * T]

    def pivot(self, k):
        if k > 0:  # the pivot row block must have had round k-1's update
            assert k - self.b0 in self.done.get(k - 1, set()), ("pivot before its row block's update", k)
        s = self.slab.numpy()
        kl = k - self.b0
        D = self._blk(s, kl, k)
        for p in range(T):
            D[:] = np.maximum(D, np.minimum(D[:, p:p + 1], D[p:p + 1, :].copy()))
        for J in range(self.Cp // T):
            if J != k:
                P = self._blk(s, kl, J)
                P[:] = np.maximum(P, maxmin(D, P))

    def panel(self, k):
        if self.b0 <= k < self.b1:
            return self.slab[(k - self.b0) * T:(k - self.b0 + 1) * T]
        return self.P[k % 2]

    def update(self, k):
        self.update_part(k, 0)

    def update_part(self, k, part):
        s = self.slab.numpy()
        own = self.b0 <= k < self.b1
        nl = k + 1 - self.b0 if self.b0 <= k + 1 < self.b1 else -1
        row = self.panel(k).numpy()
        D = row[:, k * T:(k + 1) * T]
        mine = [I for I in range(self.b1 - self.b0) if not (own and I == k - self.b0)]
        if part == 1:
            mine = [I for I in mine if I == nl]
        elif part == 2:
            mine = [I for I in mine if I != nl]
        done = self.done.setdefault(k, set())
        assert not done & set(mine), ("row block updated twice", k)
        done.update(mine)
        for I in mine:
            Cb = self._blk(s, I, k)
            Cb[:] = np.maximum(Cb, maxmin(Cb, D))
        for I in mine:
            for J in range(self.Cp // T):
                if J != k:
                    X = self._blk(s, I, J)
                    X[:] = np.maximum(X, maxmin(self._blk(s, I, k), row[:, J * T:(J + 1) * T]))

    def finalize(self):
        rows = min(self.b1 * T, self.C) - self.b0 * T
        out = self.slab.numpy()[:rows, :self.C].copy()
        for r in range(rows):
            if self.b0 * T + r < self.C:
                out[r, self.b0 * T + r] = 0
        return torch.from_numpy(out)

    def check(self):
        pass

    def close(self):
        pass


def test_bounds_and_owners():
    for R in (1, 2, 5, 17, 512):
        for parts in range(1, min(R, 9) + 1):
            b = row_block_bounds(R, parts)
            assert b[0][0] == 0 and b[-1][1] == R and all(x[1] == y[0] for x, y in zip(b, b[1:]))
            sizes = [hi - lo for lo, hi in b]
            assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1
            for k in range(R):
                lo, hi = b[owner_of(k, b)]
                assert lo <= k < hi
    with pytest.raises(ValueError):
        row_block_bounds(3, 4)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, d_np, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from scalingelections_b200.sharded import strongest_paths_sharded

        d = torch.from_numpy(d_np)
        rows, (r0, r1) = strongest_paths_sharded(d, shard_factory=ModelShard)
        np.save(os.path.join(out_dir, f"rows{rank}.npy"), rows.numpy())
        np.save(os.path.join(out_dir, f"range{rank}.npy"), np.array([r0, r1]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("C,world", [(300, 2), (520, 2), (400, 3)])
def test_sharded_rounds_over_gloo(tmp_path, orc, C, world):
    rng = np.random.default_rng(C)
    V = 101
    d = orc.tally([rng.permutation(C) for _ in range(V)])
    mp.spawn(_worker, args=(world, _free_port(), d, str(tmp_path)), nprocs=world, join=True)
    got = np.zeros((C, C), dtype=np.int64)
    covered = 0
    for r in range(world):
        r0, r1 = np.load(tmp_path / f"range{r}.npy")
        got[r0:r1] = np.load(tmp_path / f"rows{r}.npy")
        covered += r1 - r0
    assert covered == C
    assert np.array_equal(got.astype(np.uint32), orc.strongest_paths(d, "blocked", tile=16))
