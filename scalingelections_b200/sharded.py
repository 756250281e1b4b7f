"""One election's widest-path closure sharded across GPUs by row blocks (include/se.h,
se_shard_*). No reference counterpart: the reference closes one matrix on one GPU
(scaling_elections.cu:490-578).

Each rank holds a contiguous range of the R = ceil(C / 128) row blocks. Round k has one
exchange: the rank holding row block k closes the pivot tile and updates its pivot-row panel,
and that panel (128 x Cp cells) is broadcast to the others. Every rank then updates its own
rows. The remainder work, nearly all of it, splits evenly across the ranks; each round moves
one panel over NVLink, 16 MiB at C = 65536 in 16-bit lanes.

On two or more ranks the rounds run in look-ahead order: in round k the rank holding row
block k+1 updates that row block first (closing the next pivot tile in the same launch) and
its pivot-row panel, and the broadcast of panel k+1 starts asynchronously before every rank
updates the rest of its rows for round k. So the panel, and the next pivot's chain, overlap
round k's remainder instead of following it; receivers keep one panel buffer per round parity.
One rank has nothing to overlap and runs each round whole (the split launches cost it 4 % at
C = 16384).

``strongest_paths_sharded`` runs the rounds with ``torch.distributed`` (NCCL on GPUs); each
rank needs the whole preference matrix on its GPU and gets back its own rows.
``strongest_paths_virtual`` runs the same rounds with several shards in one process on one
GPU, the broadcast being a device-to-device copy. It exercises the sharded data flow where
only one GPU is available.
"""
from __future__ import annotations

import ctypes
from bisect import bisect_right
from typing import Callable

import torch

from . import _lib
from ._lib import LANES_U16, LANES_U32, check

TILE = 128


def row_block_bounds(R: int, parts: int) -> list[tuple[int, int]]:
    """Contiguous row-block ranges [b0, b1) for `parts` shards, sizes differing by at most one."""
    if parts < 1 or parts > R:
        raise ValueError(f"cannot split {R} row blocks into {parts} non-empty shards")
    q, r = divmod(R, parts)
    out, b = [], 0
    for p in range(parts):
        n = q + (1 if p < r else 0)
        out.append((b, b + n))
        b += n
    return out


def owner_of(k: int, bounds: list[tuple[int, int]]) -> int:
    return bisect_right([b0 for b0, _ in bounds], k) - 1


def _lanes_for(d: torch.Tensor, lanes) -> tuple[int, int]:
    if isinstance(lanes, (tuple, list)):
        return int(lanes[0]), int(lanes[1])
    if lanes in (LANES_U16, LANES_U32):
        return int(lanes), 0
    # Automatic: 16-bit lanes when every count fits them unshifted (one device-to-host read).
    hi = int(d.view(torch.int32).max().item()) if d.numel() else 0
    return (LANES_U16, 0) if 0 <= hi <= 0xFFFF else (LANES_U32, 0)


class Shard:
    """Row blocks [b0, b1) of one election's working matrix on this GPU."""

    def __init__(self, C: int, b0: int, b1: int, lanes: int = LANES_U16, value_offset: int = 0, device=None):
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.C, self.b0, self.b1 = int(C), int(b0), int(b1)
        L = _lib.lib()
        self.L = L
        need = L.se_shard_workspace_bytes(self.C, self.b0, self.b1, int(lanes))
        if need < 0:
            raise ValueError("invalid shard")
        self.work = torch.empty(need, dtype=torch.uint8, device=self.device)
        self.handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            check(L.se_shard_create(self.C, self.b0, self.b1, int(lanes), int(value_offset), self.work.data_ptr(), need,
                                    ctypes.byref(self.handle)))
        self.panel_bytes = int(L.se_shard_panel_bytes(self.handle))

    def _stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    def init(self, d: torch.Tensor) -> None:
        if d.shape != (self.C, self.C) or d.dtype != torch.uint32 or d.device != self.device or d.stride(1) != 1:
            raise ValueError("d must be the whole uint32 [C, C] matrix on this shard's device, rows contiguous")
        self._d = d
        with torch.cuda.device(self.device):
            check(self.L.se_shard_init(self.handle, d.data_ptr(), d.stride(0), self._stream()))

    def pivot(self, k: int) -> None:
        with torch.cuda.device(self.device):
            check(self.L.se_shard_pivot(self.handle, int(k), self._stream()))

    def panel(self, k: int) -> torch.Tensor:
        """The bytes of pivot-row panel k: what the owner sends, where the others receive."""
        off = int(self.L.se_shard_panel_offset(self.handle, int(k)))
        if off < 0:
            raise ValueError("round out of range")
        return self.work[off:off + self.panel_bytes]

    def update(self, k: int) -> None:
        with torch.cuda.device(self.device):
            check(self.L.se_shard_update(self.handle, int(k), self._stream()))

    def update_part(self, k: int, part: int) -> None:
        """Round k's update in parts: 1 row block k+1 alone (closing the next pivot tile),
        2 every other row; 0 both (se_shard_update_part)."""
        with torch.cuda.device(self.device):
            check(self.L.se_shard_update_part(self.handle, int(k), int(part), self._stream()))

    def finalize(self) -> torch.Tensor:
        rows = min(self.b1 * TILE, self.C) - self.b0 * TILE
        out = torch.empty((max(rows, 0), self.C), dtype=torch.uint32, device=self.device)
        if rows > 0:
            with torch.cuda.device(self.device):
                check(self.L.se_shard_finalize(self.handle, out.data_ptr(), self.C, self._stream()))
        return out

    def check(self) -> None:
        with torch.cuda.device(self.device):
            check(self.L.se_shard_check(self.handle, self._stream()))

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.L.se_shard_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def strongest_paths_sharded(d: torch.Tensor, *, group=None, lanes=None,
                            shard_factory: Callable | None = None) -> tuple[torch.Tensor, tuple[int, int]]:
    """The closure of the whole uint32 [C, C] matrix d, sharded over the ranks of `group`
    (torch.distributed, initialised by the caller; every rank passes the same d). Returns this
    rank's rows of the strongest-path matrix and their range [row0, row1). Bit-identical to
    the single-GPU closure. Needs at least as many row blocks (ceil(C / 128)) as ranks.
    shard_factory(C, b0, b1, lanes, value_offset) may stand in for Shard (tests use a CPU model
    of the same rounds)."""
    import torch.distributed as dist

    C = int(d.shape[0])
    R = (C + TILE - 1) // TILE
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    bounds = row_block_bounds(R, world)
    lane_bits, offset = _lanes_for(d, lanes)
    make = shard_factory or (lambda C_, b0, b1, lb, off: Shard(C_, b0, b1, lb, off, device=d.device))
    b0, b1 = bounds[rank]
    sh = make(C, b0, b1, lane_bits, offset)
    sh.init(d)

    def send(k):  # every rank, same order: the broadcast of panel k, in flight until waited
        owner = owner_of(k, bounds)
        src = owner if group is None else dist.get_global_rank(group, owner)
        return dist.broadcast(sh.panel(k), src=src, group=group, async_op=True)

    if owner_of(0, bounds) == rank:
        sh.pivot(0)
    work = send(0)
    lookahead = world > 1
    for k in range(R):
        work.wait()  # panel k is here (for NCCL: the caller's stream waits for it)
        if not lookahead:
            sh.update(k)
            if k + 1 < R:
                if owner_of(k + 1, bounds) == rank:
                    sh.pivot(k + 1)
                work = send(k + 1)
        elif k + 1 < R:
            if owner_of(k + 1, bounds) == rank:
                sh.update_part(k, 1)
                sh.pivot(k + 1)
            work = send(k + 1)
            sh.update_part(k, 2)
        else:
            sh.update(k)
    out = sh.finalize()
    sh.check()
    sh.close()
    return out, (b0 * TILE, min(b1 * TILE, C))


def strongest_paths_virtual(d: torch.Tensor, parts: int, *, lanes=None, lookahead: bool = True) -> torch.Tensor:
    """The same rounds with `parts` shards in one process on d's GPU, panels copied device to
    device; returns the whole strongest-path matrix. Exercises the sharded data flow on one GPU.
    No shard ever waits on another: every launch of a round comes after the copy it reads.
    lookahead: the order of strongest_paths_sharded (row block k+1 and its pivot panel first);
    False: pivot, broadcast, whole update per round. Both give identical results."""
    C = int(d.shape[0])
    R = (C + TILE - 1) // TILE
    bounds = row_block_bounds(R, parts)
    lane_bits, offset = _lanes_for(d, lanes)
    shards = [Shard(C, b0, b1, lane_bits, offset, device=d.device) for b0, b1 in bounds]

    def send(k):
        o = owner_of(k, bounds)
        src = shards[o].panel(k)
        for p, sh in enumerate(shards):
            if p != o:
                sh.panel(k).copy_(src)

    try:
        for sh in shards:
            sh.init(d)
        # The look-ahead order of strongest_paths_sharded, one stream.
        shards[owner_of(0, bounds)].pivot(0)
        send(0)
        for k in range(R):
            if not lookahead:
                if k > 0:
                    shards[owner_of(k, bounds)].pivot(k)
                    send(k)
                for sh in shards:
                    sh.update(k)
            elif k + 1 < R:
                o = owner_of(k + 1, bounds)
                shards[o].update_part(k, 1)
                shards[o].pivot(k + 1)
                send(k + 1)
                for sh in shards:
                    sh.update_part(k, 2)
            else:
                for sh in shards:
                    sh.update(k)
        rows = [sh.finalize() for sh in shards]
        for sh in shards:
            sh.check()
        return torch.cat([r.view(torch.int32) for r in rows], dim=0).view(torch.uint32)
    finally:
        for sh in shards:
            sh.close()
