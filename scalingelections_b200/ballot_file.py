"""Packed ballot files, and their tally streamed through the GPU in chunks.

The reference has no on-disk ballot format: ``build_pairwise_preferences``
(scaling_elections.py:51-88) takes in-memory rank vectors, one NumPy array per voter. This
module stores the same ballots, ordered candidate ids with the most preferred first and
possibly incomplete, as one contiguous id array at the narrowest width that holds every id
(1, 2 or 4 bytes). Ragged ballots add V + 1 int64 offsets; a file in which every ballot
lists all C candidates has none. ``tally_file`` reads such a file in chunks of ballots into
pinned buffers with parallel ``pread`` calls and overlaps each chunk's host-to-device copy
with the tally of the previous chunk (``se_tally_ex`` with ``SE_TALLY_ACCUMULATE``). Device
memory stays bounded by the chunk size, so the number of ballots is limited only by the file.

File layout (little-endian; every section starts on a 64-byte boundary)::

    offset  type   field
    0       8s     magic b"SEBALLOT"
    8       u32    version (1)
    12      u32    id_bytes: 1, 2 or 4 (uint8, uint16 or int32 ids)
    16      u64    V, the number of ballots
    24      u32    C, the number of candidates: every id is in [0, C)
    28      u32    flags: bit 0 set when every ballot lists exactly C ids (no offsets section)
    32      u64    n_ids, the total number of ids
    40      u64    byte offset of the ids section
    48      u64    byte offset of the offsets section (V + 1 int64, first 0), or 0
    56      u64    reserved, 0

Incomplete ballots follow the reference's completion rule when tallied: the missing ids
take the places after the listed ones, in ascending id order (scaling_elections.py:75-83).
"""
from __future__ import annotations

import os
import struct
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass
from typing import Iterator

import numpy as np
import torch

from . import _lib
from ._lib import SchulzeError, check

MAGIC = b"SEBALLOT"
VERSION = 1
HEADER = struct.Struct("<8sIIQIIQQQQ")
FLAG_COMPLETE = 1
_ALIGN = 64
_ID_DTYPES = {1: np.uint8, 2: np.uint16, 4: np.int32}

SE_TALLY_ACCUMULATE = 1
SE_TALLY_NO_SYNC = 2
SE_TALLY_KEEP_ERROR = 4


def id_width(num_candidates: int) -> int:
    """Bytes per id: the narrowest of 1, 2, 4 that holds ids in [0, C)."""
    C = int(num_candidates)
    if C <= 1 << 8:
        return 1
    if C <= 1 << 16:
        return 2
    if C <= 1 << 31:
        return 4
    raise ValueError("too many candidates")


def _align(x: int) -> int:
    return (x + _ALIGN - 1) // _ALIGN * _ALIGN


@dataclass(frozen=True)
class Header:
    id_bytes: int
    num_voters: int
    num_candidates: int
    flags: int
    num_ids: int
    ids_offset: int
    offsets_offset: int

    @property
    def complete(self) -> bool:
        return bool(self.flags & FLAG_COMPLETE)


def _as_csr(voter_rankings) -> tuple[np.ndarray | None, np.ndarray | None, list | None, int]:
    """(ids, offsets, rankings, max id + 1). A 2-D array yields ids and offsets directly; a
    sequence of arrays is kept as is and written in pieces."""
    if isinstance(voter_rankings, np.ndarray) and voter_rankings.ndim == 2:
        V, L = voter_rankings.shape
        ids = np.ascontiguousarray(voter_rankings).reshape(-1)
        offsets = np.arange(V + 1, dtype=np.int64) * L
        if ids.size and int(ids.min()) < 0:
            raise ValueError("candidate ids must be non-negative")
        return ids, offsets, None, (int(ids.max()) + 1 if ids.size else 0)
    if hasattr(voter_rankings, "ids") and hasattr(voter_rankings, "offsets"):
        ids = np.asarray(voter_rankings.ids)
        offsets = np.asarray(voter_rankings.offsets, dtype=np.int64)
        if ids.size and int(ids.min()) < 0:
            raise ValueError("candidate ids must be non-negative")
        return ids, offsets, None, (int(ids.max()) + 1 if ids.size else 0)
    rankings = [np.asarray(r) for r in voter_rankings]
    hi = 0
    for r in rankings:
        if r.size == 0:
            # The reference calls np.max on every ballot (scaling_elections.py:64-65).
            raise ValueError("zero-size array to reduction operation maximum which has no identity")
        if int(r.min()) < 0:
            raise ValueError("candidate ids must be non-negative")
        hi = max(hi, int(r.max()) + 1)
    return None, None, rankings, hi


def write_ballots(path: str | os.PathLike, voter_rankings, num_candidates: int | None = None, *,
                  id_bytes: int | None = None) -> Header:
    """Write ballots (a 2-D array of complete rankings, a sequence of 1-D rankings, or an
    ``api.Ballots``) to ``path``. C defaults to max id + 1 (the reference's rule,
    scaling_elections.py:63-66); id_bytes defaults to the narrowest width for C."""
    ids, offsets, rankings, hi = _as_csr(voter_rankings)
    C = int(num_candidates) if num_candidates is not None else max(hi, 1)
    if C < max(hi, 1):
        raise ValueError(f"a ballot names candidate {hi - 1}, outside [0, {C})")
    width = int(id_bytes) if id_bytes is not None else id_width(C)
    if width not in _ID_DTYPES or width < id_width(C):
        raise ValueError(f"id width {width} cannot hold {C} candidates")
    if rankings is not None:
        lens = np.fromiter((r.size for r in rankings), dtype=np.int64, count=len(rankings))
        offsets = np.zeros(len(rankings) + 1, dtype=np.int64)
        np.cumsum(lens, out=offsets[1:])
    V = len(offsets) - 1
    n_ids = int(offsets[-1]) if V > 0 else 0
    lens = np.diff(offsets)
    if V > 0 and (lens == 0).any():
        raise ValueError("zero-size array to reduction operation maximum which has no identity")
    complete = V > 0 and bool((lens == C).all())
    ids_off = _align(HEADER.size)
    offs_off = 0 if complete else _align(ids_off + n_ids * width)
    dtype = _ID_DTYPES[width]
    with open(path, "wb") as f:
        f.write(HEADER.pack(MAGIC, VERSION, width, V, C, FLAG_COMPLETE if complete else 0, n_ids, ids_off,
                            offs_off, 0))
        f.write(b"\0" * (ids_off - HEADER.size))
        if rankings is None:
            f.write(np.ascontiguousarray(ids, dtype=dtype).tobytes())
        else:
            step = 1 << 16  # ballots per write
            for v0 in range(0, V, step):
                f.write(np.concatenate(rankings[v0:v0 + step]).astype(dtype, copy=False).tobytes())
        if not complete:
            f.write(b"\0" * (offs_off - (ids_off + n_ids * width)))
            f.write(np.ascontiguousarray(offsets, dtype=np.int64).tobytes())
    return Header(width, V, C, FLAG_COMPLETE if complete else 0, n_ids, ids_off, offs_off)


def read_header(path: str | os.PathLike) -> Header:
    size = os.path.getsize(path)
    with open(path, "rb") as f:
        raw = f.read(HEADER.size)
    if len(raw) < HEADER.size:
        raise ValueError("not a ballot file: too short")
    magic, version, width, V, C, flags, n_ids, ids_off, offs_off, _ = HEADER.unpack(raw)
    if magic != MAGIC:
        raise ValueError("not a ballot file: bad magic")
    if version != VERSION:
        raise ValueError(f"unsupported ballot file version {version}")
    if width not in _ID_DTYPES or C < 1 or width < id_width(C):
        raise ValueError("corrupt ballot file header (id width or candidate count)")
    complete = bool(flags & FLAG_COMPLETE)
    if complete and (n_ids != V * C or offs_off != 0):
        raise ValueError("corrupt ballot file header (complete ballots)")
    if ids_off % _ALIGN or ids_off < HEADER.size or ids_off + n_ids * width > size:
        raise ValueError("truncated or corrupt ballot file (ids)")
    if not complete and (offs_off % _ALIGN or offs_off < ids_off + n_ids * width or offs_off + (V + 1) * 8 > size):
        raise ValueError("truncated or corrupt ballot file (offsets)")
    return Header(width, V, C, flags, n_ids, ids_off, offs_off)


class BallotFile:
    """A ballot file, memory-mapped read-only."""

    def __init__(self, path: str | os.PathLike):
        self.path = os.fspath(path)
        self.header = h = read_header(self.path)
        dtype = _ID_DTYPES[h.id_bytes]
        self.ids = (np.memmap(self.path, dtype=dtype, mode="r", offset=h.ids_offset, shape=(h.num_ids,))
                    if h.num_ids else np.zeros(0, dtype=dtype))
        if h.complete:
            self.offsets = None
        else:
            self.offsets = np.memmap(self.path, dtype=np.int64, mode="r", offset=h.offsets_offset,
                                     shape=(h.num_voters + 1,))
            if h.num_voters and (self.offsets[0] != 0 or self.offsets[-1] != h.num_ids):
                raise ValueError("corrupt ballot file: offsets do not span the ids")

    @property
    def num_voters(self) -> int:
        return self.header.num_voters

    @property
    def num_candidates(self) -> int:
        return self.header.num_candidates

    def __len__(self) -> int:
        return self.num_voters

    def span(self, v0: int, v1: int) -> tuple[int, int]:
        """Id range [a, b) of ballots [v0, v1)."""
        if self.offsets is None:
            C = self.num_candidates
            return v0 * C, v1 * C
        return int(self.offsets[v0]), int(self.offsets[v1])

    def ballot(self, v: int) -> np.ndarray:
        a, b = self.span(v, v + 1)
        return np.asarray(self.ids[a:b], dtype=np.int64)

    def csr(self, v0: int = 0, v1: int | None = None) -> tuple[np.ndarray, np.ndarray]:
        """Ballots [v0, v1) as (int32 ids, int64 offsets starting at 0)."""
        v1 = self.num_voters if v1 is None else v1
        a, b = self.span(v0, v1)
        ids = np.asarray(self.ids[a:b], dtype=np.int32)
        if self.offsets is None:
            offs = np.arange(v1 - v0 + 1, dtype=np.int64) * self.num_candidates
        else:
            offs = np.asarray(self.offsets[v0:v1 + 1], dtype=np.int64) - a
        return ids, offs

    def chunks(self, max_ballots: int) -> Iterator[tuple[int, int]]:
        """Consecutive ballot ranges [v0, v1) of at most max_ballots ballots."""
        step = max(1, int(max_ballots))
        for v0 in range(0, self.num_voters, step):
            yield v0, min(v0 + step, self.num_voters)


def _pread_pieces(fd: int, dst: np.ndarray, file_offset: int, pool: ThreadPoolExecutor, threads: int) -> list:
    """Queues parallel pread calls that fill the byte view dst from the file at file_offset,
    about two pieces per thread (at least 1 MiB each); returns their futures."""
    buf = dst.view(np.uint8).reshape(-1)
    n = buf.size
    mv = memoryview(buf)
    piece = max(1 << 20, -(-n // (2 * threads)))

    def read(a: int) -> None:
        b = min(a + piece, n)
        got = 0
        while a + got < b:
            r = os.preadv(fd, [mv[a + got:b]], file_offset + a + got)
            if r <= 0:
                raise ValueError("truncated ballot file")
            got += r

    return [pool.submit(read, a) for a in range(0, n, piece)]


def default_chunk_ballots(num_candidates: int, positions_bytes: int = 1 << 30) -> int:
    """Ballots per chunk so that the places buffer (ballots x roundup(C, 128) x 4 bytes) stays
    near positions_bytes."""
    Cq = (int(num_candidates) + 127) // 128 * 128
    return int(max(32, min(1 << 23, positions_bytes // (Cq * 4))))


def tally_file(path: str | os.PathLike, *, device=None, chunk_ballots: int | None = None,
               out: torch.Tensor | None = None, threads: int | None = None,
               stats: dict | None = None) -> torch.Tensor:
    """Pairwise preference counts (uint32 [C, C] on ``device``) of every ballot in the file,
    streamed through the GPU in chunks of ``chunk_ballots``. Equals ``build_pairwise_preferences``
    of the same ballots, including ballots that repeat an id (counted pair by pair, as the
    reference does). Raises ValueError for an id outside [0, C)."""
    bf = BallotFile(path)
    h = bf.header
    threads = int(threads) if threads else min(32, os.cpu_count() or 1)
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    V, C = h.num_voters, h.num_candidates
    if out is None:
        out = torch.zeros((C, C), dtype=torch.uint32, device=dev)
    else:
        if out.shape != (C, C) or out.dtype != torch.uint32 or out.device != dev or out.stride(1) != 1:
            raise ValueError("out must be a uint32 [C, C] tensor with contiguous rows on the device")
        out.view(torch.int32).zero_()
    if V == 0:
        return out
    nv = int(chunk_ballots) if chunk_ballots else default_chunk_ballots(C)
    nv = max(1, min(nv, V))
    width = h.id_bytes
    # The largest id span of any chunk sizes the id buffers.
    if bf.offsets is None:
        max_ids = nv * C
    else:
        starts = np.asarray(bf.offsets[::nv], dtype=np.int64)
        ends = np.asarray(bf.offsets[np.minimum(np.arange(nv, V + nv, nv), V)], dtype=np.int64)
        max_ids = int((ends - starts[:len(ends)]).max())
    id_dtype = {1: torch.uint8, 2: torch.int16, 4: torch.int32}[width]
    np_dtype = {1: np.uint8, 2: np.int16, 4: np.int32}[width]
    L = _lib.lib()
    need = L.se_tally_workspace_bytes(nv, C)
    if need < 0:
        raise ValueError("invalid chunk size")
    work = torch.empty(need, dtype=torch.uint8, device=dev)
    ragged = bf.offsets is not None
    # Three pinned host buffers: the reads of chunk n + 1 are queued before the wait for chunk n,
    # so the reader threads run on across chunk boundaries while a third buffer still feeds the
    # copy of chunk n - 1. Two device buffers: the copy of chunk n waits for the tally of n - 2.
    nh = 3
    host_ids = [torch.empty(max(max_ids, 1), dtype=id_dtype, pin_memory=True) for _ in range(nh)]
    dev_ids = [torch.empty(max(max_ids, 1), dtype=id_dtype, device=dev) for _ in range(2)]
    # The whole offsets array goes to the device once (8 bytes per ballot); each chunk's tally
    # reads its slice there with id_base = the chunk's first id. Per-chunk host copies of it
    # would run in this thread between the readers' calls, each one waiting for the GIL.
    all_offs = torch.from_numpy(np.array(bf.offsets, dtype=np.int64)).to(dev) if ragged else None  # a writable copy
    chunks = list(bf.chunks(nv))
    with torch.cuda.device(dev):
        compute = torch.cuda.current_stream(dev)
        copy = torch.cuda.Stream(dev)
        copied = [torch.cuda.Event() for _ in range(nh)]
        consumed = [torch.cuda.Event() for _ in range(2)]
        host_used = [False] * nh
        dev_used = [False, False]
        fd = os.open(bf.path, os.O_RDONLY)
        wait_s = 0.0
        pending: dict[int, list] = {}
        try:
            with ThreadPoolExecutor(max_workers=max(1, threads)) as pool:

                def queue_read(n: int) -> None:
                    hb = n % nh
                    if host_used[hb]:
                        copied[hb].synchronize()  # the copy out of this pinned buffer has finished
                    v0, v1 = chunks[n]
                    a, z = bf.span(v0, v1)
                    pending[n] = _pread_pieces(fd, host_ids[hb][:z - a].numpy().view(np_dtype),
                                               h.ids_offset + a * width, pool, threads)

                queue_read(0)
                for n, (v0, v1) in enumerate(chunks):
                    if n + 1 < len(chunks):
                        queue_read(n + 1)
                    hb, db = n % nh, n & 1
                    a, z = bf.span(v0, v1)
                    t0 = time.perf_counter()
                    for f in pending.pop(n):
                        f.result()
                    wait_s += time.perf_counter() - t0
                    with torch.cuda.stream(copy):
                        if dev_used[db]:
                            copy.wait_event(consumed[db])  # the tally of two chunks ago is done with it
                        dev_ids[db][:z - a].copy_(host_ids[hb][:z - a], non_blocking=True)
                        copied[hb].record(copy)
                    host_used[hb] = True
                    compute.wait_event(copied[hb])
                    flags = SE_TALLY_ACCUMULATE | SE_TALLY_NO_SYNC | (SE_TALLY_KEEP_ERROR if n else 0)
                    offs_ptr = all_offs.data_ptr() + 8 * v0 if ragged else None
                    check(L.se_tally_ex(dev_ids[db].data_ptr(), width, offs_ptr, a, v1 - v0, C, flags, out.data_ptr(),
                                        out.stride(0), work.data_ptr(), need, compute.cuda_stream))
                    consumed[db].record(compute)
                    dev_used[db] = True
        finally:
            for fs in pending.values():  # an error left reads queued: let them finish before closing
                for f in fs:
                    f.exception()
            os.close(fd)
        code = int(work[:4].view(torch.int32).cpu().item())  # synchronises the compute stream
    if stats is not None:
        stats.update(chunks=-(-V // nv), chunk_ballots=nv, read_wait_s=wait_s, file_bytes=os.path.getsize(bf.path),
                     read_threads=threads)
    if code == 2:
        raise ValueError(f"a ballot names a candidate outside [0, {C})")
    if code:
        raise SchulzeError(_lib.SE_ERR_DEVICE, f"tally kernel reported device error {code}")
    return out
