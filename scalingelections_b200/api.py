"""Host-side API: the reference's entry points for the Schulze GPU path, over libse.

Mirrors, name for name, what ``scaling_elections.py`` imports from the native module and the
Python functions on its hot path:

=============================  ============================================================
``compute_strongest_paths``    scaling_elections.cu:863-989 (bound at :1034-1038)
``log_gpus``                   scaling_elections.cu:996-1016
``build_pairwise_preferences`` scaling_elections.py:51-88
``get_winner_and_ranking``     scaling_elections.py:274-296
=============================  ============================================================

plus device-resident forms (``*_device``) that take and return CUDA tensors, for callers that
keep matrices in HBM between steps. Every compute path runs the sm_100a kernels; there is no
CPU fallback (``allow_gpu=False`` raises).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Sequence

import numpy as np
import torch

from . import _lib
from ._lib import LANES_AUTO, LANES_U16, LANES_U32, SchulzeError, check

# Tile sizes the reference's GPU driver accepts (scaling_elections.cu:895-901). The value
# only selects the reference's kernel template; the result does not depend on it, and this
# implementation always runs its own 128-cell tiles.
REFERENCE_GPU_TILES = (4, 8, 16, 32)


def _require_cuda() -> None:
    if not torch.cuda.is_available():
        raise RuntimeError("No CUDA devices available")


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _workspace(nbytes: int, device) -> torch.Tensor:
    # The caching allocator returns 512-byte aligned blocks and recycles them across calls.
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)


# Pageable host matrices reach the device through two pinned chunks: while one chunk's copy
# to the device runs, host threads fill the other (NumPy releases the GIL for large copies).
_STAGE_CHUNK = 64 << 20
_STAGE_THREADS = 8
_stage_state: dict = {}


def _stage_to_device(a: np.ndarray, dev) -> torch.Tensor:
    """A C-contiguous host array to a new CUDA uint8 tensor of its bytes, through pinned staging."""
    from concurrent.futures import ThreadPoolExecutor

    src = a.reshape(-1).view(np.uint8)
    n = src.size
    out = torch.empty(n, dtype=torch.uint8, device=dev)
    st = _stage_state.get(dev)
    if st is None:
        st = {"bufs": [torch.empty(_STAGE_CHUNK, dtype=torch.uint8, pin_memory=True) for _ in range(2)],
              "events": [torch.cuda.Event() for _ in range(2)], "used": [False, False],
              "pool": ThreadPoolExecutor(max_workers=_STAGE_THREADS)}
        _stage_state[dev] = st
    part = -(-_STAGE_CHUNK // _STAGE_THREADS)

    def fill(dst: np.ndarray, lo: int, hi: int) -> None:
        futures = [st["pool"].submit(np.copyto, dst[x - lo:min(x + part, hi) - lo], src[x:min(x + part, hi)])
                   for x in range(lo, hi, part)]
        for f in futures:
            f.result()

    stream = torch.cuda.current_stream(dev)
    for i, lo in enumerate(range(0, n, _STAGE_CHUNK)):
        hi = min(lo + _STAGE_CHUNK, n)
        b = i & 1
        if st["used"][b]:
            st["events"][b].synchronize()  # this buffer's previous copy has left
        buf = st["bufs"][b]
        fill(buf.numpy(), lo, hi)
        out[lo:hi].copy_(buf[:hi - lo], non_blocking=True)
        st["events"][b].record(stream)
        st["used"][b] = True
    return out


def _to_device_u32(a: np.ndarray | torch.Tensor, dev) -> torch.Tensor:
    """Host uint32 array -> CUDA uint32 tensor, copied through an int32 view (torch's uint32
    is a storage-only dtype). Large pageable NumPy arrays go through pinned staging."""
    if (isinstance(a, np.ndarray) and a.dtype.itemsize == 4 and a.nbytes >= 2 * _STAGE_CHUNK
            and torch.cuda.is_available()):
        a = np.ascontiguousarray(a)
        dev = torch.device(dev) if not isinstance(dev, int) else torch.device("cuda", dev)
        with torch.cuda.device(dev):
            return _stage_to_device(a, dev).view(torch.int32).view(a.shape).view(torch.uint32)
    t = a if isinstance(a, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(a))
    t = t.view(torch.int32)
    return t.to(device=dev, non_blocking=t.is_pinned()).view(torch.uint32)


def _to_host_u32(t: torch.Tensor, pinned: bool = False) -> np.ndarray:
    if pinned:
        host = torch.empty(t.shape, dtype=torch.int32, pin_memory=True)
        host.copy_(t.view(torch.int32), non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return host.numpy().view(np.uint32)
    return t.view(torch.int32).cpu().numpy().view(np.uint32)


def _check_matrix(t: torch.Tensor, name: str) -> tuple[int, int]:
    if t.dim() != 2 or t.shape[0] != t.shape[1]:
        raise ValueError(f"{name} must be a square matrix")
    if t.dtype != torch.uint32:
        raise TypeError(f"{name} must be uint32")
    if not t.is_cuda:
        raise ValueError(f"{name} must be on a CUDA device")
    if t.shape[0] > 0 and t.stride(1) != 1:
        raise ValueError(f"{name} rows must be contiguous")
    return t.shape[0], (t.stride(0) if t.shape[0] > 0 else 1)


# ------------------------------------------------------------------------------------------
# Device-resident entry points
# ------------------------------------------------------------------------------------------
def closure_workspace_bytes(num_candidates: int, lanes: int = LANES_AUTO, dataflow: bool = False) -> int:
    """Workspace bytes of the closure. dataflow=True sizes it for every schedule at its fastest:
    the dataflow form (mode 2), the second AT buffer of modes 5, 6 and 8, and the split panel
    tiles of modes 1, 3, 4, 6, 7 and 8 up to C = 3584: a few MiB more than the
    plain workspace. With the plain one those modes run their tiles whole, the automatic
    schedule runs 1 where it would pick 5, 6 or 8, and modes 2, 5, 6 and 8 set explicitly fail."""
    L = _lib.lib()
    fn = L.se_closure_workspace_bytes_flow if dataflow else L.se_closure_workspace_bytes
    n = fn(int(num_candidates), int(lanes), 0)
    if n < 0:
        raise ValueError("invalid closure size")
    return n


_closure_mode = 0


def set_closure_mode(mode: int) -> None:
    """The closure's schedule (same results in every one): 0 automatic by size (default),
    1 round by round, 2 the dataflow form, 3 round by round with the panels on the wide
    micro-tile, 4 as 3 with each pivot tile closed by its own wide launch, 5 as 3 on two
    streams so the next round's chain overlaps the current remainder, 6 each round's
    remainder and the next round's panels in one launch, 7 as 3 with every tile on the wide
    micro-tile, 8 as 6 on the wide micro-tile (include/se.h)."""
    global _closure_mode
    check(_lib.lib().se_closure_set_mode(int(mode)))
    _closure_mode = int(mode)


BUILTIN_CLOSURE_VARIANTS = ((1024, 7), (4096, 8), (1 << 20, 6))


def closure_schedule(num_candidates: int, lanes: int = LANES_U16, workspace_bytes: int | None = None) -> int:
    """The schedule (1 to 8) a closure of this size would run now (host-only query). The
    workspace defaults to what strongest_paths_device allocates; -1 for no candidates."""
    if int(num_candidates) < 1:
        return -1
    if workspace_bytes is None:
        workspace_bytes = closure_workspace_bytes(num_candidates, lanes, dataflow=True)
    return int(_lib.lib().se_closure_schedule(int(num_candidates), int(lanes), int(workspace_bytes)))


def set_closure_variants(table: Sequence[tuple[int, int]]) -> None:
    """The automatic schedule's table: (max_C, mode) pairs, first match wins, modes 1 or 3-8;
    sizes above every entry run mode 1. An empty table clears it (every size then runs mode 1;
    the library starts with the table measured on B200, {1024: 7, 4096: 8, 2**20: 6}).
    autotune.tune_closure measures the modes per size bucket and installs its winners through
    this."""
    n = len(table)
    max_c = (ctypes.c_int * max(n, 1))(*[int(c) for c, _ in table])
    modes = (ctypes.c_int * max(n, 1))(*[int(m) for _, m in table])
    check(_lib.lib().se_closure_set_variant_table(max_c, modes, n))


def strongest_paths_device(preferences: torch.Tensor, *, lanes: int = LANES_AUTO, out: torch.Tensor | None = None,
                           workspace: torch.Tensor | None = None) -> torch.Tensor:
    """Widest-path closure of a CUDA uint32 [C, C] preference matrix; returns uint32 [C, C]
    on the same device (diagonal 0), bit-identical to compute_strongest_paths_numba_serial.

    lanes: LANES_U16 (every count < 65536), LANES_U32, or LANES_AUTO (checked on the device,
    one 4-byte read back). workspace: used as given when it holds closure_workspace_bytes(C,
    lanes) bytes (below the dataflow=True size the automatic schedule runs what fits, as
    closure_schedule reports, and modes 2, 5, 6 and 8 set explicitly fail); else a full one is
    allocated (and cached)."""
    C, ld = _check_matrix(preferences, "preferences")
    if out is None:
        out = torch.empty((C, C), dtype=torch.uint32, device=preferences.device)
    Co, ldo = _check_matrix(out, "out")
    if Co != C:
        raise ValueError("out has the wrong shape")
    if C == 0:
        return out
    # A workspace the caller passes is used as it is when it holds the plain size (the library
    # then runs the schedules that fit it); otherwise the full one, with which every schedule
    # runs at its fastest (the second AT buffer of modes 2, 5, 6 and 8 and the split panel
    # tiles of small closures: a few MiB more).
    need = closure_workspace_bytes(C, lanes, dataflow=False)
    if workspace is None or workspace.numel() * workspace.element_size() < need:
        workspace = _workspace(closure_workspace_bytes(C, lanes, dataflow=True), preferences.device)
    have = workspace.numel() * workspace.element_size()
    with torch.cuda.device(preferences.device):
        check(_lib.lib().se_closure(preferences.data_ptr(), ld, C, out.data_ptr(), ldo, int(lanes), 0,
                                    workspace.data_ptr(), have, _stream()))
    return out


def strongest_paths_enqueue(preferences: torch.Tensor, *, lanes: int, value_offset: int = 0,
                            out: torch.Tensor | None = None, workspace: torch.Tensor | None = None) -> torch.Tensor:
    """The closure of strongest_paths_device queued on the current stream without waiting
    (se_closure_enqueue): returns ``out`` as soon as the work is queued. lanes is LANES_U16 or
    LANES_U32 (LANES_AUTO would read the matrix back). The call's error word stays in
    ``workspace``, which must not serve another closure before closure_check(workspace) has
    read it; pass one (of closure_workspace_bytes(C, lanes, dataflow=True) bytes for every
    schedule at its fastest) to check it later."""
    if lanes not in (LANES_U16, LANES_U32):
        raise ValueError("lanes must be LANES_U16 or LANES_U32")
    C, ld = _check_matrix(preferences, "preferences")
    if out is None:
        out = torch.empty((C, C), dtype=torch.uint32, device=preferences.device)
    Co, ldo = _check_matrix(out, "out")
    if Co != C:
        raise ValueError("out has the wrong shape")
    if C == 0:
        return out
    if workspace is None:
        raise ValueError("pass the workspace: closure_check reads the call's error word from it")
    have = workspace.numel() * workspace.element_size()
    with torch.cuda.device(preferences.device):
        check(_lib.lib().se_closure_enqueue(preferences.data_ptr(), ld, C, out.data_ptr(), ldo, int(lanes),
                                            int(value_offset), workspace.data_ptr(), have, _stream()))
    return out


def closure_check(workspace: torch.Tensor) -> None:
    """Waits for the current stream and raises if the closure queued with this workspace
    reported a device error or a value outside its 16-bit window (se_closure_check)."""
    with torch.cuda.device(workspace.device):
        check(_lib.lib().se_closure_check(workspace.data_ptr(), _stream()))


def tally_workspace_bytes(num_voters: int, num_candidates: int) -> int:
    n = _lib.lib().se_tally_workspace_bytes(int(num_voters), int(num_candidates))
    if n < 0:
        raise ValueError("invalid tally size")
    return n


def tally_device(ids: torch.Tensor, offsets: torch.Tensor, num_candidates: int, *, out: torch.Tensor | None = None,
                 workspace: torch.Tensor | None = None) -> torch.Tensor:
    """Pairwise preference counts from CSR ballots on the device: ids int32 (concatenated
    ballots, most preferred first), offsets int64 [V + 1]. Returns uint32 [C, C]."""
    if ids.dtype != torch.int32 or offsets.dtype != torch.int64 or not ids.is_cuda or not offsets.is_cuda:
        raise TypeError("ids must be CUDA int32 and offsets CUDA int64")
    C = int(num_candidates)
    V = offsets.numel() - 1
    if V < 0:
        raise ValueError("offsets must hold V + 1 entries")
    if V > 0:
        # The kernels trust the CSR bounds; check them here (one small device-to-host read).
        bad = (offsets[0] != 0) | (offsets[-1] != ids.numel()) | (offsets[1:] < offsets[:-1]).any()
        if bool(bad):
            raise ValueError("offsets must start at 0, never decrease and end at len(ids)")
    if out is None:
        out = torch.empty((C, C), dtype=torch.uint32, device=ids.device)
    Co, ldo = _check_matrix(out, "out")
    need = tally_workspace_bytes(V, C)
    if workspace is None or workspace.numel() * workspace.element_size() < need:
        workspace = _workspace(need, ids.device)
    with torch.cuda.device(ids.device):
        check(_lib.lib().se_tally(ids.data_ptr(), offsets.data_ptr(), V, C, out.data_ptr(), ldo,
                                  workspace.data_ptr(), need, _stream()))
    return out


def rank_device(strongest_paths: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
    """(wins, ranking) int32 CUDA tensors: wins[i] = #{j: S[i][j] > S[j][i]}; ranking lists
    candidates by wins descending, ties by ascending index."""
    C, ld = _check_matrix(strongest_paths, "strongest_paths")
    wins = torch.empty(C, dtype=torch.int32, device=strongest_paths.device)
    ranking = torch.empty(C, dtype=torch.int32, device=strongest_paths.device)
    if C:
        with torch.cuda.device(strongest_paths.device):
            check(_lib.lib().se_rank(strongest_paths.data_ptr(), ld, C, wins.data_ptr(), ranking.data_ptr(),
                                     _stream()))
    return wins, ranking


# ------------------------------------------------------------------------------------------
# Reference-compatible host entry points
# ------------------------------------------------------------------------------------------
def _host_u32_matrix(preferences) -> np.ndarray | torch.Tensor:
    if isinstance(preferences, torch.Tensor):
        t = preferences.detach()
        if t.dim() != 2:
            raise RuntimeError("Number of dimensions must be two")
        if t.shape[0] != t.shape[1]:
            raise RuntimeError("Preferences matrix must be square")
        if t.dtype != torch.uint32:
            t = torch.from_numpy(t.cpu().numpy().astype(np.uint32))
        return t.contiguous()
    a = np.asarray(preferences)
    if a.ndim != 2:
        raise RuntimeError("Number of dimensions must be two")
    if a.shape[0] != a.shape[1]:
        raise RuntimeError("Preferences matrix must be square")
    # pybind11's array_t<uint32, c_style> force-casts any dtype and layout (cu:864).
    return np.ascontiguousarray(a.astype(np.uint32, copy=False))


def compute_strongest_paths(preferences, *, allow_tma: bool = False, allow_gpu: bool = False,
                            tile_size: int = 0, lanes: int = LANES_AUTO) -> np.ndarray:
    """Drop-in for the reference's native ``compute_strongest_paths``
    (scaling_elections.cu:863-989): preferences (C x C, any dtype, cast to uint32) in, a new
    C-contiguous uint32 strongest-path matrix out, diagonal 0.

    Error behaviour follows the reference: RuntimeError("Number of dimensions must be two"),
    RuntimeError("Preferences matrix must be square"), RuntimeError("Unsupported tile size")
    for a GPU tile outside {4, 8, 16, 32}. ``allow_tma`` is accepted and has no effect (every
    kernel here stages through TMA). ``allow_gpu=False`` selects the reference's OpenMP CPU
    path, which this GPU-only library does not provide: it raises RuntimeError.

    Unlike the reference's GPU path, any C works (no C % tile_size == 0 requirement)."""
    P = _host_u32_matrix(preferences)
    if not allow_gpu:
        raise RuntimeError("CPU path not provided: this module runs the closure on the GPU only "
                           "(pass allow_gpu=True)")
    if int(tile_size) not in REFERENCE_GPU_TILES:
        raise RuntimeError("Unsupported tile size")
    _require_cuda()
    C = P.shape[0]
    if C == 0:
        return np.zeros((0, 0), dtype=np.uint32)
    d = _to_device_u32(P, torch.cuda.current_device())
    out = strongest_paths_device(d, lanes=lanes)
    return _to_host_u32(out, pinned=True)


class ClosureStream:
    """Closures of a sequence of host preference matrices of one size, pipelined over copies.

    ``compute_strongest_paths`` copies a matrix in, closes it and copies the result out, one
    step after another. Here, while election k closes on the compute stream, election k + 1's
    matrix is copied in and election k - 1's result is copied out on two copy streams, so in
    steady state a step costs the closure alone (or the copies, when they are slower). Each
    closure runs through ``se_closure_enqueue`` and is checked with ``se_closure_check`` when
    its result is handed out. Two device slots (input, output, workspace) alternate.

    lanes: LANES_U16 (with ``value_offset``, a kept count v is held as v - value_offset, which
    must lie in [1, 65535]) or LANES_U32. A count outside the 16-bit window raises
    SchulzeError(SE_ERR_OVERFLOW) when that election's result is handed out.

    Results are new arrays in pinned host memory from torch's pinned-memory cache. Pinning a
    fresh block of C x C words takes a long time (a quarter second at C = 16384), so the
    constructor fills the cache with the three result blocks a steady stream keeps alive (two
    in flight, one with the caller); warm_results=0 skips that."""

    def __init__(self, num_candidates: int, *, lanes: int = LANES_U16, value_offset: int = 0, device=None,
                 warm_results: int = 3):
        _require_cuda()
        if lanes not in (LANES_U16, LANES_U32):
            raise ValueError("lanes must be LANES_U16 or LANES_U32")
        self.C = int(num_candidates)
        if self.C < 1:
            raise ValueError("Number of candidates must be positive")
        self.lanes, self.value_offset = int(lanes), int(value_offset)
        self.dev = torch.device("cuda", torch.cuda.current_device() if device is None else torch.device(device).index)
        C = self.C
        self.work_bytes = closure_workspace_bytes(C, self.lanes, dataflow=True)  # every schedule at its fastest
        with torch.cuda.device(self.dev):
            self.d_in = [torch.empty((C, C), dtype=torch.int32, device=self.dev) for _ in range(2)]
            self.d_out = [torch.empty((C, C), dtype=torch.int32, device=self.dev) for _ in range(2)]
            self.work = [_workspace(self.work_bytes, self.dev) for _ in range(2)]
            self.compute = torch.cuda.Stream(self.dev)
            self.h2d = torch.cuda.Stream(self.dev)
            self.d2h = torch.cuda.Stream(self.dev)
            self.checks = torch.cuda.Stream(self.dev)
            self.copied_in = [torch.cuda.Event() for _ in range(2)]
            self.closed = [torch.cuda.Event() for _ in range(2)]
            self.copied_out = [torch.cuda.Event() for _ in range(2)]
        blocks = [torch.empty((C, C), dtype=torch.int32, pin_memory=True) for _ in range(max(0, warm_results))]
        del blocks  # back to the cache, ready for map()

    def _host_in(self, m) -> torch.Tensor:
        t = m if isinstance(m, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(_host_u32_matrix(m)))
        if t.shape != (self.C, self.C):
            raise ValueError(f"every matrix must be {self.C} x {self.C}")
        if t.dtype == torch.uint32:
            t = t.view(torch.int32)
        elif t.dtype != torch.int32:
            t = torch.from_numpy(np.ascontiguousarray(t.cpu().numpy().astype(np.uint32)).view(np.int32))
        return t.contiguous()

    def map(self, matrices):
        """Yields the strongest-path matrix (uint32 [C, C], pinned host memory) of every input
        matrix, in order. Inputs in pinned memory are copied asynchronously; others through
        the driver's staging, which blocks this thread but not the GPU."""
        L = _lib.lib()
        pending = []  # (slot, host output) in flight
        k = 0
        with torch.cuda.device(self.dev):
            for m in matrices:
                b = k & 1
                src = self._host_in(m)
                with torch.cuda.stream(self.h2d):
                    if k >= 2:
                        self.h2d.wait_event(self.closed[b])  # election k - 2 no longer reads d_in[b]
                    self.d_in[b].copy_(src, non_blocking=True)
                    self.copied_in[b].record(self.h2d)
                self.compute.wait_event(self.copied_in[b])
                if k >= 2:
                    self.compute.wait_event(self.copied_out[b])  # d_out[b] and work[b] are free again
                check(L.se_closure_enqueue(self.d_in[b].data_ptr(), self.C, self.C, self.d_out[b].data_ptr(), self.C,
                                           self.lanes, self.value_offset, self.work[b].data_ptr(), self.work_bytes,
                                           self.compute.cuda_stream))
                self.closed[b].record(self.compute)
                host = torch.empty((self.C, self.C), dtype=torch.int32, pin_memory=True)
                with torch.cuda.stream(self.d2h):
                    self.d2h.wait_event(self.closed[b])
                    host.copy_(self.d_out[b], non_blocking=True)
                    self.copied_out[b].record(self.d2h)
                pending.append((b, host))
                k += 1
                if len(pending) == 2:
                    yield self._finish(*pending.pop(0))
            while pending:
                yield self._finish(*pending.pop(0))

    def _finish(self, b: int, host: torch.Tensor) -> np.ndarray:
        # The check runs on a stream of its own that waits for this slot's result copy only:
        # on the output stream it would also wait for the next election's copy, and so for
        # the closure running now.
        self.checks.wait_event(self.copied_out[b])
        check(_lib.lib().se_closure_check(self.work[b].data_ptr(), self.checks.cuda_stream))
        return host.numpy().view(np.uint32)


def log_gpus() -> None:
    """Prints every CUDA device as scaling_elections.cu:996-1016 does."""
    L = _lib.lib()
    n = ctypes.c_int(0)
    check(L.se_device_count(ctypes.byref(n)))
    for i in range(n.value):
        name = ctypes.create_string_buffer(256)
        sms, major, minor = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        mem = ctypes.c_double()
        check(L.se_device_info(i, name, 256, ctypes.byref(sms), ctypes.byref(mem), ctypes.byref(major),
                               ctypes.byref(minor)))
        print(f"Device {i}: {name.value.decode()}")
        print(f"\tSMs: {sms.value}")
        print(f"\tGlobal mem: {mem.value:.2f}GB")
        print(f"\tCUDA Cap: {major.value}.{minor.value}")


@dataclass
class Ballots:
    """Ballots in CSR form: ballot v is ids[offsets[v]:offsets[v+1]], most preferred first."""
    ids: np.ndarray      # int32
    offsets: np.ndarray  # int64, V + 1 entries
    num_candidates: int  # max id + 1 (at least 1), as scaling_elections.py:63-66

    @property
    def num_voters(self) -> int:
        return len(self.offsets) - 1

    @classmethod
    def from_rankings(cls, voter_rankings: Sequence[np.ndarray] | np.ndarray) -> "Ballots":
        if isinstance(voter_rankings, np.ndarray) and voter_rankings.ndim == 2:
            V, L = voter_rankings.shape
            if L == 0 and V > 0:
                raise ValueError("zero-size array to reduction operation maximum which has no identity")
            ids = np.ascontiguousarray(voter_rankings, dtype=np.int32).reshape(-1)
            offsets = np.arange(V + 1, dtype=np.int64) * L
        else:
            rankings = [np.asarray(r) for r in voter_rankings]
            lens = np.fromiter((r.size for r in rankings), dtype=np.int64, count=len(rankings))
            if (lens == 0).any():
                # The reference calls np.max on every ballot (py:64-65).
                raise ValueError("zero-size array to reduction operation maximum which has no identity")
            offsets = np.zeros(len(rankings) + 1, dtype=np.int64)
            np.cumsum(lens, out=offsets[1:])
            ids = (np.concatenate(rankings).astype(np.int32, copy=False) if rankings
                   else np.zeros(0, dtype=np.int32))
        if ids.size and int(ids.min()) < 0:
            raise ValueError("candidate ids must be non-negative")
        C = max(1, int(ids.max()) + 1) if ids.size else 1
        return cls(np.ascontiguousarray(ids), offsets, C)


def _tally_host(ballots: Ballots, dev) -> torch.Tensor:
    ids = torch.from_numpy(ballots.ids).to(dev, non_blocking=False)
    offs = torch.from_numpy(ballots.offsets).to(dev, non_blocking=False)
    try:
        return tally_device(ids, offs, ballots.num_candidates)
    except SchulzeError as e:
        if e.status == _lib.SE_ERR_DEVICE and "candidate" in str(e):
            raise ValueError(str(e)) from e
        raise


def build_pairwise_preferences(voter_rankings: Sequence[np.ndarray] | np.ndarray) -> np.ndarray:
    """GPU form of scaling_elections.py:51-88: uint32 [C, C] with d[i][j] = number of voters
    ranking i above j, C = max id + 1. A ballot whose length differs from C gets the ids it
    lacks appended in ascending order (py:75-83). A ballot that repeats an id is counted pair
    by pair like the reference's (py:46-48): d[x][y] gains one for every position of x before
    a position of y, so the diagonal and counts above V can be non-zero."""
    _require_cuda()
    b = Ballots.from_rankings(voter_rankings)
    d = _tally_host(b, torch.cuda.current_device())
    return _to_host_u32(d)


def get_winner_and_ranking(candidates: list, strongest_paths) -> tuple:
    """GPU form of scaling_elections.py:274-296: (winner, ranked candidates), ranking by the
    number of pairwise wins, descending, ties in candidate order."""
    _require_cuda()
    n = len(candidates)
    if n == 0:
        raise IndexError("list index out of range")
    S = strongest_paths[:n, :n]
    if isinstance(S, torch.Tensor):
        S = _to_device_u32(_host_u32_matrix(S.cpu()), torch.cuda.current_device())
    else:
        S = _to_device_u32(np.ascontiguousarray(np.asarray(S).astype(np.uint32, copy=False)),
                           torch.cuda.current_device())
    _, ranking = rank_device(S)
    order = ranking.cpu().numpy()
    ranked = [candidates[i] for i in order]
    return ranked[0], ranked


@dataclass
class SchulzeResult:
    winner: int
    ranking: np.ndarray            # int32 [C]
    wins: np.ndarray               # int32 [C]
    strongest_paths: np.ndarray | None


def schulze(voter_rankings: Sequence[np.ndarray] | np.ndarray, *, return_paths: bool = False) -> SchulzeResult:
    """Whole Schulze election on the GPU: tally -> closure -> ranking, matrices kept in HBM.
    The closure's lanes are chosen on the device from the kept counts: 16-bit (shifted if need
    be) whenever they fit a 16-bit window, else 32-bit."""
    _require_cuda()
    b = Ballots.from_rankings(voter_rankings)
    dev = torch.cuda.current_device()
    d = _tally_host(b, dev)
    # Permutation ballots keep every count within (V/2, V], a 16-bit window up to 131070
    # ballots; ballots that repeat an id can raise counts above V, which the measured window
    # also covers.
    S = strongest_paths_device(d, lanes=LANES_AUTO)
    wins, ranking = rank_device(S)
    ranking_h = ranking.cpu().numpy()
    return SchulzeResult(int(ranking_h[0]), ranking_h, wins.cpu().numpy(),
                         _to_host_u32(S) if return_paths else None)
