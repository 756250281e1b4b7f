"""Continuous-batching Schulze server on one GPU.

Requests are ballot sets (V ballots of C candidates, int32 [V, C]) in device memory or in host
memory; host ballots are copied into the server's HBM block when the request is admitted, on
the submission stream, and that copy counts against the budget until the tally is done.
The server admits a request when its working memory fits the HBM budget (an arena carved
from one preallocated block) and hands it to the serving engine (include/se.h, se_engine_*):
one persistent kernel that tallies, closes and ranks every admitted election, task by task,
and keeps running while requests join, so requests that arrive while others are on the GPU
are processed alongside them. Completion is observed through host-mapped memory; latency is
measured from a request's arrival to the poll that sees it finished.

No reference counterpart: the reference runs one election per call on the host's thread.
"""
from __future__ import annotations

import bisect
import ctypes
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import check
from .batch import lanes_for_voters

ALIGN = 256


class Arena:
    """First-fit allocator over [0, capacity) with coalescing frees; offsets are ALIGN-aligned.
    Pure host bookkeeping: it hands out offsets into one device block."""

    def __init__(self, capacity: int):
        self.capacity = int(capacity) // ALIGN * ALIGN
        self._starts = [0]               # free extents, sorted by start
        self._sizes = {0: self.capacity}
        self.used = 0

    def alloc(self, nbytes: int) -> int | None:
        n = (int(nbytes) + ALIGN - 1) // ALIGN * ALIGN
        for idx, start in enumerate(self._starts):
            size = self._sizes[start]
            if size >= n:
                del self._sizes[start]
                self._starts.pop(idx)
                if size > n:
                    self._starts.insert(idx, start + n)
                    self._sizes[start + n] = size - n
                self.used += n
                return start
        return None

    def free(self, offset: int, nbytes: int) -> None:
        n = (int(nbytes) + ALIGN - 1) // ALIGN * ALIGN
        self.used -= n
        idx = bisect.bisect_left(self._starts, offset)
        start, size = offset, n
        # merge with the following extent
        if idx < len(self._starts) and self._starts[idx] == start + size:
            nxt = self._starts.pop(idx)
            size += self._sizes.pop(nxt)
        # merge with the preceding extent
        if idx > 0:
            prev = self._starts[idx - 1]
            if prev + self._sizes[prev] == start:
                self._sizes[prev] += size
                return
        self._starts.insert(idx, start)
        self._sizes[start] = size

    @property
    def free_bytes(self) -> int:
        return self.capacity - self.used


def request_bytes(V: int, C: int) -> dict:
    """Device bytes of one request's buffers, each ALIGN-aligned. "positions" (the ballot
    places, usually the largest part) is a separate block, released when the tally is done."""

    def al(x):
        return (int(x) + ALIGN - 1) // ALIGN * ALIGN

    L = _lib.lib()
    scratch = L.se_engine_request_scratch_bytes(int(V), int(C))
    positions = L.se_engine_request_positions_bytes(int(V), int(C))
    if scratch < 0 or positions < 0:
        raise ValueError("invalid request shape")
    parts = {
        "prefs": al(4 * C * C),
        "out": al(4 * C * C),
        "wins": al(4 * C),
        "ranking": al(4 * C),
        "scratch": al(scratch),
    }
    parts["main"] = sum(parts.values())
    parts["positions"] = al(positions)
    parts["total"] = parts["main"] + parts["positions"]
    return parts


@dataclass
class Ticket:
    rid: int
    V: int
    C: int
    arrival: float
    offset: int = -1
    nbytes: int = 0
    pos_offset: int = -1
    pos_nbytes: int = 0
    ids_offset: int = -1       # host ballots: their copy in the server's block, until tallied
    ids_nbytes: int = 0
    cancelled: bool = False
    slot: int = -1
    gen: int = 0
    admitted: float = 0.0
    finished: float = 0.0
    status: int = -1
    ranking: np.ndarray | None = None
    strongest_paths: np.ndarray | None = None
    keep_paths: bool = False
    views: dict = field(default_factory=dict)
    parts: dict | None = None  # request_bytes(V, C), computed once

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class Server:
    """budget_bytes: HBM admission budget for the requests' working memory (ballots are the
    caller's). ctas_per_sm: engine CTAs per SM. idle_ms: the engine kernel exits after this
    long without work and is relaunched by the next submit or poll.

    priority: the order in which requests that are waiting together are admitted. The engine
    gives lower slots first claim on work, so admission order is priority order. "arrival"
    admits the oldest first. "largest" admits the most work first (C^3 + V C^2), which shortens
    the tail of a burst, at the cost of the small requests in it. Requests that arrive alone
    are unaffected."""

    def __init__(self, budget_bytes: int = 40 << 30, max_slots: int = 1024, ctas_per_sm: int = 2,
                 idle_ms: int = 20, device: int | None = None, priority: str = "arrival"):
        if priority not in ("arrival", "largest"):
            raise ValueError("priority must be 'arrival' or 'largest'")
        self.priority = priority
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        L = _lib.lib()
        self.L = L
        with torch.cuda.device(self.device):
            self.block = torch.empty(int(budget_bytes), dtype=torch.uint8, device=self.device)
            self.arena = Arena(budget_bytes)
            nbytes = L.se_engine_workspace_bytes(max_slots)
            if nbytes < 0:
                raise ValueError("bad max_slots")
            self.engine_ws = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            self.engine = ctypes.c_void_p()
            check(L.se_engine_create(self.engine_ws.data_ptr(), nbytes, max_slots, ctas_per_sm, idle_ms,
                                     ctypes.byref(self.engine)))
            self.stream = torch.cuda.Stream(device=self.device)
        self.max_slots = max_slots
        self.by_slot: dict[int, Ticket] = {}
        self._poll_slots = (ctypes.c_int * max_slots)()
        self._poll_status = (ctypes.c_uint32 * max_slots)()
        self.base_ptr = self.block.data_ptr()

    # -- admission -------------------------------------------------------------------------
    def try_submit(self, ticket: Ticket, ballots: torch.Tensor | np.ndarray) -> bool:
        """Admit and publish one request if its memory fits and a slot is free; else False.
        ballots: int32 [V, C], one ballot per row listing each of the C candidates once, most
        preferred first; a CUDA tensor (used in place), or host memory (a tensor, pinned for an
        asynchronous copy, or a NumPy array), copied into the server's block on admission."""
        if len(self.by_slot) >= self.max_slots:
            return False
        V, C = ticket.V, ticket.C
        if isinstance(ballots, np.ndarray):
            ballots = torch.from_numpy(np.ascontiguousarray(ballots, dtype=np.int32))
        if ballots.shape != (V, C) or ballots.dtype != torch.int32:
            raise ValueError("ballots must be an int32 [V, C] tensor or array")
        on_host = not ballots.is_cuda
        lanes, offset = lanes_for_voters(V)
        if lanes != 16:
            raise ValueError("the server handles up to 131070 ballots per request")
        if ticket.parts is None:
            ticket.parts = request_bytes(V, C)
        parts = ticket.parts
        ids_bytes = (4 * V * C + ALIGN - 1) // ALIGN * ALIGN if on_host else 0
        if parts["total"] + ids_bytes > self.arena.free_bytes:
            return False
        blocks = []
        for n in (parts["main"], parts["positions"], ids_bytes):
            o = self.arena.alloc(n) if n else -1
            if o is None:
                for o2, n2 in blocks:
                    if o2 >= 0:
                        self.arena.free(o2, n2)
                return False
            blocks.append((o, n))
        (off, _), (pos_off, _), (ids_off, _) = blocks
        ticket.offset, ticket.nbytes = off, parts["main"]
        ticket.pos_offset, ticket.pos_nbytes = pos_off, parts["positions"]
        pos = off
        ptrs = {}
        for name in ("prefs", "out", "wins", "ranking", "scratch"):
            ptrs[name] = self.base_ptr + pos
            ticket.views[name] = (pos, parts[name])
            pos += parts[name]
        with torch.cuda.device(self.device):
            if on_host:
                # A plain copy (no dtype or layout change) is a copy-engine transfer, which runs
                # beside the resident engine; it precedes the request's descriptor on the stream.
                ticket.ids_offset, ticket.ids_nbytes = ids_off, ids_bytes
                dst = self.block[ids_off:ids_off + 4 * V * C].view(torch.int32).view(V, C)
                with torch.cuda.stream(self.stream):
                    dst.copy_(ballots.contiguous(), non_blocking=ballots.is_pinned())
                ids_ptr = dst.data_ptr()
            else:
                ids_ptr = ballots.data_ptr()
            rq = _lib.Request(ids_ptr, None, V, C, offset, ptrs["prefs"], ptrs["out"], ptrs["wins"],
                              ptrs["ranking"], ptrs["scratch"], parts["scratch"], self.base_ptr + pos_off,
                              parts["positions"])
            slot, gen = ctypes.c_int(), ctypes.c_uint32()
            check(self.L.se_engine_submit(self.engine, ctypes.byref(rq), self.stream.cuda_stream, ctypes.byref(slot),
                                          ctypes.byref(gen)))
        ticket.slot, ticket.gen = slot.value, gen.value
        ticket.admitted = time.perf_counter()
        self.by_slot[ticket.slot] = ticket
        ticket._ballots = ballots  # keep alive until done (a pinned source until its copy ends)
        return True

    def cancel(self, ticket: Ticket) -> bool:
        """Cancels a request. One still waiting for admission is dropped by the next admit()
        and never reaches the GPU. One already admitted keeps its tasks on the engine, which
        cannot stop a task midway; its memory returns to the arena when the engine finishes
        it, and poll() then drops it instead of returning it. Returns True if the request was
        waiting (nothing of it ran), False if it was in flight or already done."""
        if ticket.status >= 0:
            return False
        ticket.cancelled = True
        return ticket.slot < 0

    # -- completion ------------------------------------------------------------------------
    def admit(self, pending: list[Ticket], ballots_of, now: float, max_bypass_s: float = 0.25) -> int:
        """Admits pending requests in priority order (see the class docstring). A request that
        does not fit yet may be passed by others that do, unless the oldest has waited longer
        than max_bypass_s: then admission is strictly by arrival and nothing passes it (no
        starvation). Returns how many were admitted."""
        admitted = 0
        if any(t.cancelled for t in pending):
            pending[:] = [t for t in pending if not t.cancelled]
        strict = bool(pending) and now - pending[0].arrival > max_bypass_s
        order = list(range(len(pending)))
        if self.priority == "largest" and not strict:
            order.sort(key=lambda x: -(pending[x].C ** 3 + pending[x].V * pending[x].C ** 2))
        taken = set()
        smallest_failed = None
        for x in order:
            t = pending[x]
            if t.parts is None:
                t.parts = request_bytes(t.V, t.C)
            # A request at least as large as one that just failed cannot fit either.
            if smallest_failed is None or t.parts["total"] < smallest_failed:
                if self.try_submit(t, ballots_of(t)):
                    taken.add(x)
                    admitted += 1
                    continue
                smallest_failed = t.parts["total"] if smallest_failed is None else min(smallest_failed,
                                                                                       t.parts["total"])
            if strict or len(self.by_slot) >= self.max_slots or self.arena.free_bytes < (1 << 20):
                break
        if taken:
            pending[:] = [t for i, t in enumerate(pending) if i not in taken]
        return admitted

    def poll(self) -> list[Ticket]:
        n = ctypes.c_int(0)
        check(self.L.se_engine_poll_tallied(self.engine, self._poll_slots, self.max_slots, ctypes.byref(n)))
        for x in range(n.value):
            t = self.by_slot.get(self._poll_slots[x])
            if t is not None:
                self._release_ballots(t)
        check(self.L.se_engine_poll(self.engine, self._poll_slots, self._poll_status, self.max_slots, ctypes.byref(n)))
        now = time.perf_counter()
        done = []
        for x in range(n.value):
            t = self.by_slot.pop(self._poll_slots[x])
            t.finished = now
            t.status = int(self._poll_status[x])
            self._collect(t)
            if not t.cancelled:
                done.append(t)
        return done

    def _release_ballots(self, t: Ticket) -> None:
        """The ballot places and a host request's copied ballots, once its tally is done."""
        if t.pos_offset >= 0:
            self.arena.free(t.pos_offset, t.pos_nbytes)
            t.pos_offset = -1
        if t.ids_offset >= 0:
            self.arena.free(t.ids_offset, t.ids_nbytes)
            t.ids_offset = -1

    def _view(self, t: Ticket, name: str, shape, dtype) -> torch.Tensor:
        pos, _ = t.views[name]
        n = int(np.prod(shape)) * torch.empty(0, dtype=dtype).element_size()
        return self.block[pos:pos + n].view(dtype).view(*shape)

    def _collect(self, t: Ticket) -> None:
        if not t.cancelled:
            with torch.cuda.device(self.device):
                t.ranking = self._view(t, "ranking", (t.C,), torch.int32).cpu().numpy()
                if t.keep_paths:
                    S = self._view(t, "out", (t.C, t.C), torch.int32)
                    t.strongest_paths = S.cpu().numpy().view(np.uint32)
        self.arena.free(t.offset, t.nbytes)
        self._release_ballots(t)
        t._ballots = None

    @property
    def in_flight(self) -> int:
        return len(self.by_slot)

    KINDS = ("positions", "tally", "small", "pivot", "panels", "remainder", "output_wins", "ranking")

    def stats(self, profile: bool = False) -> dict:
        launches, grid, fl = ctypes.c_int64(), ctypes.c_int(), ctypes.c_int()
        busy = (ctypes.c_double * 8)()
        tasks = (ctypes.c_int64 * 8)()
        search = ctypes.c_double()
        check(self.L.se_engine_stats(self.engine, ctypes.byref(launches), ctypes.byref(grid), ctypes.byref(fl),
                                     busy if profile else None, tasks if profile else None,
                                     ctypes.byref(search) if profile else None))
        out = {"engine_launches": launches.value, "grid": grid.value, "in_flight": fl.value}
        if profile:
            out["busy_cta_ms"] = {k: busy[i] for i, k in enumerate(self.KINDS)}
            out["tasks"] = {k: tasks[i] for i, k in enumerate(self.KINDS)}
            out["search_cta_ms"] = search.value
        return out

    def close(self) -> None:
        """Stops the engine kernel (waiting for it) and frees its host state. The device
        buffers stay valid until the Server itself is released, so close() before that."""
        if self.engine:
            self.L.se_engine_destroy(self.engine)
            self.engine = ctypes.c_void_p()

    def __enter__(self) -> "Server":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class LoadResult:
    offered_rate: float
    achieved_rate: float
    p50_ms: float
    p99_ms: float
    mean_ms: float
    n: int
    makespan_s: float


def run_arrivals(server: Server, requests: list[tuple[int, int, torch.Tensor]], arrival_times: list[float],
                 keep_paths: bool = False, stall_s: float = 60.0) -> tuple[list[Ticket], float]:
    """Drives the server with requests (V, C, ballots) arriving at the given offsets (seconds
    from start): admits each as soon as it has arrived and fits, polls completions, and
    returns the finished tickets and the makespan. Ballots in host memory are copied to the
    device inside each request's latency window (from arrival). Raises if nothing completes
    for stall_s seconds while requests are in flight, or if a request can never fit the
    budget."""
    order = np.argsort(arrival_times, kind="stable")
    pending: list[Ticket] = []
    done: list[Ticket] = []
    nxt = 0
    t0 = time.perf_counter()
    n = len(requests)
    last_progress = t0
    host = {"admit_s": 0.0, "poll_s": 0.0, "iterations": 0}
    while len(done) < n:
        host["iterations"] += 1
        now_abs = time.perf_counter()
        if server.in_flight and now_abs - last_progress > stall_s:
            raise RuntimeError(f"no request finished for {stall_s:.0f} s ({server.in_flight} in flight)")
        now = now_abs - t0
        while nxt < n and arrival_times[order[nxt]] <= now:
            i = int(order[nxt])
            V, C, b = requests[i]
            t = Ticket(rid=i, V=V, C=C, arrival=t0 + arrival_times[i], keep_paths=keep_paths)
            t.parts = request_bytes(V, C)
            ids = 0 if getattr(b, "is_cuda", False) else (4 * V * C + ALIGN - 1) // ALIGN * ALIGN
            if t.parts["total"] + ids > server.arena.capacity:
                raise ValueError(f"request {i} needs {t.parts['total'] + ids} bytes, more than the whole budget")
            pending.append(t)
            nxt += 1
        if pending:
            ta = time.perf_counter()
            server.admit(pending, lambda t: requests[t.rid][2], ta)
            host["admit_s"] += time.perf_counter() - ta
        tp = time.perf_counter()
        finished = server.poll()
        host["poll_s"] += time.perf_counter() - tp
        if finished or not server.in_flight:
            last_progress = time.perf_counter()
        done.extend(finished)
        if not pending and nxt < n and server.in_flight == 0:
            time.sleep(max(0.0, min(0.001, arrival_times[order[nxt]] - (time.perf_counter() - t0))))
    server.last_host_stats = host
    return done, time.perf_counter() - t0


def summarize(tickets: list[Ticket], offered_rate: float, makespan: float) -> LoadResult:
    lat = np.array([t.latency for t in tickets]) * 1e3
    return LoadResult(offered_rate, len(tickets) / makespan, float(np.percentile(lat, 50)),
                      float(np.percentile(lat, 99)), float(lat.mean()), len(tickets), makespan)
