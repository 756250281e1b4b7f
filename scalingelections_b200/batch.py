"""Batched closure: many independent elections of uneven size closed (and ranked) by one
persistent launch per lane mode, optionally replayed as a CUDA graph (include/se.h,
se_batch_*). No reference counterpart: the reference closes one matrix per call
(scaling_elections.cu:863-989).
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import torch

from . import _lib
from ._lib import LANES_U16, LANES_U32, check
from .api import _check_matrix, _workspace


def lanes_for_voters(num_voters: int) -> tuple[int, int]:
    """(lane_bits, value_offset) for a tally of num_voters ballots. A kept count d[i][j] > d[j][i]
    with d[i][j] + d[j][i] = V lies in (V/2, V], so storing it as d - V//2 fits 16 bits for
    every V <= 131070; below 65536 no shift is needed."""
    V = int(num_voters)
    if V < 65536:
        return LANES_U16, 0
    if V <= 131070:
        return LANES_U16, V // 2
    return LANES_U32, 0


class BatchedElections:
    """A prepared batch. ``preferences`` are CUDA uint32 [C_e, C_e] matrices (any row stride
    with contiguous rows); results land in ``strongest_paths``, ``wins`` and ``rankings``.

    lanes: per election, LANES_U16 or LANES_U32, or (lanes, value_offset) pairs such as
    lanes_for_voters() returns; None picks from each matrix's maximum (one device-to-host
    read for the whole batch). micro_tiles: per election, 8 (the default 8 x 8-word micro-tile)
    or 4 (the wide 8 x 4-word one, 256-thread CTAs; 16-bit lanes), run as separate persistent
    launches; None is 8 everywhere. order: 0 runs small elections (C <= 128) after the tiled
    ones, 1 before them. ctas_per_sm: persistent CTAs per SM (0 = as many as fit). An autotuned
    table (scalingelections_b200.autotune) supplies lanes, micro-tiles, order and ctas_per_sm
    per size bucket. The batch keeps references to every buffer it uses."""

    def __init__(self, preferences: Sequence[torch.Tensor], lanes: Sequence | None = None, *,
                 ranking: bool = True, order: int = 0, ctas_per_sm: int = 0,
                 micro_tiles: Sequence[int] | None = None):
        if not preferences:
            raise ValueError("empty batch")
        self.device = preferences[0].device
        self.prefs = list(preferences)
        shapes = [_check_matrix(p, "preferences") for p in self.prefs]
        if any(p.device != self.device for p in self.prefs):
            raise ValueError("all matrices must be on one device")
        if lanes is None:
            with torch.cuda.device(self.device):
                maxima = torch.stack([p.view(torch.int32).max() if p.numel() else
                                      torch.zeros((), dtype=torch.int32, device=self.device)
                                      for p in self.prefs]).cpu()
            # A negative int32 view means a u32 value >= 2^31.
            lanes = [LANES_U16 if 0 <= int(m) <= 0xFFFF else LANES_U32 for m in maxima]
        pairs = [(int(x[0]), int(x[1])) if isinstance(x, (tuple, list)) else (int(x), 0) for x in lanes]
        self.lanes = [p[0] for p in pairs]
        self.offsets = [p[1] for p in pairs]
        if len(self.lanes) != len(self.prefs):
            raise ValueError("one lane mode per election")
        self.micro_tiles = [8] * len(self.prefs) if micro_tiles is None else [int(m) for m in micro_tiles]
        if len(self.micro_tiles) != len(self.prefs):
            raise ValueError("one micro-tile per election")
        self.outs, self.wins, self.rankings = [], [], []
        arr = (_lib.Election * len(self.prefs))()
        for e, (p, (C, ld)) in enumerate(zip(self.prefs, shapes)):
            if C == 0:
                raise ValueError("an election needs at least one candidate")
            out = torch.empty((C, C), dtype=torch.uint32, device=self.device)
            self.outs.append(out)
            w = r = None
            if ranking:
                w = torch.empty(C, dtype=torch.int32, device=self.device)
                r = torch.empty(C, dtype=torch.int32, device=self.device)
            self.wins.append(w)
            self.rankings.append(r)
            arr[e] = _lib.Election(p.data_ptr(), ld, out.data_ptr(), C, w.data_ptr() if w is not None else None,
                                   r.data_ptr() if r is not None else None, C, self.lanes[e], self.offsets[e],
                                   self.micro_tiles[e])
        self._arr = arr
        L = _lib.lib()
        need = L.se_batch_workspace_bytes(len(self.prefs), ctypes.cast(arr, ctypes.c_void_p))
        if need < 0:
            raise _lib.SchulzeError(_lib.SE_ERR_INVALID, _lib.last_error() or "invalid batch")
        self.workspace = _workspace(need, self.device)
        self.plan = _lib.BatchPlan()
        with torch.cuda.device(self.device):
            check(L.se_batch_prepare(len(self.prefs), ctypes.cast(arr, ctypes.c_void_p), self.workspace.data_ptr(),
                                     need, int(order), int(ctas_per_sm), ctypes.byref(self.plan)))
        self._graph = False

    @property
    def strongest_paths(self) -> list[torch.Tensor]:
        return self.outs

    def task_counts(self) -> tuple[int, int, int]:
        """Tasks of the three persistent launches: 16-bit lanes, 32-bit lanes, 16-bit lanes on
        the wide micro-tile."""
        L = _lib.lib()
        return tuple(L.se_batch_task_count(ctypes.byref(self.plan), q) for q in range(3))

    def run(self) -> None:
        """Enqueue the whole batch on the current stream (asynchronous)."""
        with torch.cuda.device(self.device):
            check(_lib.lib().se_batch_run(ctypes.byref(self.plan), torch.cuda.current_stream().cuda_stream))

    def build_graph(self) -> None:
        with torch.cuda.device(self.device):
            check(_lib.lib().se_batch_graph_build(ctypes.byref(self.plan)))
        self._graph = True

    def launch_graph(self) -> None:
        if not self._graph:
            self.build_graph()
        with torch.cuda.device(self.device):
            check(_lib.lib().se_batch_graph_launch(ctypes.byref(self.plan), torch.cuda.current_stream().cuda_stream))

    KINDS = ("small", "pivot", "row_panel", "col_panel", "remainder")

    def profile(self) -> dict:
        """CTA-milliseconds busy per task kind, tasks run and CTA-milliseconds spent waiting on
        dependencies, accumulated over the runs since the plan's last reset (each run resets)."""
        busy = (ctypes.c_double * 5)()
        tasks = (ctypes.c_int64 * 5)()
        wait = ctypes.c_double()
        with torch.cuda.device(self.device):
            check(_lib.lib().se_batch_profile(ctypes.byref(self.plan), busy, tasks, ctypes.byref(wait),
                                              torch.cuda.current_stream().cuda_stream))
        return {"busy_cta_ms": dict(zip(self.KINDS, busy)), "tasks": dict(zip(self.KINDS, tasks)),
                "wait_cta_ms": wait.value}

    def set_wait_limit(self, seconds: float) -> None:
        """Limit of one dependency wait of the persistent kernel (default 5 s). A wait that
        runs out ends the run with an error that check() raises; the GPU stays usable. Applies
        to later runs; a built graph is released and rebuilt on the next launch_graph()."""
        check(_lib.lib().se_batch_set_wait_limit(ctypes.byref(self.plan), int(max(0.0, seconds) * 1e9)))
        self._graph = False

    def check(self) -> None:
        """Raise if a kernel of the last run reported an error (synchronises the stream)."""
        with torch.cuda.device(self.device):
            check(_lib.lib().se_batch_check(ctypes.byref(self.plan), torch.cuda.current_stream().cuda_stream))

    def close(self) -> None:
        """Releases the captured CUDA graph, if any."""
        if getattr(self, "plan", None) is not None and self._graph:
            _lib.lib().se_batch_release(ctypes.byref(self.plan))
            self._graph = False

    def __enter__(self) -> "BatchedElections":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def strongest_paths_batched(preferences: Sequence[torch.Tensor], lanes: Sequence[int] | None = None):
    """One-shot batched closure + ranking: returns (strongest paths, wins, rankings) lists."""
    b = BatchedElections(preferences, lanes)
    b.run()
    b.check()
    return b.outs, b.wins, b.rankings
