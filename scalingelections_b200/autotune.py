"""Autotuners for the batched closure and for the single-election closure.

tune_closure: for each size bucket of the single-election closure it times the round-by-round
schedules on a sample matrix and installs the fastest per bucket in the library's variant
table (se_closure_set_variant_table), which the automatic schedule reads:
  1  panels and pivots on the default micro-tile (8 x 8 words per thread, four warps in
     16-bit lanes), the next pivot fused into the remainder launch;
  3  panels on the wide micro-tile (8 x 4 words per thread, eight warps);
  4  as 3, and every pivot tile closed by its own launch on the wide micro-tile;
  5  as 3 on two streams: the next round's pivot row and column, pivot and panels overlap
     the current round's remaining remainder tiles;
  6  each round's remainder and the next round's panels in one launch, the panels in the
     remainder's last wave.
The schedules differ where the per-round chain (pivot, then panels) is not hidden behind the
remainder: small and medium C.

The batched closure's tuner (tune):

For each election-size bucket it times, on the GPU, the batched persistent closure of a
sample batch in both lane modes and keeps the faster, and in 16-bit lanes (C > 128) both
register micro-tiles of the tile tasks:
  lanes        16-bit (shifted by V // 2 when counts exceed 16 bits) or 32-bit;
  micro_tile   8 (8 x 8 words per thread, 128-thread CTAs) or 4 (8 x 4 words, 256-thread
               CTAs, each kind in its own persistent launch), the wide one only when it is at
               least 2 % faster.
Then, over a mixed sample with the same number of elections in every bucket (a log-uniform
spread of sizes, like a real batch), it times every pair of the settings that belong to the
whole persistent launch rather than to one election:
  ctas_per_sm  persistent CTAs per SM (1 or 2);
  order        elections of at most 128 candidates after the tiled ones, or before.
A per-bucket CTA count would be tuned on a few elections of one size, where one election's
chain of pivot rounds dominates, and would not carry over to a mixed launch. The tile is
128 x 128 cells everywhere. Results are stored as JSON and looked up per election.
"""
from __future__ import annotations

import json
import os
from pathlib import Path
from typing import Sequence

import numpy as np
import torch

from ._lib import LANES_U16, LANES_U32
from .batch import BatchedElections, lanes_for_voters

BUCKETS = [(1, 32), (33, 64), (65, 128), (129, 256), (257, 512), (513, 1024), (1025, 2048), (2049, 4096)]


def default_path() -> Path:
    env = os.environ.get("SE_AUTOTUNE_PATH")
    return Path(env) if env else Path.home() / ".cache" / "scalingelections_b200" / "autotune.json"


def bucket_of(C: int) -> int:
    for b, (lo, hi) in enumerate(BUCKETS):
        if lo <= C <= hi:
            return b
    return len(BUCKETS) - 1


def _sample_batch(lo: int, hi: int, n: int, V: int, seed: int, device) -> list[torch.Tensor]:
    """Random tallies of V ballots (complete ballots: d[i][j] + d[j][i] = V)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        C = int(rng.integers(lo, hi + 1))
        up = rng.integers(0, V + 1, size=(C, C), dtype=np.int64)
        d = np.triu(up, 1)
        d = d + np.triu(V - up, 1).T
        out.append(torch.from_numpy(d.astype(np.uint32).view(np.int32)).to(device).view(torch.uint32))
    return out


def _time(prefs, lanes, order, ctas, reps: int, micro_tiles=None) -> float:
    b = BatchedElections(prefs, lanes, order=order, ctas_per_sm=ctas, micro_tiles=micro_tiles)
    b.build_graph()
    b.launch_graph()
    b.check()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        b.launch_graph()
    e1.record(s)
    torch.cuda.synchronize()
    b.check()
    ms = e0.elapsed_time(e1) / reps
    b.close()
    return ms


def tune(V: int = 100000, per_bucket: int = 48, reps: int = 3, seed: int = 0, path: Path | None = None,
         device=None) -> dict:
    """Runs the search and writes the table; returns it. V is the ballot count of the sample
    tallies (above 65535 so both lane modes are legal only through the shifted 16-bit window)."""
    device = device or torch.device("cuda", torch.cuda.current_device())
    table = {"V_sample": V, "buckets": {}}
    for b, (lo, hi) in enumerate(BUCKETS):
        n = per_bucket if hi <= 1024 else max(4, per_bucket // 8)
        prefs = _sample_batch(lo, hi, n, V, seed + b, device)
        results = {}
        for lanes in (LANES_U16, LANES_U32):
            lane_pair = lanes_for_voters(V) if lanes == LANES_U16 else (LANES_U32, 0)
            if lane_pair[0] != lanes:
                continue
            results[f"u{lanes}"] = _time(prefs, [lane_pair] * len(prefs), 0, 2, reps)
        best = min(results, key=results.get)
        micro = 8
        if best == "u16" and hi > 128:  # the wide micro-tile, for elections with tile tasks
            lane_pair = lanes_for_voters(V)
            results["u16_wide"] = _time(prefs, [lane_pair] * len(prefs), 0, 2, reps, [4] * len(prefs))
            # A margin: the queues run one after another, so a split that noise decides only
            # costs the launches' balance.
            micro = 4 if results["u16_wide"] < 0.98 * results["u16"] else 8
        table["buckets"][str(b)] = {"range": [lo, hi], "lanes": int(best[1:]), "micro_tile": micro, "ms": results}
        del prefs
    mixed = []
    for b, (lo, hi) in enumerate(BUCKETS[:-1]):
        mixed += _sample_batch(lo, hi, max(2, per_bucket // 2), V, seed + 100 + b, device)
    lanes = [(LANES_U32, 0) if table["buckets"][str(bucket_of(int(p.shape[0])))]["lanes"] == 32
             else lanes_for_voters(V) for p in mixed]
    micro = choose_micro_tiles(table, [int(p.shape[0]) for p in mixed], lanes)
    launch = {(o, c): _time(mixed, lanes, o, c, reps, micro) for o in (0, 1) for c in (1, 2)}
    order, ctas = min(launch, key=launch.get)
    table["order"] = int(order)
    table["ctas_per_sm"] = int(ctas)
    table["launch_ms"] = {f"order{o}/ctas{c}": v for (o, c), v in launch.items()}
    p = Path(path) if path else default_path()
    p.parent.mkdir(parents=True, exist_ok=True)
    p.write_text(json.dumps(table, indent=1) + "\n")
    return table


CLOSURE_BUCKETS = [1024, 2048, 3072, 4096, 6144, 8192, 12288]  # upper bounds of the size buckets
CLOSURE_MODES = (1, 3, 4, 5, 6, 7, 8)


def tune_closure(sizes: Sequence[int] | None = None, reps: int = 5, V: int = 4096, seed: int = 0,
                 install: bool = True, device=None) -> dict:
    """Times the closure schedules CLOSURE_MODES at one size per bucket (the bucket's upper
    bound by default; 16-bit lanes, a random tally of V ballots) and returns
    {"sizes": {C: {mode: ms}}, "table": [(max_C, best mode), ...]}; installs the table in the
    library when `install`. Buckets above the last size keep mode 1."""
    from . import api

    device = device or torch.device("cuda", torch.cuda.current_device())
    sizes = list(sizes or CLOSURE_BUCKETS)
    out = {"sizes": {}, "table": []}
    s = torch.cuda.current_stream()
    try:
        for n, C in enumerate(sizes):
            d = _sample_batch(C, C, 1, V, seed + n, device)[0]
            work = torch.empty(api.closure_workspace_bytes(C, LANES_U16, dataflow=True), dtype=torch.uint8,
                               device=device)
            res = torch.empty_like(d)
            times = {}
            for mode in CLOSURE_MODES:
                api.set_closure_mode(mode)
                api.strongest_paths_device(d, lanes=LANES_U16, out=res, workspace=work)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(s)
                for _ in range(reps):
                    api.strongest_paths_device(d, lanes=LANES_U16, out=res, workspace=work)
                e1.record(s)
                torch.cuda.synchronize()
                times[mode] = e0.elapsed_time(e1) / reps
            out["sizes"][int(C)] = times
            out["table"].append((int(C), int(min(times, key=times.get))))
            del d, work, res
    finally:
        api.set_closure_mode(0)
    if install:
        api.set_closure_variants(out["table"])
    return out


def load(path: Path | None = None) -> dict | None:
    p = Path(path) if path else default_path()
    return json.loads(p.read_text()) if p.exists() else None


def choose(table: dict | None, Cs: Sequence[int], Vs: Sequence[int]) -> tuple[list, int, int]:
    """(lanes per election, order, ctas_per_sm) for a batch: per-bucket lane modes from the
    table (falling back to the widest legal 16-bit window), and the table's launch settings
    (0 CTAs per SM, i.e. as many as fit, without a table)."""
    lanes = []
    for C, V in zip(Cs, Vs):
        entry = (table or {}).get("buckets", {}).get(str(bucket_of(int(C))))
        pair = lanes_for_voters(int(V))
        if entry and entry["lanes"] == 32:
            pair = (LANES_U32, 0)
        lanes.append(pair)
    order = int((table or {}).get("order", 0))
    ctas = int((table or {}).get("ctas_per_sm", 0))
    return lanes, order, ctas


def choose_micro_tiles(table: dict | None, Cs: Sequence[int], lanes: Sequence) -> list[int]:
    """Micro-tile per election (BatchedElections micro_tiles): the bucket's tuned one for
    16-bit lanes, else the default 8 (32-bit lanes have the default only)."""
    out = []
    for C, lp in zip(Cs, lanes):
        entry = (table or {}).get("buckets", {}).get(str(bucket_of(int(C))))
        lb = int(lp[0]) if isinstance(lp, (tuple, list)) else int(lp)
        out.append(int(entry.get("micro_tile", 8)) if entry and lb == LANES_U16 else 8)
    return out
