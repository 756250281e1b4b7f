"""CPU oracle for the Schulze path: TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg (plus its
``--impl reference`` arm) may import this module, and only as the checker or the timed CPU
baseline. The product package ``scalingelections_b200`` never imports it.

Wraps ``oracle.c`` (a C restatement of the reference's algorithm, each function citing the
``scaling_elections.py`` lines it follows) and, where it was built, the reference's own CPU
closure compiled unmodified from ``scaling_elections.cu`` into ``oracle/_ref``, and its CUDA
build (the reference's own GPU kernels, for sm_100a) into ``oracle/_ref/gpu``.
"""
from __future__ import annotations

import ctypes
import importlib.machinery
import importlib.util
import os
import subprocess
import sysconfig
from pathlib import Path
from typing import Sequence

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"
REF_PATH = HERE / "_ref" / ("scaling_elections" + sysconfig.get_config_var("EXT_SUFFIX"))
REF_GPU_PATH = HERE / "_ref" / "gpu" / ("scaling_elections" + sysconfig.get_config_var("EXT_SUFFIX"))

_lib = None
_ref = None
_ref_gpu = None

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")


def reference_dir() -> Path | None:
    """The reference checkout named by SE_REFERENCE_DIR, when that directory holds its sources."""
    d = os.environ.get("SE_REFERENCE_DIR")
    return Path(d) if d and (Path(d) / "scaling_elections.cu").exists() else None


def build(reference: bool = True) -> None:
    """Compile liboracle.so and, when SE_REFERENCE_DIR names the reference sources, oracle/_ref."""
    subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
    ref = reference_dir()
    if reference and ref is not None:
        for target in ("ref", "ref_gpu"):
            subprocess.run(["make", "-s", "-C", str(HERE), target, f"REF={ref}"], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build(reference=False)
        L = ctypes.CDLL(str(LIB_PATH))
        L.or_tally_scatter.argtypes = [_i32p, _i64p, ctypes.c_int64, ctypes.c_int, _u32p]
        L.or_tally_positions.argtypes = [_i32p, _i64p, ctypes.c_int64, ctypes.c_int, _u32p, _i32p]
        L.or_defeats.argtypes = [_u32p, ctypes.c_int64, ctypes.c_int, _u32p]
        L.or_defeats.restype = None
        L.or_closure_serial.argtypes = [_u32p, ctypes.c_int]
        L.or_closure_serial.restype = None
        L.or_closure_blocked.argtypes = [_u32p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.or_closure_blocked.restype = None
        L.or_rank.argtypes = [_u32p, ctypes.c_int64, ctypes.c_int, _i32p, _i32p]
        L.or_widest_from.argtypes = [_u32p, ctypes.c_int64, ctypes.c_int, ctypes.c_int, _u32p]
        L.or_rim_decode.argtypes = [_i64p, ctypes.c_int64, ctypes.c_int, _i64p]
        _lib = L
    return _lib


def to_csr(voter_rankings: Sequence[np.ndarray]) -> tuple[np.ndarray, np.ndarray]:
    """Ballots as (ids int32, offsets int64). A 2-D array is taken as one ballot per row."""
    if isinstance(voter_rankings, np.ndarray) and voter_rankings.ndim == 2:
        V, L = voter_rankings.shape
        ids = np.ascontiguousarray(voter_rankings, dtype=np.int32).reshape(-1)
        return ids, np.arange(V + 1, dtype=np.int64) * L
    lens = np.fromiter((len(r) for r in voter_rankings), dtype=np.int64, count=len(voter_rankings))
    offsets = np.zeros(len(lens) + 1, dtype=np.int64)
    np.cumsum(lens, out=offsets[1:])
    ids = (np.concatenate([np.asarray(r, dtype=np.int32) for r in voter_rankings])
           if len(lens) else np.zeros(0, np.int32))
    return np.ascontiguousarray(ids), offsets


def num_candidates(voter_rankings: Sequence[np.ndarray]) -> int:
    """scaling_elections.py:63-66: max id + 1, at least 1."""
    ids, _ = to_csr(voter_rankings)
    return int(max(1, int(ids.max()) + 1)) if ids.size else 1


def tally(voter_rankings: Sequence[np.ndarray], method: str = "scatter") -> np.ndarray:
    """build_pairwise_preferences (scaling_elections.py:51-88) restated in C."""
    ids, offsets = to_csr(voter_rankings)
    C = num_candidates(voter_rankings)
    d = np.zeros((C, C), dtype=np.uint32)
    V = len(offsets) - 1
    if method == "scatter":
        rc = lib().or_tally_scatter(ids, offsets, V, C, d)
    else:
        pos = np.empty(V * C, dtype=np.int32)
        rc = lib().or_tally_positions(ids, offsets, V, C, d, pos)
    if rc != 0:
        raise ValueError("malformed ballot (id out of range or repeated)")
    return d


def defeats(preferences: np.ndarray) -> np.ndarray:
    d = np.ascontiguousarray(preferences, dtype=np.uint32)
    C = d.shape[0]
    S = np.empty((C, C), dtype=np.uint32)
    lib().or_defeats(d, C, C, S)
    return S


def strongest_paths(preferences: np.ndarray, method: str = "serial", tile: int = 16,
                    threads: int = 0) -> np.ndarray:
    """compute_strongest_paths_numba_serial (py:91-125) or _numba_parallel (py:162-271)."""
    S = defeats(preferences)
    C = S.shape[0]
    if method == "serial":
        lib().or_closure_serial(S, C)
    elif method == "blocked":
        lib().or_closure_blocked(S, C, tile, threads)
    else:
        raise ValueError(method)
    return S


def widest_rows(preferences: np.ndarray, sources) -> np.ndarray:
    """Rows `sources` of the closure, each by an O(C^2) bottleneck Dijkstra (independent of
    any Floyd-Warshall ordering). Returns uint32 [len(sources), C]."""
    S0 = defeats(preferences)
    C = S0.shape[0]
    out = np.empty((len(sources), C), dtype=np.uint32)
    for n, s in enumerate(sources):
        row = np.empty(C, dtype=np.uint32)
        if lib().or_widest_from(S0, C, C, int(s), row) != 0:
            raise MemoryError("or_widest_from")
        out[n] = row
    return out


def wins_and_ranking(strongest: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """get_winner_and_ranking (scaling_elections.py:274-296): (wins, ranking) as int32."""
    S = np.ascontiguousarray(strongest, dtype=np.uint32)
    C = S.shape[0]
    wins = np.empty(C, dtype=np.int32)
    ranking = np.empty(C, dtype=np.int32)
    if lib().or_rank(S, C, C, wins, ranking) != 0:
        raise MemoryError("or_rank")
    return wins, ranking


def winner_and_ranking(strongest: np.ndarray, candidates: list | None = None):
    """Same return shape as the reference: (winner, ranked candidate list)."""
    _, ranking = wins_and_ranking(strongest)
    cands = list(range(strongest.shape[0])) if candidates is None else candidates
    ranked = [cands[i] for i in ranking]
    return ranked[0], ranked


def mallows_ballots(V: int, C: int, phi: float, seed: int) -> np.ndarray:
    """The same ballots as scalingelections_b200.ballots.mallows_ballots (same seed, same
    random stream), with the insertion decode done in C for speed. Test-input generation."""
    from scalingelections_b200 import ballots as B

    rng = np.random.default_rng(seed)
    pi0 = rng.permutation(C).astype(np.int32)
    slots = np.ascontiguousarray(B._insertion_positions(rng, V, C, phi))
    final = np.empty((V, C), dtype=np.int64)
    if lib().or_rim_decode(slots, V, C, final) != 0:
        raise RuntimeError("insertion decode failed")
    out = np.empty((V, C), dtype=np.int32)
    np.put_along_axis(out, final, np.broadcast_to(pi0, (V, C)), axis=1)
    return out


def reference_gpu():
    """The reference's own CUDA module (scaling_elections.cu built by `make ref_gpu` for
    sm_100a), or None. Loaded like reference_cpu(), outside sys.modules."""
    global _ref_gpu
    if _ref_gpu is None and REF_GPU_PATH.exists():
        loader = importlib.machinery.ExtensionFileLoader("scaling_elections", str(REF_GPU_PATH))
        spec = importlib.util.spec_from_file_location("scaling_elections", str(REF_GPU_PATH), loader=loader)
        mod = importlib.util.module_from_spec(spec)
        loader.exec_module(mod)
        _ref_gpu = mod
    return _ref_gpu


def reference_cpu():
    """The reference's own CPU module (scaling_elections.cu built by `make ref`), or None.

    Loaded under its own name without entering sys.modules, so it never shadows the
    product's drop-in module of the same name."""
    global _ref
    if _ref is None and REF_PATH.exists():
        loader = importlib.machinery.ExtensionFileLoader("scaling_elections", str(REF_PATH))
        spec = importlib.util.spec_from_file_location("scaling_elections", str(REF_PATH), loader=loader)
        mod = importlib.util.module_from_spec(spec)
        loader.exec_module(mod)
        _ref = mod
    return _ref
