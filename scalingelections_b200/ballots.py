"""Seeded synthetic ballot generators (host side, NumPy).

The reference draws its benchmark ballots with unseeded ``np.random.permutation``
(scaling_elections.py:477-481) or draws a random preference matrix directly
(``np.random.randint(0, C, (C, C))``, :473-476). This module gives seeded equivalents, plus a
Mallows-model sampler (not in the reference) written from the model's definition:

Mallows(pi0, phi): P(pi) proportional to phi ** kendall_tau(pi, pi0). Sampled with the
repeated insertion model: the items of pi0 are inserted one at a time; item i (0-based)
lands at position j in {0, ..., i} with probability proportional to phi ** (i - j), so
phi = 1 is uniform and phi -> 0 reproduces pi0.
"""
from __future__ import annotations

import numpy as np


def uniform_ballots(V: int, C: int, seed: int) -> np.ndarray:
    """V independent uniform random permutations of 0..C-1, as an int32 [V, C] array
    (row v = ballot v, most preferred first)."""
    rng = np.random.default_rng(seed)
    base = np.broadcast_to(np.arange(C, dtype=np.int32), (V, C))
    return rng.permuted(base, axis=1).astype(np.int32, copy=False)


def random_preferences(C: int, seed: int, high: int | None = None) -> np.ndarray:
    """The reference's "--num-voters 0" input: uint32 [C, C] uniform in [0, high) with
    high = C by default (scaling_elections.py:474-476), seeded."""
    rng = np.random.default_rng(seed)
    hi = C if high is None else high
    return rng.integers(0, hi, size=(C, C), dtype=np.uint64).astype(np.uint32)


def _insertion_positions(rng: np.random.Generator, V: int, C: int, phi: float) -> np.ndarray:
    """Insertion slot j_i in [0, i] for each voter and item, P(j) ~ phi ** (i - j)."""
    i = np.arange(C, dtype=np.float64)
    u = rng.random((V, C))
    if phi >= 1.0:
        disp = np.floor(u * (i + 1.0))
    else:
        # Truncated geometric displacement d = i - j in [0, i]: inverse CDF of
        # P(d) = phi^d (1 - phi) / (1 - phi^(i+1)).
        tail = 1.0 - np.power(phi, i + 1.0)
        disp = np.floor(np.log1p(-u * tail) / np.log(phi))
    disp = np.clip(disp, 0.0, i)
    return (i - disp).astype(np.int64)


def _decode_insertions(slots: np.ndarray) -> np.ndarray:
    """Final position of every item, given each item's insertion slot.

    Processing items from last inserted to first, item i takes the slots[i]-th still-free
    final position (0-based): later insertions only push it right. A Fenwick tree over free
    positions finds that slot in O(log C); the descent is vectorised across voters."""
    V, C = slots.shape
    size = 1
    while size < C:
        size <<= 1
    tree = np.zeros((V, size + 1), dtype=np.int32)
    # Fenwick tree with every position 1..C free: node k holds lowbit(k) positions, clipped
    # to C.
    k = np.arange(1, size + 1)
    low = k & -k
    tree[:, 1:] = np.clip(np.minimum(k, C) - (k - low), 0, None).astype(np.int32)
    pos = np.empty((V, C), dtype=np.int64)
    rows = np.arange(V)
    for item in range(C - 1, -1, -1):
        want = slots[:, item] + 1  # 1-based rank among free slots
        idx = np.zeros(V, dtype=np.int64)
        step = size
        while step:
            nxt = idx + step
            ok = nxt <= size
            t = np.where(ok, tree[rows, np.minimum(nxt, size)], 0)
            go = ok & (t < want)
            idx = np.where(go, nxt, idx)
            want = np.where(go, want - t, want)
            step >>= 1
        p = idx + 1  # 1-based free slot found
        pos[:, item] = p - 1
        j = p.copy()
        while True:
            live = j <= size
            if not live.any():
                break
            tree[rows[live], j[live]] -= 1
            j = np.where(live, j + (j & -j), j)
    return pos


def mallows_ballots(V: int, C: int, phi: float, seed: int, reference: np.ndarray | None = None) -> np.ndarray:
    """V ballots from Mallows(reference, phi) as int32 [V, C] (most preferred first).
    The reference order defaults to a seeded uniform permutation."""
    rng = np.random.default_rng(seed)
    pi0 = rng.permutation(C).astype(np.int32) if reference is None else np.asarray(reference, np.int32)
    if not 0.0 < phi <= 1.0:
        raise ValueError("phi must be in (0, 1]")
    slots = _insertion_positions(rng, V, C, phi)
    final = _decode_insertions(slots)  # final[v, i] = place of pi0[i] in ballot v
    out = np.empty((V, C), dtype=np.int32)
    np.put_along_axis(out, final, np.broadcast_to(pi0, (V, C)), axis=1)
    return out


def mallows_ballots_device(V: int, C: int, phi: float, seed: int, reference=None, device="cuda"):
    """V Mallows(reference, phi) ballots drawn on the GPU, as a CUDA int32 [V, C] tensor.
    phi = 1 gives uniform permutations. The reference order defaults to a seeded uniform
    permutation (drawn on the host). Deterministic in (seed, ballot index); not the same
    stream of ballots as the host sampler above."""
    import torch

    from . import _lib

    if reference is None:
        reference = np.random.default_rng(seed).permutation(C).astype(np.int32)
    ref = torch.from_numpy(np.ascontiguousarray(reference, dtype=np.int32)).to(device)
    out = torch.empty((V, C), dtype=torch.int32, device=device)
    L = _lib.lib()
    need = L.se_mallows_workspace_bytes(int(V), int(C))
    if need < 0:
        raise ValueError("invalid ballot shape")
    work = torch.empty(max(need, 256), dtype=torch.uint8, device=device)
    with torch.cuda.device(out.device):
        _lib.check(L.se_mallows_ballots(int(V), int(C), float(phi), int(seed) & (2**64 - 1), ref.data_ptr(),
                                        out.data_ptr(), work.data_ptr(), need,
                                        torch.cuda.current_stream().cuda_stream))
    return out


def random_preferences_device(C: int, seed: int, high: int | None = None, device="cuda"):
    """The reference's random benchmark matrix (scaling_elections.py:473-476: values uniform in
    [0, C)) drawn on the GPU as a CUDA uint32 [C, C] tensor: a counter-based, seeded draw,
    not NumPy's stream (``random_matrix_host`` restates it on the host)."""
    import torch

    from . import _lib

    out = torch.empty((C, C), dtype=torch.uint32, device=device)
    with torch.cuda.device(out.device):
        _lib.check(_lib.lib().se_random_preferences(int(C), int(high or 0), int(seed) & (2**64 - 1), out.data_ptr(),
                                                    max(int(C), 1), torch.cuda.current_stream().cuda_stream))
    return out


def _splitmix64(x: np.ndarray) -> np.ndarray:
    x = x + np.uint64(0x9E3779B97F4A7C15)
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def random_matrix_host(C: int, seed: int, high: int | None = None) -> np.ndarray:
    """Host restatement of random_preferences_device, bit for bit (for checking and for
    callers without a GPU)."""
    high = np.uint64(high or C)
    with np.errstate(over="ignore"):
        x = np.arange(C * C, dtype=np.uint64)
        h = _splitmix64(np.uint64(int(seed) & (2**64 - 1)) ^ _splitmix64(x))
        v = ((h >> np.uint64(32)) * high) >> np.uint64(32)
    return v.astype(np.uint32).reshape(C, C)
