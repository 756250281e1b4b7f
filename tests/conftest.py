import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def golden_names():
    return sorted(json.loads((GOLDEN / "index.json").read_text()).keys())


def load_golden(name):
    """A golden case. Cases kept small store hashes and ballots only: their preference matrix is
    re-tallied here by the oracle's scatter form and must match the reference's tally hash."""
    with np.load(GOLDEN / f"{name}.npz") as z:
        case = {k: z[k] for k in z.files}
    if "preferences" not in case:
        import hashlib

        from oracle import oracle

        d = oracle.tally(ballots_of(case), "scatter")
        assert hashlib.sha256(d.tobytes()).hexdigest() == str(case["tally_sha256"]), name
        case["preferences"] = d
    return case


def has_repeats(case):
    """True if some ballot of the case names a candidate twice."""
    return any(len(np.unique(b)) != len(b) for b in ballots_of(case))


def ballots_of(case):
    """The CSR ballots of a golden case as a list of arrays (the reference's input shape)."""
    ids, offs = case["ids"], case["offsets"]
    return [ids[offs[v]:offs[v + 1]] for v in range(len(offs) - 1)]


def chain_matrix(C, seed, order="shuffled", low=1000, high=61000, noise=100, base=0):
    """A preference matrix whose strongest paths run the length of the matrix.

    Candidates perm[0] -> perm[1] -> ... -> perm[C-1] defeat each other by chain weights w drawn
    from [low, high); the reverse counts are zero, and every other pair counts below `noise`.
    Every off-diagonal count is then raised by `base` (a shifted window of values). A path with a
    noise edge is weaker than any chain edge, so the strongest path from perm[s] to perm[t]
    (s < t) is the chain's segment: base + min(w[s:t]). `order` is "shuffled", "ascending"
    (the chain follows the indices, so it crosses pivots in loop order) or "descending"
    (against it). Returns (P, perm, w)."""
    rng = np.random.default_rng(seed)
    perm = {"shuffled": rng.permutation(C), "ascending": np.arange(C), "descending": np.arange(C)[::-1]}[order]
    P = rng.integers(0, noise, size=(C, C), dtype=np.uint64)
    w = rng.integers(low, high, size=max(C - 1, 0), dtype=np.uint64)
    P[perm[:-1], perm[1:]] = w
    P[perm[1:], perm[:-1]] = 0
    P += np.uint64(base)
    np.fill_diagonal(P, 0)
    return P.astype(np.uint32), perm, w


def chain_forward_ok(S, perm, w, base=0):
    """True if S holds the known strength of every forward pair of a chain_matrix."""
    for s in range(len(perm) - 1):
        want = np.minimum.accumulate(w[s:]) + np.uint64(base)
        if not np.array_equal(S[perm[s], perm[s + 1:]].astype(np.uint64), want):
            return False
    return True


def cyclic_ballots(C, seed, max_count=5):
    """Ballots whose strongest paths run around a cycle in single steps.

    Ballot r ranks perm[r], perm[r + 1], ..., perm[C - 1], perm[0], ..., perm[r - 1] (the order
    rotated by r), cast by n[r] voters (n in [1, max_count]); N = sum(n). Then perm[s] beats
    perm[s + 1] (cyclically) by N - n[s + 1], every kept defeat is a forward jump around the
    cycle, and a jump over the rotations (s, t] is never stronger than the single steps across
    them. So the strongest path from perm[s] to perm[t] is the chain of single steps, with
    strength N - max(n[u] for u in (s, t], cyclically). Needs C > 2 * max_count.
    Returns (ballots int32 [N, C], perm, n)."""
    rng = np.random.default_rng(seed)
    perm = rng.permutation(C)
    n = rng.integers(1, max_count + 1, size=C)
    ballots = np.concatenate([np.tile(np.roll(perm, -r), (int(n[r]), 1)) for r in range(C)])
    return ballots.astype(np.int32), perm, n


def cyclic_strongest_paths(perm, n):
    """The closed-form strongest-path matrix of cyclic_ballots(...)."""
    C, N = len(perm), int(n.sum())
    S = np.zeros((C, C), dtype=np.uint32)
    for s in range(C):
        u = (s + 1 + np.arange(C - 1)) % C  # perm[s + 1], perm[s + 2], ... around the cycle
        S[perm[s], perm[u]] = N - np.maximum.accumulate(n[u])
    return S


def cyclic_tally(perm, n):
    """The preference matrix of cyclic_ballots(...): voters of rotation r rank perm[s] above
    perm[t] unless r lies in (s, t] (for s < t), so d[perm[s]][perm[t]] = N - n[s+1 .. t] and
    d[perm[t]][perm[s]] = n[s+1 .. t]."""
    C = len(perm)
    P = np.concatenate([[0], np.cumsum(n)]).astype(np.int64)  # P[k] = n[0] + ... + n[k-1]
    s = np.arange(C)[:, None]
    t = np.arange(C)[None, :]
    between = np.abs(P[t + 1] - P[s + 1])  # voters of the rotations strictly after min(s, t) up to max(s, t)
    d_rot = np.where(s < t, P[-1] - between, between)
    np.fill_diagonal(d_rot, 0)
    d = np.zeros((C, C), dtype=np.uint32)
    d[np.ix_(perm, perm)] = d_rot
    return d


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle

    oracle.lib()
    return oracle
