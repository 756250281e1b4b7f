"""Generates the golden fixtures in this directory from the REFERENCE implementation.

Run where the reference sources are present (they are never copied into this repository):

    SE_REFERENCE_DIR=<reference checkout> python tests/golden/make_golden.py [--ref DIR]

It imports the reference's ``scaling_elections.py`` by path (its module-level import of the
native extension is satisfied by a stub, since only the Numba/NumPy functions are used) and
runs, on seeded inputs:
  * build_pairwise_preferences           (scaling_elections.py:51-88)
  * compute_strongest_paths_numba_serial (scaling_elections.py:91-125)
  * compute_strongest_paths_numba_parallel, tile 16, where C % 16 == 0 (py:162-271)
  * get_winner_and_ranking               (scaling_elections.py:274-296)
and the participation-paradox ballots of validate_paradox.py:26-28 through the same calls.
Each case is stored as a compressed .npz holding its inputs and the reference's outputs, so
the fixtures do not depend on any random generator at test time. With --configs it writes
the configuration-size cases instead (see config_cases): hashes of the reference's outputs on
ballots regenerated from a seed, since the inputs would be tens of megabytes.
"""
from __future__ import annotations

import argparse
import hashlib
import importlib.util
import json
import multiprocessing
import os
import sys
import tempfile
import time
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def load_reference(ref_dir: Path):
    stub = types.ModuleType("scaling_elections")
    stub.log_gpus = lambda: None
    stub.compute_strongest_paths = lambda *a, **k: None
    saved = sys.modules.get("scaling_elections")
    sys.modules["scaling_elections"] = stub
    try:
        spec = importlib.util.spec_from_file_location("reference_scaling_elections", ref_dir / "scaling_elections.py")
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
    finally:
        if saved is None:
            del sys.modules["scaling_elections"]
        else:
            sys.modules["scaling_elections"] = saved
    return mod


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def csr(rankings):
    lens = np.array([len(r) for r in rankings], dtype=np.int64)
    offs = np.zeros(len(rankings) + 1, dtype=np.int64)
    np.cumsum(lens, out=offs[1:])
    ids = np.concatenate([np.asarray(r, dtype=np.int32) for r in rankings])
    return ids, offs


def config_cases(ref, only: list[str] | None = None) -> None:
    """Configuration-size cases kept as hashes: the ballots are regenerated from their seed by
    scalingelections_b200.ballots at test time, so only the reference's outputs are stored.
      * config_c4096_v4096: C = 4096, V = 4096 uniform permutations (seed 4096), the
        single-election configuration with the reference's tile sweep. Closure by the tiled and
        the serial Numba paths (checked equal). A few minutes on 8 cores.
      * config_c16384_v4096: C = 16384, V = 4096 Mallows(0.8) ballots (seed 16384), the
        headline size. Closure by the tiled Numba path only (the serial one would take hours;
        the two are equal at every size checked). About an hour on 8 cores.
    Each: tally by build_pairwise_preferences, ranking by get_winner_and_ranking."""
    from scalingelections_b200.ballots import mallows_ballots, uniform_ballots

    cases = {
        "config_c4096_v4096": (4096, 4096, 4096, None, "scalingelections_b200.ballots.uniform_ballots(V, C, seed)",
                               True),
        "config_c16384_v4096": (16384, 4096, 16384, 0.8,
                                "scalingelections_b200.ballots.mallows_ballots(V, C, phi, seed)", False),
    }
    for name, (C, V, seed, phi, how, serial) in cases.items():
        if only and name not in only:
            continue
        B = uniform_ballots(V, C, seed=seed) if phi is None else mallows_ballots(V, C, phi, seed=seed)
        d = ref.build_pairwise_preferences(list(B))
        del B
        d = np.ascontiguousarray(d, dtype=np.uint32)
        S = ref.compute_strongest_paths_numba_parallel(d, tile_size=16)
        if serial:
            assert np.array_equal(S, ref.compute_strongest_paths_numba_serial(d))
        winner, ranking = ref.get_winner_and_ranking(list(range(C)), S)
        case = dict(C=C, V=V, seed=seed, phi=phi, ballots=how, tally_sha256=sha(d), strongest_sha256=sha(S),
                    winner=int(winner), ranking=[int(x) for x in ranking])
        (HERE / f"{name}.json").write_text(json.dumps(case) + "\n")
        print(name, {k: v for k, v in case.items() if k != "ranking"}, flush=True)


def _tally_slice(job) -> str:
    """Worker of parallel_tally: the reference's build_pairwise_preferences over ballots
    [lo, hi) of the seeded Mallows ballots, saved to `out`."""
    ref_dir, V, C, phi, seed, lo, hi, out = job
    sys.path.insert(0, str(HERE.parent.parent))
    from oracle import oracle

    ref = load_reference(Path(ref_dir))
    B = oracle.mallows_ballots(V, C, phi, seed=seed)[lo:hi]
    d = ref.build_pairwise_preferences(list(B))
    assert d.shape == (C, C)  # every slice holds complete permutations: max id + 1 == C
    np.save(out, np.ascontiguousarray(d, dtype=np.uint32))
    return out


def parallel_tally(ref_dir: Path, V: int, C: int, phi: float, seed: int, workers: int) -> np.ndarray:
    """build_pairwise_preferences (py:51-88) over all V ballots, run as `workers` processes each
    on a contiguous slice of voters, the slice matrices summed. The tally is a sum over voters
    (py:72-86: every ballot adds into the same matrix), and every slice has the same candidate
    count (complete permutations), so the sum is the single call's result."""
    bounds = np.linspace(0, V, workers + 1).astype(int)
    with tempfile.TemporaryDirectory(dir=os.environ.get("SE_GOLDEN_TMP")) as tmp:
        jobs = [(str(ref_dir), V, C, phi, seed, int(lo), int(hi), str(Path(tmp) / f"part{n}.npy"))
                for n, (lo, hi) in enumerate(zip(bounds[:-1], bounds[1:])) if hi > lo]
        with multiprocessing.get_context("spawn").Pool(len(jobs)) as pool:
            parts = pool.map(_tally_slice, jobs)
        d = np.zeros((C, C), dtype=np.uint32)
        for part in parts:
            d += np.load(part, mmap_mode="r")
    return d


def large_cases(ref, ref_dir: Path, workers: int) -> None:
    """The configuration sizes beyond a Numba closure's reach here.

    The closure is the reference's own OpenMP CPU path (compute_strongest_paths with
    allow_gpu=False, scaling_elections.cu:738-849), compiled unmodified into oracle/_ref, at
    tile 16. It equals the Numba closures wherever C is a multiple of the tile; this is first
    checked at C = 16384 against the hash that the tiled Numba closure (py:162-271) produced
    for config_c16384_v4096, on the reference's tally of the same ballots.

      * config_c32768_v4096: C = 32768, V = 4096 Mallows(0.8) ballots (seed 32768). The tally
        by build_pairwise_preferences over voter slices in parallel, the closure as above, the
        ranking by get_winner_and_ranking (py:274-296)."""
    from oracle import oracle

    omp = oracle.reference_cpu()
    if omp is None:
        raise SystemExit("oracle/_ref is not built: make -C oracle ref")
    c16 = json.loads((HERE / "config_c16384_v4096.json").read_text())
    t0 = time.time()
    d = parallel_tally(ref_dir, c16["V"], c16["C"], c16["phi"], c16["seed"], workers)
    assert sha(d) == c16["tally_sha256"], "sliced tally differs from the stored single-call tally"
    t1 = time.time()
    S = omp.compute_strongest_paths(d, allow_gpu=False, allow_tma=False, tile_size=16)
    assert sha(S) == c16["strongest_sha256"], "OpenMP closure differs from the stored Numba closure"
    print(f"C=16384: sliced tally {t1 - t0:.0f} s and OpenMP closure {time.time() - t1:.0f} s "
          "equal the stored reference hashes", flush=True)
    del d, S

    C, V, seed, phi = 32768, 4096, 32768, 0.8
    t0 = time.time()
    d = parallel_tally(ref_dir, V, C, phi, seed, workers)
    t1 = time.time()
    print(f"C={C}: tally {t1 - t0:.0f} s", flush=True)
    S = omp.compute_strongest_paths(d, allow_gpu=False, allow_tma=False, tile_size=16)
    t2 = time.time()
    print(f"C={C}: closure {t2 - t1:.0f} s", flush=True)
    winner, ranking = ref.get_winner_and_ranking(list(range(C)), S)
    print(f"C={C}: ranking {time.time() - t2:.0f} s", flush=True)
    case = dict(C=C, V=V, seed=seed, phi=phi,
                ballots="oracle.mallows_ballots(V, C, phi, seed): scalingelections_b200.ballots.mallows_ballots "
                        "with the insertion decode in C",
                tally="build_pairwise_preferences over voter slices, summed",
                closure="scaling_elections.cu compute_strongest_paths(allow_gpu=False, tile_size=16), OpenMP",
                tally_sha256=sha(d), strongest_sha256=sha(S), winner=int(winner),
                ranking=[int(x) for x in ranking])
    (HERE / "config_c32768_v4096.json").write_text(json.dumps(case) + "\n")
    print("config_c32768_v4096", {k: v for k, v in case.items() if k != "ranking"}, flush=True)


def repeat_cases(ballots_case) -> None:
    """Ballots that name a candidate more than once. The reference counts every ordered pair of
    such a ballot (py:46-48), diagonal included, and completes it only when its length differs
    from C (py:75): a repeat of length C keeps its absent ids absent, a shorter or longer one
    gets them appended."""
    # Hand-made: the three cases of the completion rule, a ballot of one id, runs of one id.
    hand = [[0, 1, 0, 1], [2, 2, 1], [3, 3, 3, 3], [0, 0], [4, 0, 4, 1, 4, 2, 4, 3, 4], [1], [4, 3, 2, 1, 0],
            [2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2], [0, 1, 2, 3, 4]]
    ballots_case("repeats_c5_v9", [np.array(r) for r in hand])
    # Random: lengths 1 .. 2C, ids drawn with replacement, beside permutation ballots of the
    # same election (complete and incomplete) so that both kinds share 32-voter chunks.
    rng = np.random.default_rng(17)
    C = 37
    mixed = []
    for v in range(150):
        kind = v % 3
        if kind == 0:
            mixed.append(rng.integers(0, C, size=rng.integers(1, 2 * C + 1)))
        elif kind == 1:
            mixed.append(rng.permutation(C)[: rng.integers(1, C + 1)])
        else:
            r = rng.permutation(C)
            r[rng.integers(0, C)] = r[rng.integers(0, C)]  # length C, one id possibly twice
            mixed.append(r)
    mixed.append(np.arange(C))
    ballots_case("repeats_c37_v151", mixed)
    # Long ballots past the 2048-candidate limit of the shared-memory place rows' first kernel
    # (one CTA per ballot): permutations with a few repeats, some of length C, some shorter.
    rng = np.random.default_rng(18)
    C = 2500
    long_b = []
    for v in range(40):
        r = rng.permutation(C)
        if v % 4 == 1:
            r[rng.integers(0, C, size=3)] = r[0]
        elif v % 4 == 2:
            r = r[: rng.integers(C // 2, C)]
            r[-1] = r[1]
        elif v % 4 == 3:
            r = np.concatenate([r, r[:5]])
        long_b.append(r)
    ballots_case("repeats_c2500_v40", long_b, store_full=False, store_input=False)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("SE_REFERENCE_DIR"),
                    help="directory holding scaling_elections.py (default: $SE_REFERENCE_DIR)")
    ap.add_argument("--configs", action="store_true", help="(re)generate only the configuration-size cases")
    ap.add_argument("--only", nargs="*", help="with --configs: these cases only")
    ap.add_argument("--large", action="store_true",
                    help="the C = 32768 case (tally in parallel slices, the reference's OpenMP closure), "
                         "after checking that closure against the stored Numba hash at C = 16384")
    ap.add_argument("--workers", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--repeats", action="store_true",
                    help="(re)generate only the cases whose ballots repeat candidate ids")
    args = ap.parse_args()
    if not args.ref:
        ap.error("pass --ref or set SE_REFERENCE_DIR to the reference checkout")
    ref = load_reference(Path(args.ref))
    sys.path.insert(0, str(HERE.parent.parent))
    if args.large:
        large_cases(ref, Path(args.ref), args.workers)
        return
    if args.configs:
        config_cases(ref, args.only)
        return
    from scalingelections_b200.ballots import mallows_ballots, random_preferences, uniform_ballots

    index = json.loads((HERE / "index.json").read_text()) if args.repeats else {}

    def closure_case(name: str, P: np.ndarray, extra: dict | None = None, store_full: bool = True,
                     store_input: bool = True):
        P = np.ascontiguousarray(P, dtype=np.uint32)
        S = ref.compute_strongest_paths_numba_serial(P)
        C = P.shape[0]
        if C % 16 == 0 and C >= 16:
            S_tiled = ref.compute_strongest_paths_numba_parallel(P, tile_size=16)
            assert np.array_equal(S, S_tiled), name
        winner, ranking = ref.get_winner_and_ranking(list(range(C)), S)
        data = dict(ranking=np.asarray(ranking, np.int32), winner=np.int32(winner), strongest_sha256=np.array(sha(S)))
        if store_input:
            data["preferences"] = P
        if store_full:
            data["strongest"] = S
        if extra:
            data.update(extra)
        np.savez_compressed(HERE / f"{name}.npz", **data)
        index[name] = dict(C=int(C), winner=int(winner), strongest_sha256=sha(S), full=store_full)

    def ballots_case(name: str, rankings, store_full: bool = True, store_input: bool = True):
        d = ref.build_pairwise_preferences(rankings)
        ids, offs = csr(rankings)
        closure_case(name, d, dict(ids=ids, offsets=offs, tally_sha256=np.array(sha(d))), store_full, store_input)
        index[name]["V"] = int(len(rankings))
        index[name]["tally_sha256"] = sha(d)

    if args.repeats:
        repeat_cases(ballots_case)
        (HERE / "index.json").write_text(json.dumps(index, indent=1, sort_keys=True) + "\n")
        return

    # Participation paradox (validate_paradox.py:26-28): candidates Python, Rust, Go, Java.
    base = ([[0, 3, 1, 2]] + [[0, 3, 2, 1]] * 2 + [[1, 0, 2, 3]] * 2 + [[2, 3, 1, 0]] * 4 + [[3, 0, 1, 2]])
    ballots_case("paradox_before", [np.array(r) for r in base])
    ballots_case("paradox_after", [np.array(r) for r in base + [[3, 0, 2, 1]]])

    # The reference's default single election: C=128, V=2000 uniform permutations.
    ballots_case("uniform_c128_v2000", list(uniform_ballots(2000, 128, seed=1)))
    # Uneven sizes around the 128-cell tile, and tiny ones.
    for C, V, seed in [(1, 3, 2), (2, 5, 3), (3, 7, 4), (37, 101, 5), (129, 64, 6), (200, 333, 7)]:
        ballots_case(f"uniform_c{C}_v{V}", list(uniform_ballots(V, C, seed=seed)))
    # Mallows ballots (near-ties) at a size with several pivot rounds.
    ballots_case("mallows_c300_v500_phi08", list(mallows_ballots(500, 300, 0.8, seed=8)))
    # Incomplete ballots: random prefixes of random permutations (completion rule py:75-83).
    rng = np.random.default_rng(9)
    inc = []
    for _ in range(150):
        perm = rng.permutation(40)
        inc.append(perm[: rng.integers(1, 41)])
    inc.append(np.arange(40))  # makes sure max id + 1 == 40
    ballots_case("incomplete_c40_v151", inc)
    # Random preference matrices, the reference's --num-voters 0 mode (py:474-476), including
    # tiny value ranges that force ties and values beyond 16 bits.
    for C, high, seed in [(5, 2, 10), (64, 4, 11), (100, None, 12), (256, None, 13), (77, 2**32 - 1, 14),
                          (130, 70000, 15)]:
        closure_case(f"random_c{C}_hi{high if high else C}", random_preferences(C, seed, high))
    # A larger case kept as a hash only.
    ballots_case("uniform_c512_v600", list(uniform_ballots(600, 512, seed=16)), store_full=False)

    (HERE / "index.json").write_text(json.dumps(index, indent=1, sort_keys=True) + "\n")
    print(json.dumps(index, indent=1))


if __name__ == "__main__":
    main()
