"""Generates the golden fixtures in this directory from the REFERENCE implementation.

Run where the reference sources are present (they are never copied into this repository):

    python tests/golden/make_golden.py [--ref /root/reference]

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
import sys
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


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--configs", action="store_true", help="(re)generate only the configuration-size cases")
    ap.add_argument("--only", nargs="*", help="with --configs: these cases only")
    args = ap.parse_args()
    ref = load_reference(Path(args.ref))
    sys.path.insert(0, str(HERE.parent.parent))
    if args.configs:
        config_cases(ref, args.only)
        return
    from scalingelections_b200.ballots import mallows_ballots, random_preferences, uniform_ballots

    index = {}

    def closure_case(name: str, P: np.ndarray, extra: dict | None = None, store_full: bool = True):
        P = np.ascontiguousarray(P, dtype=np.uint32)
        S = ref.compute_strongest_paths_numba_serial(P)
        C = P.shape[0]
        if C % 16 == 0 and C >= 16:
            S_tiled = ref.compute_strongest_paths_numba_parallel(P, tile_size=16)
            assert np.array_equal(S, S_tiled), name
        winner, ranking = ref.get_winner_and_ranking(list(range(C)), S)
        data = dict(preferences=P, ranking=np.asarray(ranking, np.int32), winner=np.int32(winner),
                    strongest_sha256=np.array(sha(S)))
        if store_full:
            data["strongest"] = S
        if extra:
            data.update(extra)
        np.savez_compressed(HERE / f"{name}.npz", **data)
        index[name] = dict(C=int(C), winner=int(winner), strongest_sha256=sha(S), full=store_full)

    def ballots_case(name: str, rankings, store_full: bool = True):
        d = ref.build_pairwise_preferences(rankings)
        ids, offs = csr(rankings)
        closure_case(name, d, dict(ids=ids, offsets=offs, tally_sha256=np.array(sha(d))), store_full)
        index[name]["V"] = int(len(rankings))
        index[name]["tally_sha256"] = sha(d)

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
