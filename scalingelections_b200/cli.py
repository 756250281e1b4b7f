"""Command-line benchmark of the Schulze path, with the reference script's flags and report.

Two modes:

``python -m scalingelections_b200.cli [flags]``
    This package's own driver. It takes the flags of the reference script's command line
    (scaling_elections.py:361-417) plus ``--seed``, ``--lanes`` and ``--device-ballots``,
    and prints the same report: configuration, one timed block per implementation, election
    results. Preferences are drawn exactly as the reference draws them (py:470-480:
    ``np.random.randint`` for a random matrix, ``np.random.permutation`` per voter) from
    NumPy's global generator seeded with ``--seed``. The same seed therefore gives the reference script
    the same matrix, and so the same strongest paths and winner. The driver also avoids two
    pitfalls of the reference's command line at large C:
      * the reference runs the serial Numba closure for the winner even under ``--no-serial``
        (py:546-552); here the winner always comes from the GPU result;
      * the reference ranks in a pure-Python C^2 loop (py:274-296); here the ranking runs on
        the GPU (``rank_device``).
    This package has no CPU closure, so ``--run-cpu`` reports that and the serial block is
    replaced by a cross-check: the GPU closure in both lane modes (packed 16-bit and 32-bit)
    must give the same matrix.

``python -m scalingelections_b200.cli --reference-script PATH [flags]``
    Runs the unmodified reference script as ``__main__`` with ``scaling_elections`` bound to
    this package's drop-in module. NumPy's global generator is seeded with ``--seed``
    first. The script's own flags pass through untouched; it then benchmarks the
    ``compute_strongest_paths`` of this package under its "Tiled GPU" labels and validates it
    against its own serial Numba closure.
"""
from __future__ import annotations

import argparse
import runpy
import sys
import time

import numpy as np


def format_time(elapsed_sec: float) -> str:
    """Milliseconds below a second, else seconds with two decimals (as scaling_elections.py:299-305)."""
    elapsed_ms = elapsed_sec * 1000
    return f"{int(elapsed_ms)} ms" if elapsed_ms < 1000 else f"{elapsed_sec:.2f} s"


def format_throughput(cells_per_sec: float) -> str:
    """T/G/M/K cells^3 per second with one decimal (as scaling_elections.py:308-317)."""
    for scale, unit in ((1e12, "T"), (1e9, "G"), (1e6, "M")):
        if cells_per_sec >= scale:
            return f"{cells_per_sec / scale:.1f} {unit}cells³/s"
    return f"{cells_per_sec / 1e3:.1f} Kcells³/s"


def parser() -> argparse.ArgumentParser:
    ap = argparse.ArgumentParser(description="Benchmark the Schulze method on B200")
    ap.add_argument("--num-voters", type=int, default=0,
                    help="ballots to draw and tally; 0 draws a random preference matrix instead")
    ap.add_argument("--num-candidates", type=int, default=256, help="candidates C (the matrix is C x C)")
    ap.add_argument("--run-cpu", action="store_true", help="accepted; this package has no CPU closure")
    ap.add_argument("--run-gpu", action="store_true", help="time the GPU closure")
    ap.add_argument("--no-serial", action="store_true", help="skip the 16-bit against 32-bit lane cross-check")
    ap.add_argument("--cpu-tile-size", type=int, default=16, help="accepted and ignored (no CPU closure here)")
    ap.add_argument("--gpu-tile-size", type=int, default=32,
                    help="checked against 4, 8, 16 and 32 like the reference's; the kernels use 128-cell tiles")
    ap.add_argument("--warmup", type=int, default=1, help="untimed runs before timing (default %(default)s)")
    ap.add_argument("--repeat", type=int, default=1, help="timed runs, averaged (default %(default)s)")
    ap.add_argument("--seed", type=int, default=None, help="seed NumPy's global generator, for a repeatable input")
    ap.add_argument("--lanes", choices=["auto", "16", "32"], default="auto", help="closure lanes: auto picks 16 bits whenever the counts fit")
    ap.add_argument("--device-ballots", action="store_true",
                    help="Draw the random matrix, or uniform ballots tallied in place, on the GPU "
                         "(fast at large V x C; not NumPy's stream)")
    ap.add_argument("--reference-script", default=None,
                    help="Run this unmodified scaling_elections.py against the drop-in module instead")
    return ap


def run_reference_script(path: str, seed: int | None, argv: list[str]) -> None:
    """Execute the reference script as __main__ with the drop-in bound as scaling_elections."""
    from .dropin import scaling_elections as dropin

    if seed is not None:
        np.random.seed(seed)
    saved_mod = sys.modules.get("scaling_elections")
    saved_argv = sys.argv
    sys.modules["scaling_elections"] = dropin
    sys.argv = [path] + argv
    try:
        runpy.run_path(path, run_name="__main__")
    finally:
        sys.argv = saved_argv
        if saved_mod is None:
            sys.modules.pop("scaling_elections", None)
        else:
            sys.modules["scaling_elections"] = saved_mod


def draw_preferences(num_candidates: int, num_voters: int, device_ballots: bool):
    """The reference's input (py:470-480) from NumPy's global generator, or GPU ballots."""
    import torch

    from . import api
    from .ballots import mallows_ballots_device

    C, V = num_candidates, num_voters
    if V == 0 and device_ballots:
        from .ballots import random_preferences_device

        return api._to_host_u32(random_preferences_device(C, seed=int(np.random.randint(0, 2**31 - 1))))
    if V == 0:
        return np.random.randint(0, C, (C, C)).astype(np.uint32)
    if device_ballots:
        seed = int(np.random.randint(0, 2**31 - 1))
        ballots = mallows_ballots_device(V, C, 1.0, seed=seed)
        ids = ballots.reshape(-1)
        offsets = torch.arange(V + 1, dtype=torch.int64, device=ids.device) * C
        return api._to_host_u32(api.tally_device(ids, offsets, C))
    rankings = [np.random.permutation(C) for _ in range(V)]
    return api.build_pairwise_preferences(rankings)


def bench(callback, preferences, warmup: int, repeat: int):
    """(average seconds, last result), with the reference's warm-up lines (py:320-356)."""
    for i in range(warmup):
        t0 = time.time()
        callback(preferences)
        dt = time.time() - t0
        print(f"  Warm-up {i + 1}/{warmup}: {format_time(dt)}" if warmup > 1 else f"  Warm-up: {format_time(dt)}")
    times, result = [], None
    for _ in range(max(1, repeat)):
        t0 = time.time()
        result = callback(preferences)
        times.append(time.time() - t0)
    return sum(times) / len(times), result


def main(argv: list[str] | None = None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    args, rest = parser().parse_known_args(argv)
    if args.reference_script:
        passthrough = _drop_option(_drop_option(argv, "--reference-script"), "--seed")
        run_reference_script(args.reference_script, args.seed, passthrough)
        return 0
    if rest:
        parser().error(f"unrecognized arguments: {' '.join(rest)}")

    from . import api
    from ._lib import LANES_AUTO, LANES_U16, LANES_U32

    C, V = args.num_candidates, args.num_voters
    if args.seed is not None:
        np.random.seed(args.seed)
    print("=== Schulze Voting Algorithm (B200) ===")
    print()
    try:
        api.log_gpus()
    except Exception as e:
        print(f"✗ Could not detect GPU: {e}")
    print("Configuration:")
    voters_str = f"{V:,}" if V > 0 else "random"
    print(f"  Problem size: {C:,} candidates × {voters_str} voters")
    if args.run_gpu:
        print(f"  GPU tile: {args.gpu_tile_size} × {args.gpu_tile_size} (kernels: 128 × 128)")
    print(f"  Lanes: {args.lanes}")
    print(f"  Seed: {args.seed if args.seed is not None else 'unseeded'}")
    print(f"  Warmup: {args.warmup}, Repeat: {args.repeat}")
    print()
    print("Generating preferences...")
    preferences = draw_preferences(C, V, args.device_ballots)
    print()
    print("─── Benchmarking ───────────────────────────────────")
    print()

    lanes = {"auto": LANES_AUTO, "16": LANES_U16, "32": LANES_U32}[args.lanes]

    def closure(lane_mode):
        def run(p):
            return api.compute_strongest_paths(p, allow_gpu=True, allow_tma=False, tile_size=args.gpu_tile_size,
                                               lanes=lane_mode)
        return run

    result = None
    if args.run_cpu:
        print("→ Tiled CPU")
        print("  ✗ Benchmark failed: this package has no CPU implementation")
        print()
    if args.run_gpu or not args.no_serial:
        print(f"→ Tiled GPU (B200, {args.lanes} lanes)")
        try:
            t, result = bench(closure(lanes), preferences, args.warmup, args.repeat)
            avg = f"{format_time(t)} (avg of {args.repeat})" if args.repeat > 1 else format_time(t)
            print(f"  Run:     {avg} │ {format_throughput(C ** 3 / t)}")
        except Exception as e:
            print(f"  ✗ Benchmark failed: {e}")
        print()
    if result is not None and not args.no_serial:
        other = LANES_U32 if lanes != LANES_U32 else LANES_U16
        name = "32-bit" if other == LANES_U32 else "16-bit"
        print(f"→ Cross-check (B200, {name} lanes)")
        try:
            check = closure(other)(preferences)
            same = np.array_equal(check, result)
            print("  ✓ Results validated" if same else "  ✗ Results don't match baseline!")
        except Exception as e:  # e.g. 16-bit lanes cannot hold these values
            print(f"  - Skipped: {e}")
        print()

    if result is None:
        result = api.compute_strongest_paths(preferences, allow_gpu=True, tile_size=args.gpu_tile_size, lanes=lanes)
    import torch

    paths = api._to_device_u32(result, torch.device("cuda", torch.cuda.current_device()))
    wins, ranking = api.rank_device(paths)
    ranking = ranking.cpu().tolist()
    print("─── Election Results ───────────────────────────────")
    print()
    print(f"  Winner: Candidate #{ranking[0]}")
    if len(ranking) >= 5:
        print(f"  Top 5:  #{ranking[0]}, #{ranking[1]}, #{ranking[2]}, #{ranking[3]}, #{ranking[4]}")
    print()
    return 0


def _drop_option(argv: list[str], name: str) -> list[str]:
    out, skip = [], False
    for a in argv:
        if skip:
            skip = False
            continue
        if a == name:
            skip = True
            continue
        if a.startswith(name + "="):
            continue
        out.append(a)
    return out


if __name__ == "__main__":
    sys.exit(main())
