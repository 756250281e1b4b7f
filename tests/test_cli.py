"""The command-line harness: the unmodified reference script run against the drop-in module
(CPU parts only here: its serial Numba closure picks the winner), and the report helpers
against the reference's own (scaling_elections.py:299-317)."""
import os
import runpy
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from scalingelections_b200 import cli

ROOT = Path(__file__).resolve().parent.parent
REF = Path(os.environ.get("SE_REFERENCE_DIR", "")) / "scaling_elections.py"
needs_ref = pytest.mark.skipif(not os.environ.get("SE_REFERENCE_DIR") or not REF.exists(),
                               reason="reference script not present (set SE_REFERENCE_DIR)")


def reference_namespace():
    from scalingelections_b200.dropin import scaling_elections as dropin

    saved = sys.modules.get("scaling_elections")
    sys.modules["scaling_elections"] = dropin
    try:
        return runpy.run_path(str(REF), run_name="reference_script")
    finally:
        if saved is None:
            sys.modules.pop("scaling_elections", None)
        else:
            sys.modules["scaling_elections"] = saved


@needs_ref
def test_report_helpers_match_reference():
    ns = reference_namespace()
    for t in (0.0004, 0.5, 0.999, 1.0, 12.345, 3600.0):
        assert cli.format_time(t) == ns["format_time"](t)
    for x in (12.0, 999.0, 1e3, 5.5e6, 1e9, 2.25e12, 7.7e14):
        assert cli.format_throughput(x) == ns["format_throughput"](x)


def test_drop_option():
    assert cli._drop_option(["--seed", "3", "--a", "--seed=4", "x"], "--seed") == ["--a", "x"]


def test_parser_accepts_reference_flags():
    args = cli.parser().parse_args(["--num-voters", "10", "--num-candidates", "64", "--run-cpu", "--run-gpu",
                                    "--no-serial", "--cpu-tile-size", "16", "--gpu-tile-size", "32",
                                    "--warmup", "2", "--repeat", "3"])
    assert (args.num_voters, args.num_candidates, args.warmup, args.repeat) == (10, 64, 2, 3)


def winner_line(out: str) -> str:
    return [ln for ln in out.splitlines() if "Winner: Candidate #" in ln][0]


@needs_ref
def test_unmodified_reference_script_through_the_harness(orc):
    """The reference's own CLI runs with the drop-in bound (no GPU here: its serial Numba closure
    runs and picks the winner). The seeded input is NumPy's global stream, so the oracle on the
    same seeded ballots names the same winner, and two runs agree."""
    C, V, seed = 24, 60, 11
    cmd = [sys.executable, "-m", "scalingelections_b200.cli", "--reference-script", str(REF),
           "--num-candidates", str(C), "--num-voters", str(V), "--seed", str(seed)]
    env = dict(os.environ, PYTHONPATH=str(ROOT), CUDA_VISIBLE_DEVICES="")
    runs = [subprocess.run(cmd, capture_output=True, text=True, env=env, cwd=ROOT, timeout=600) for _ in range(2)]
    for r in runs:
        assert r.returncode == 0, r.stderr[-2000:]
        assert "=== Schulze Voting Algorithm (Python) ===" in r.stdout
    assert winner_line(runs[0].stdout) == winner_line(runs[1].stdout)
    np.random.seed(seed)
    rankings = [np.random.permutation(C) for _ in range(V)]
    S = orc.strongest_paths(orc.tally(rankings), "serial")
    winner, _ = orc.winner_and_ranking(S)
    assert winner_line(runs[0].stdout).strip() == f"Winner: Candidate #{winner}"
