"""The package's own command line on the GPU: same seeded input as the reference script, the
same winner as the oracle, and the lane-mode cross-check passing."""
import numpy as np
import pytest

from scalingelections_b200 import cli

pytestmark = pytest.mark.gpu


def lines_with(out, key):
    return [ln.strip() for ln in out.splitlines() if key in ln]


@pytest.mark.parametrize("C,V", [(300, 0), (257, 120)])
def test_cli_winner_matches_oracle(capsys, orc, C, V):
    seed = 5
    assert cli.main(["--num-candidates", str(C), "--num-voters", str(V), "--run-gpu", "--seed", str(seed),
                     "--repeat", "2"]) == 0
    out = capsys.readouterr().out
    assert lines_with(out, "Results validated"), out
    np.random.seed(seed)
    if V == 0:
        P = np.random.randint(0, C, (C, C)).astype(np.uint32)
    else:
        P = orc.tally([np.random.permutation(C) for _ in range(V)])
    S = orc.strongest_paths(P, "blocked", tile=32)
    winner, ranking = orc.winner_and_ranking(S)
    assert lines_with(out, "Winner:") == [f"Winner: Candidate #{winner}"]
    assert lines_with(out, "Top 5:") == ["Top 5:  " + ", ".join(f"#{r}" for r in ranking[:5])]


def test_cli_no_serial_and_cpu_flag(capsys):
    assert cli.main(["--num-candidates", "64", "--run-gpu", "--run-cpu", "--no-serial", "--seed", "1"]) == 0
    out = capsys.readouterr().out
    assert "no CPU implementation" in out and "Cross-check" not in out and "Winner: Candidate #" in out


def test_cli_device_ballots(capsys):
    assert cli.main(["--num-candidates", "2048", "--num-voters", "4096", "--device-ballots", "--run-gpu",
                     "--no-serial", "--seed", "2"]) == 0
    assert "Winner: Candidate #" in capsys.readouterr().out
