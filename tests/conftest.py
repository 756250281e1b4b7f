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


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle

    oracle.lib()
    return oracle
