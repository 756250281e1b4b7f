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
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


def ballots_of(case):
    """The CSR ballots of a golden case as a list of arrays (the reference's input shape)."""
    ids, offs = case["ids"], case["offsets"]
    return [ids[offs[v]:offs[v + 1]] for v in range(len(offs) - 1)]


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle

    oracle.lib()
    return oracle
