"""bench.py's reference arm (``--impl reference``) runs on host cores only, so its JSON line
can be checked without a GPU: the line carries the contract's keys (impl, cpu_baseline, an e2e
object with no copies), and under several ranks only rank 0 prints it."""
import json
import os
import subprocess
import sys

from conftest import ROOT

SMALL = ["--impl", "reference", "--steps", "1", "--warmup", "0", "--cpu-sample", "256"]


def run_bench(args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], capture_output=True, text=True,
                          timeout=600, env=e, cwd=ROOT)


def test_reference_arm_prints_one_contract_line():
    r = run_bench(SMALL)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["unit"] == "Gcells/s" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 0 and d["n_gpus"] == 1
    assert d["config"]["candidates"] == 16384  # the workload it stands in for
    cpu = d["cpu_baseline"]
    assert cpu["kind"] in ("reference", "port") and cpu["cores"] >= 1 and cpu["value"] == d["value"]
    assert "C=256" in cpu["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "Gcells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["gpu_launches"] == 0


def test_reference_arm_prints_nothing_on_other_ranks():
    r = run_bench(SMALL, env={"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr
    assert not r.stdout.strip()


def test_gpus_flag_launches_one_rank_per_gpu():
    """--gpus N outside torchrun re-launches bench.py under torch.distributed.run with N
    ranks; on this host (no GPU) the launch check joins them with gloo."""
    r = run_bench(["--gpus", "2", "--workload", "launch-check"], env={"CUDA_VISIBLE_DEVICES": ""})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert sorted(d["rank"] for d in lines) == [0, 1]
    assert all(d["world_size"] == 2 and d["ranks_seen"] == 2 for d in lines)
