#!/usr/bin/env python
"""Benchmark of the Schulze widest-path closure on B200 (the headline workload).

Workload: one election with C = 16384 candidates and V = 4096 voters whose ballots are drawn
from a Mallows model (dispersion 0.8) around a seeded reference order. Ballots are drawn on
the GPU, tallied on the GPU, and the tally stays in HBM. A "step" is one full widest-path
closure of that C x C matrix (u16 lanes, legal because every count is at most V < 65536).

  value  C^3 relaxations per second ("cells/s", the reference's metric,
         scaling_elections.py:499), device-resident input and output, max over ranks.
  e2e    the same metric through the public host API compute_strongest_paths(): the
         preference matrix starts in pinned host memory and the strongest-path matrix returns
         to pinned host memory every step (1 GiB each way).

The matrix (0.5 GiB in u16, 1 GiB in u32) is larger than the 126 MB L2, so no flush is
needed between steps. ``--impl reference`` times the reference's own CPU closure (its OpenMP
path compiled unmodified into oracle/_ref) on a bounded sample of the same workload.

Multi-GPU (torchrun): every rank closes its own independent election (elections are the
unit of parallelism; there is no collective on the data path), so scaling is weak.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

def metric_name(C: int) -> str:
    return f"Gcells/s (C^3/t), single-election widest-path closure, C={C}"
UNIT = "Gcells/s"
# se_rank places up to this many candidates from per-CTA histograms of the wins, larger C by
# counting over strips (kHistMaxC in csrc/rank.cu).
RANK_HIST_MAX_C = 49152


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--candidates", type=int, default=16384)
    ap.add_argument("--voters", type=int, default=4096)
    ap.add_argument("--phi", type=float, default=0.8)
    ap.add_argument("--input", choices=["mallows", "random"], default="mallows",
                    help="closure input: tallied Mallows ballots, or the reference's random matrix mode")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--lanes", type=int, default=16, choices=[0, 16, 32])
    ap.add_argument("--closure-mode", type=int, default=0, choices=[0, 1, 2, 3, 4, 5, 6, 7, 8],
                    help="the closure's schedule: 0 automatic by size (default), 1 round by round, 2 dataflow, "
                         "3 wide panels, 4 wide panels and pivot launches, 5 two streams, 6 one launch per round, "
                         "7 every tile wide, 8 one launch per round, wide (include/se.h)")
    ap.add_argument("--workspace", choices=["full", "plain"], default="full",
                    help="closure workspace of the headline step: full (every schedule at its fastest, the "
                         "default) or plain (se_closure_workspace_bytes: no second pivot-panel buffer and no "
                         "split tiles)")
    ap.add_argument("--cpu-sample", type=int, default=4096, help="C of the bounded CPU sample")
    ap.add_argument("--cpu-full-size", action="store_true",
                    help="reference arm: also time one closure at the workload's full size (minutes)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["closure", "batch", "serve", "ingest", "sharded", "reference-gpu",
                                           "launch-check"],
                    default="closure",
                    help="closure: the headline single election; batch: many mixed elections; "
                         "serve: Poisson arrivals on the continuous-batching server")
    ap.add_argument("--requests", type=int, default=200, help="serve: requests per offered load")
    ap.add_argument("--loads", default="0.3,0.6,0.9", help="serve: offered loads as fractions of capacity")
    ap.add_argument("--budget-gb", type=float, default=40.0, help="serve: HBM admission budget")
    ap.add_argument("--serve-priority", choices=["arrival", "largest"], default="arrival",
                    help="serve: admission order of requests waiting together")
    ap.add_argument("--serve-ballots", choices=["host", "device"], default="host",
                    help="serve: ballots wait in pinned host memory (copied on admission) or on the device")
    ap.add_argument("--tight-budget-gb", type=float, default=4.0,
                    help="serve: budget of the extra load point where admission binds (0: skip it)")
    ap.add_argument("--no-extras", action="store_true",
                    help="closure: only the headline (skip the other configurations' objects)")
    ap.add_argument("--no-batch", action="store_true", help="closure: skip the batch object")
    ap.add_argument("--no-serve", action="store_true", help="closure: skip the serve object")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="closure: skip timing the reference's own CUDA path on the headline matrix")
    ap.add_argument("--sharded-candidates", type=int, default=32768,
                    help="closure under torchrun: C of the one election closed by all ranks together")
    ap.add_argument("--elections", type=int, default=4096, help="batch: number of elections")
    ap.add_argument("--max-candidates", type=int, default=2048, help="batch: largest C")
    ap.add_argument("--no-autotune", action="store_true", help="batch: skip the autotuner (use defaults)")
    ap.add_argument("--ingest-voters", type=int, default=1 << 20, help="ingest: ballots in the file")
    ap.add_argument("--ingest-candidates", type=int, default=1024, help="ingest: candidates")
    ap.add_argument("--ingest-chunk", type=int, default=1 << 16, help="ingest: ballots per streamed chunk")
    return ap.parse_args()


def config(args, world):
    return {
        "workload": (f"Schulze widest-path closure, one election per GPU: C={args.candidates} candidates, "
                     f"V={args.voters} Mallows(phi={args.phi}) ballots" if args.input == "mallows" else
                     f"Schulze widest-path closure, one election per GPU: C={args.candidates} candidates, "
                     f"random preference matrix (values uniform in [0, C), the reference's benchmark mode)"),
        "input": args.input,
        "candidates": args.candidates,
        "voters": args.voters,
        "phi": args.phi,
        "lanes": f"u{args.lanes}" if args.lanes else "auto",
        "closure_mode": {0: "automatic by size", 1: "round by round", 2: "dataflow", 3: "wide panels",
                         4: "wide panels and pivots", 5: "two streams", 6: "one launch per round",
                         7: "wide tiles", 8: "one wide launch per round"}[args.closure_mode],
        "tile": 128,
        "parallelism": f"replicas{world}" if world > 1 else "single",
        "l2": "inputs larger than L2 (0.5 GiB u16 working matrix), no flush",
    }


# ------------------------------------------------------------------------------------------
# Clock sampling during the timed region
# ------------------------------------------------------------------------------------------
class ClockSampler:
    """SM clocks and throttle reasons during a timed region: one `nvidia-smi -lms 200` process
    for the whole region (a single NVML start-up, which happens before the region opens: entry
    waits, bounded, for the first sample), its lines read by a thread, the process ended on
    exit."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples: list[list[str]] = []
        self._first = threading.Event()
        self._proc = None
        self._thr = None

    def _read(self):
        for line in self._proc.stdout:
            parts = [x.strip() for x in line.strip().split(",")]
            if len(parts) >= 8:
                self.samples.append(parts)
                self._first.set()
        self._first.set()  # the process ended (no GPU, or terminated): nothing more to wait for

    def __enter__(self):
        try:
            self._proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                           "--format=csv,noheader,nounits", "-lms", "200"],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self._proc = None
            return self
        self._thr = threading.Thread(target=self._read, daemon=True)
        self._thr.start()
        self._first.wait(10.0)
        return self

    def __exit__(self, *exc):
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()
                self._proc.wait(timeout=5)
        if self._thr is not None:
            self._thr.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 4 + i and s[4 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ------------------------------------------------------------------------------------------
# CPU baselines (the reference's own OpenMP closure, else the oracle's port)
# ------------------------------------------------------------------------------------------
def cpu_sample_matrix(args, C=None):
    """Preference matrix of the bounded CPU sample: a Mallows election with C = args.cpu_sample
    candidates and the headline's V and phi, drawn and tallied on the host (not timed)."""
    from oracle import oracle

    b = oracle.mallows_ballots(args.voters, C or args.cpu_sample, args.phi, seed=args.seed + 7)
    return oracle.tally(b, "positions")


def cpu_closure_sample(args, d):
    """Times the reference's CPU closure (its OpenMP path compiled unmodified into oracle/_ref;
    the oracle's port if that is absent) on the sample matrix d. Returns
    (cells_per_s, kind, cores, sample description, seconds)."""
    from oracle import oracle

    Cs = d.shape[0]
    cores = os.cpu_count() or 1
    ref = oracle.reference_cpu()
    if ref is not None:
        kind = "reference"
        ref.compute_strongest_paths(d[:256, :256].copy(), allow_gpu=False, allow_tma=False, tile_size=16)
        t0 = time.perf_counter()
        ref.compute_strongest_paths(d, allow_gpu=False, allow_tma=False, tile_size=16)
        t = time.perf_counter() - t0
        what = "scaling_elections.cu OpenMP closure (tile 16), compiled unmodified"
    else:
        kind = "port"
        t0 = time.perf_counter()
        oracle.strongest_paths(d, "blocked", tile=16, threads=cores)
        t = time.perf_counter() - t0
        what = "oracle blocked closure (tile 16, OpenMP)"
    sample = (f"{what}, one C={Cs}, V={args.voters} Mallows(phi={args.phi}) election ({Cs}^3 cells, {t:.2f} s) "
              f"standing in for the C={args.candidates} workload; {cores} host threads")
    return Cs ** 3 / t, kind, cores, sample, t


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    cfg = config(args, world)
    d = cpu_sample_matrix(args)
    values = []
    for i in range(args.warmup + args.steps):
        cps, kind, cores, sample, t = cpu_closure_sample(args, d)
        if i >= args.warmup:
            values.append(cps)
    v = statistics.median(values) / 1e9
    full = None
    if args.cpu_full_size:
        # One closure at the workload's own size, to check the per-cell rate of the sample.
        d_full = cpu_sample_matrix(args, C=args.candidates)
        cps_full, kind_f, cores_f, sample_f, t_full = cpu_closure_sample(args, d_full)
        full = {"value": cps_full / 1e9, "unit": UNIT, "seconds": t_full, "candidates": args.candidates,
                "sample": sample_f, "ratio_to_sample": cps_full / 1e9 / v}
    line = {
        "metric": metric_name(args.candidates), "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": args.cpu_sample ** 3 / (v * 1e9) * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded Mallows ballots)", "config": cfg,
        "impl": "reference",
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    if full is not None:
        line["full_size_point"] = full
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------
# Our arm
# ------------------------------------------------------------------------------------------
def main_launches(R: int, mode: int) -> dict:
    """What se_closure_profiled's phase_ms[3] times under schedule `mode`: the kernel, its
    launches, and the tile products they run (each 128^3 relaxations; the fused pivot's closure
    is extra and not counted). Schedule 6 runs R - 1 round launches of (R-1)^2 remainder tiles
    plus the next round's 2(R-1) panel tiles, then one plain remainder launch; the others run R
    remainder launches of (R-1)^2 tiles (schedule 5: the whole closure, remainder and panels).
    Schedules 7 and 8 run the kernels of 1 and 6 on the wide micro-tile."""
    if mode in (6, 8):
        per = (R - 1) ** 2 + 2 * (R - 1)
        return {"kernel": "round_kernel" + (" (wide micro-tile)" if mode == 8 else ""), "launches": R,
                "tiles_per_launch": per, "tiles": (R - 1) * per + (R - 1) ** 2}
    if mode == 5:
        return {"kernel": "rem_kernel and panels_kernel (two streams)", "launches": R,
                "tiles_per_launch": (R - 1) ** 2 + 2 * (R - 1), "tiles": R * ((R - 1) ** 2 + 2 * (R - 1))}
    return {"kernel": "rem_kernel" + (" (wide micro-tile)" if mode == 7 else ""), "launches": R,
            "tiles_per_launch": (R - 1) ** 2, "tiles": R * (R - 1) ** 2}


def load_traffic(lanes: int, C: int, kernel: str):
    """DRAM bytes (read + write) per launch of `kernel`, from the committed ncu summary of a
    smaller case, scaled to this C by the tiles per launch (the kernel's traffic is
    proportional to the tiles it processes)."""
    import re

    name = {"rem_kernel": "closure_rem_kernel_u16_c12288.md", "round_kernel": "closure_round_kernel_u16_c12288.md"}
    if kernel not in name:
        return None
    p = ROOT / "profiles" / name[kernel]
    if not p.exists():
        return None
    m = re.search(r"traffic_bytes_per_launch: u(\d+) C=(\d+) (\d+)", p.read_text())
    if not m or int(m.group(1)) != lanes:
        return None
    C_ref, b_ref = int(m.group(2)), int(m.group(3))
    R = lambda c: (c + 127) // 128  # noqa: E731
    tiles = (lambda c: (R(c) - 1) ** 2) if kernel == "rem_kernel" else (lambda c: (R(c) - 1) ** 2 + 2 * (R(c) - 1))
    return b_ref * tiles(C) / tiles(C_ref)


def measured_hbm_gbs() -> tuple[float, str]:
    """HBM copy bandwidth of this GPU model: the measured figure when MEASURED_PEAKS.json is
    present, else an earlier measurement on the same B200 pool."""
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        v = float(json.loads(p.read_text())["hbm_gbs"])
        return v, "measured: MEASURED_PEAKS.json hbm_gbs (STREAM-style copy)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback: 6.65 TB/s copy measured earlier on this GPU model"


def run_ours(args, world, rank, local_rank):
    import numpy as np
    import torch
    import torch.distributed as dist

    from scalingelections_b200 import _lib, api
    from scalingelections_b200.ballots import mallows_ballots_device

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    C, V = args.candidates, args.voters
    lanes = args.lanes
    L = _lib.lib()

    # Input: ballots drawn and tallied on the device, or the reference's random benchmark matrix
    # (values uniform in [0, C), scaling_elections.py:473-476) drawn on the device.
    if args.input == "random":
        from scalingelections_b200.ballots import random_preferences_device

        d = random_preferences_device(C, seed=args.seed + 1000 * rank, device=dev)
    else:
        ballots = mallows_ballots_device(V, C, args.phi, seed=args.seed + 1000 * rank, device=dev)
        offs = torch.arange(V + 1, dtype=torch.int64, device=dev) * C
        d = api.tally_device(ballots.view(-1), offs, C)
    torch.cuda.synchronize()

    # Roofline denominator: the min/max issue microbenchmark at this moment's clock.
    peak = [ctypes.c_double() for _ in range(4)]
    recipe = 3 if lanes in (0, 16) else 1
    _lib.check(L.se_minmax_peak(recipe, 65536, *[ctypes.byref(x) for x in peak]))
    peak_relax_per_clk, peak_mhz, _, peak_relax_per_s = [x.value for x in peak]

    api.set_closure_mode(args.closure_mode)
    need = api.closure_workspace_bytes(C, lanes, dataflow=args.workspace == "full")
    work = torch.empty(need, dtype=torch.uint8, device=dev)
    out = torch.empty((C, C), dtype=torch.uint32, device=dev)
    stream = torch.cuda.current_stream()

    def step():
        api.strongest_paths_device(d, lanes=lanes, out=out, workspace=work)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    cells = float(C) ** 3 * args.steps * world
    value = cells / (ms_max * 1e-3) / 1e9

    # Per-phase device time (one extra, event-instrumented closure) for the roofline.
    phase = (ctypes.c_double * 4)()
    launches = ctypes.c_int(0)
    _lib.check(L.se_closure_profiled(d.data_ptr(), C, C, out.data_ptr(), C, lanes, 0, work.data_ptr(), need,
                                     stream.cuda_stream, phase, ctypes.byref(launches)))
    R = (C + 127) // 128
    schedule = api.closure_schedule(C, lanes or 16, need)
    main = main_launches(R, schedule)
    tile_ms_avg = phase[3] / max(main["launches"], 1)
    achieved = float(main["tiles"]) * 128 ** 3 / (phase[3] * 1e-3)
    cell_bytes = 2 if lanes in (0, 16) else 4
    algo_bytes = float(main["tiles_per_launch"]) * 128 * 128 * cell_bytes * 2  # each tile read + written once

    # The reference's own CUDA path on the same matrix (regenerated from the same seed), in a
    # process of its own: run inside this one after its other legs, the same call once took 66 s
    # instead of 8.5 s, and the OpenMP sample after it ten times its usual time.
    reference_gpu = None
    if world == 1 and rank == 0 and not args.no_extras and not args.no_reference_gpu:
        reference_gpu = child_line(["--workload", "reference-gpu", "--candidates", str(C), "--voters", str(V),
                                    "--phi", str(args.phi), "--seed", str(args.seed), "--input", args.input,
                                    "--lanes", str(lanes)])

    # The tally half of the path on the same ballots (device-resident), against the integer
    # ALU pipe: B lop3 + 1 popc + 1 add per 32 voter pairs of the upper block triangle
    # (B = bits of C - 1).
    tally = None
    if args.input == "mallows":
        tw = torch.empty(api.tally_workspace_bytes(V, C), dtype=torch.uint8, device=dev)
        d2 = torch.empty_like(d)
        for _ in range(2):
            api.tally_device(ballots.view(-1), offs, C, out=d2, workspace=tw)
        t0e, t1e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0e.record(stream)
        for _ in range(3):
            api.tally_device(ballots.view(-1), offs, C, out=d2, workspace=tw)
        t1e.record(stream)
        torch.cuda.synchronize()
        tally_s = t0e.elapsed_time(t1e) / 3e3
        Rt = (C + 127) // 128
        executed = Rt * (Rt + 1) / 2 * 128 * 128 * V
        alu_peak = tally_alu_peak(torch.cuda.get_device_properties(dev).multi_processor_count, peak_mhz, C)
        tally = {"ms": tally_s * 1e3, "voters": V, "pairs_per_s": V * C * (C - 1) / 2 / tally_s,
                 "roofline": {"bound": "int_alu", "achieved": executed / tally_s / 1e12, "peak": alu_peak / 1e12,
                              "unit": "Tpairs/s", "frac": executed / tally_s / alu_peak,
                              "peak_source": TALLY_PEAK_SOURCE},
                 "same_as_input": bool(torch.equal(d2.view(torch.int32), d.view(torch.int32)))}
        del tw, d2, ballots

    # Ranking (se_rank: wins + stable places) of the closure's u32 output, which is larger
    # than L2: algorithmic bytes = the C x C u32 matrix read once.
    wins_t = torch.empty(C, dtype=torch.int32, device=dev)
    rank_t = torch.empty(C, dtype=torch.int32, device=dev)

    def rank_once():
        _lib.check(L.se_rank(out.data_ptr(), C, C, wins_t.data_ptr(), rank_t.data_ptr(), stream.cuda_stream))

    for _ in range(2):
        rank_once()
    r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    r0.record(stream)
    for _ in range(5):
        rank_once()
    r1.record(stream)
    torch.cuda.synchronize()
    rank_s = r0.elapsed_time(r1) / 5e3
    hbm_peak, hbm_source = measured_hbm_gbs()
    rank_bytes = float(C) * C * 4
    place = "place_hist_kernel" if C <= RANK_HIST_MAX_C else "place_kernel"
    ranking = {"ms": rank_s * 1e3, "kernels": ["wins_kernel", place],
               "roofline": {"bound": "hbm", "achieved": rank_bytes / rank_s / 1e9, "peak": hbm_peak, "unit": "GB/s",
                            "frac": rank_bytes / rank_s / 1e9 / hbm_peak, "algorithmic_bytes": rank_bytes,
                            "peak_source": hbm_source},
               "winner": int(rank_t[0].item())}

    # End to end through the public host API: pinned host in, pinned host out.
    e2e = None
    e2e_numpy = None
    if not args.no_e2e:
        host_in = torch.empty((C, C), dtype=torch.int32, pin_memory=True)
        host_in.copy_(d.view(torch.int32))
        host_in = host_in.view(torch.uint32)
        api.compute_strongest_paths(host_in, allow_gpu=True, tile_size=32, lanes=lanes)  # warm
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            res = api.compute_strongest_paths(host_in, allow_gpu=True, tile_size=32, lanes=lanes)
            del res
        t_e2e = time.perf_counter() - t0
        te = torch.tensor([t_e2e], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        e2e = {"value": cells / float(te.item()) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": C * C * 4, "d2h_bytes_per_step": C * C * 4}
        if world == 1 and not args.no_extras:
            # The call as the reference's script makes it: a pageable NumPy matrix in (staged
            # through pinned chunks), a new NumPy matrix out.
            np_in = host_in.numpy().copy()
            api.compute_strongest_paths(np_in, allow_gpu=True, tile_size=32, lanes=lanes)  # warm
            n_np = max(1, min(args.steps, 5))
            t0 = time.perf_counter()
            for _ in range(n_np):
                res = api.compute_strongest_paths(np_in, allow_gpu=True, tile_size=32, lanes=lanes)
                del res
            t_np = time.perf_counter() - t0
            e2e_numpy = {"value": float(C) ** 3 * n_np / t_np / 1e9, "unit": UNIT, "steps": n_np,
                         "ms_per_step": t_np / n_np * 1e3,
                         "input": "pageable NumPy uint32 matrix (the reference script's call)"}
            del np_in

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # The reference arm itself, one sample, in a process of its own (see reference_gpu).
        ref = child_line(["--impl", "reference", "--steps", "1", "--warmup", "0", "--cpu-sample",
                          str(args.cpu_sample), "--candidates", str(C), "--voters", str(V), "--phi", str(args.phi),
                          "--seed", str(args.seed)])
        cpu = ref.get("cpu_baseline", {"unavailable": ref.get("unavailable", "no line")})

    extras = {}
    if world == 1 and not args.no_extras:
        extras = run_extras(args, local_rank, d, out, host_in if e2e is not None else None, peak_mhz)
    elif world > 1 and not args.no_extras:
        del work
        torch.cuda.empty_cache()
        extras["sharded"] = measure_sharded(args, world, rank, local_rank, C=args.sharded_candidates)

    if rank == 0:
        traffic = load_traffic(lanes if lanes else 16, C, main["kernel"])
        line = {
            "metric": metric_name(args.candidates), "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": f"u{lanes}" if lanes else "u16/u32",
            "data": ("synthetic (seeded Mallows ballots drawn and tallied on the GPU)" if args.input == "mallows"
                     else "synthetic (seeded random matrix drawn on the GPU)"),
            "config": config(args, world),
            "roofline": {
                "bound": "int_minmax",
                "kernel": f"{main['kernel']}<u{lanes or 16}> (closure schedule {schedule})",
                "achieved": achieved / 1e12, "peak": peak_relax_per_s / 1e12, "unit": "Trelax/s",
                "frac": achieved / peak_relax_per_s,
                "peak_source": f"measured: se_minmax_peak recipe {recipe} in this run "
                               f"({peak_relax_per_clk:.1f} relax/SM/clk at {peak_mhz:.0f} MHz)",
                "traffic": traffic,
                "algorithmic_bytes_per_launch": algo_bytes,
                "hbm_gbs_achieved": algo_bytes / (tile_ms_avg * 1e-3) / 1e9,
                "phase_ms": {"pivot_round0": phase[0], "panels": phase[1], "main_launches": phase[3]},
                "main_launches": main,
            },
            "cpu_baseline": cpu,
            "e2e": e2e,
            "tally": tally,
            "ranking": ranking,
            "clocks": clocks.summary(),
            "gpu_launches": int(L.se_closure_launch_count(C)) * args.steps,
        }
        line.update(extras)
        if e2e_numpy is not None:
            line["e2e_numpy"] = e2e_numpy
        if reference_gpu is not None:
            line["reference_gpu"] = reference_gpu
        print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------
# The other configurations, as objects of the headline line (one GPU)
# ------------------------------------------------------------------------------------------
def closure_object(d, lanes: int, steps: int, warmup: int, local_rank: int, workload: str) -> dict:
    """Device-timed closure of the resident matrix d in the given lanes, with the remainder
    kernel's roofline against the min/max peak measured now (u16x2 or u32 recipe)."""
    import torch

    from scalingelections_b200 import _lib, api

    L = _lib.lib()
    C = int(d.shape[0])
    dev = d.device
    peak = [ctypes.c_double() for _ in range(4)]
    recipe = 3 if lanes == 16 else 1
    _lib.check(L.se_minmax_peak(recipe, 65536, *[ctypes.byref(x) for x in peak]))
    peak_relax_per_s = peak[3].value
    need = api.closure_workspace_bytes(C, lanes, dataflow=True)
    work = torch.empty(need, dtype=torch.uint8, device=dev)
    out = torch.empty((C, C), dtype=torch.uint32, device=dev)
    stream = torch.cuda.current_stream()
    # Closures of a few milliseconds are queued back to back through the stream-ordered entry
    # point, each with its own workspace (its error word is checked after the timed region), so
    # the host's return between synchronous calls does not show as device idle time.
    queued = C <= 8192
    works = [torch.empty(need, dtype=torch.uint8, device=dev) for _ in range(steps)] if queued else []
    for _ in range(warmup):
        api.strongest_paths_device(d, lanes=lanes, out=out, workspace=work)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        torch.cuda.synchronize()
        e0.record(stream)
        for i in range(steps):
            if queued:
                api.strongest_paths_enqueue(d, lanes=lanes, out=out, workspace=works[i])
            else:
                api.strongest_paths_device(d, lanes=lanes, out=out, workspace=work)
        e1.record(stream)
        torch.cuda.synchronize()
    for w in works:
        api.closure_check(w)
    del works
    ms = e0.elapsed_time(e1) / steps
    phase = (ctypes.c_double * 4)()
    launches = ctypes.c_int(0)
    _lib.check(L.se_closure_profiled(d.data_ptr(), C, C, out.data_ptr(), C, lanes, 0, work.data_ptr(), need,
                                     stream.cuda_stream, phase, ctypes.byref(launches)))
    R = (C + 127) // 128
    schedule = api.closure_schedule(C, lanes, need)
    obj = {"workload": workload, "candidates": C, "lanes": f"u{lanes}", "tile": 128, "schedule": schedule,
           "steps": steps, "warmup": warmup, "ms": ms, "value": float(C) ** 3 / (ms * 1e-3) / 1e9, "unit": UNIT,
           "phase_ms": {"pivot_round0": phase[0], "panels": phase[1], "main_launches": phase[3]},
           "gpu_launches": int(launches.value) * steps, "clocks": clocks.summary()}
    if R > 1:
        main = main_launches(R, schedule)
        achieved = float(main["tiles"]) * 128 ** 3 / (phase[3] * 1e-3)
        obj["roofline"] = {"bound": "int_minmax", "kernel": f"{main['kernel']}<u{lanes}>",
                           "achieved": achieved / 1e12, "peak": peak_relax_per_s / 1e12, "unit": "Trelax/s",
                           "frac": achieved / peak_relax_per_s,
                           "peak_source": f"measured: se_minmax_peak recipe {recipe} in this run"}
        obj["whole_closure_frac_of_peak"] = float(C) ** 3 / (ms * 1e-3) / peak_relax_per_s
    return obj, out


def election_matrix(V: int, C: int, phi: float, seed: int, dev):
    """Ballots drawn (Mallows; phi = 1 is uniform permutations) and tallied on the device."""
    import torch

    from scalingelections_b200 import api
    from scalingelections_b200.ballots import mallows_ballots_device

    b = mallows_ballots_device(V, C, phi, seed=seed, device=dev)
    offs = torch.arange(V + 1, dtype=torch.int64, device=dev) * C
    d = api.tally_device(b.view(-1), offs, C)
    return d, b, offs


def child_line(argv: list[str]) -> dict:
    """Runs this script with `argv` in a new process on the same GPU (this one waits, idle) and
    returns the JSON object of its last line."""
    env = dict(os.environ)
    for k in ("RANK", "LOCAL_RANK", "WORLD_SIZE", "LOCAL_WORLD_SIZE", "GROUP_RANK", "ROLE_RANK"):
        env.pop(k, None)
    r = subprocess.run([sys.executable, str(Path(__file__).resolve()), *argv], capture_output=True, text=True,
                       env=env, timeout=1800)
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    if r.returncode != 0 or not lines:
        return {"unavailable": f"child exited {r.returncode}: {r.stderr.strip().splitlines()[-1:] if r.stderr else ''}"}
    return json.loads(lines[-1])


def reference_gpu_leg(d_host, ours_host, local_rank: int) -> dict:
    """Baseline leg: the reference's own CUDA path (scaling_elections.cu compiled unmodified for
    sm_100a into oracle/_ref/gpu) on the same matrix, through its own host API, timed by wall
    clock around the call as the reference times it (scaling_elections.py:338-357): host init,
    managed-memory migration, kernels and the copy back."""
    from oracle import oracle

    mod = oracle.reference_gpu()
    C = int(d_host.shape[0])
    if mod is None:
        return {"unavailable": "oracle/_ref/gpu not built (the reference's sources were absent at build time)"}
    small = d_host[:256, :256].copy()
    mod.compute_strongest_paths(small, allow_gpu=True, allow_tma=False, tile_size=32)  # CUDA init, kernels loaded
    with ClockSampler(local_rank) as clocks:
        t0 = time.perf_counter()
        res = mod.compute_strongest_paths(d_host, allow_gpu=True, allow_tma=False, tile_size=32)
        t = time.perf_counter() - t0
    import numpy as np

    return {"impl": "scaling_elections.cu compute_strongest_paths(allow_gpu=True, allow_tma=False, tile_size=32), "
                    "the reference's CUDA path compiled unmodified for sm_100a",
            "candidates": C, "seconds": t, "value": float(C) ** 3 / t / 1e9, "unit": UNIT, "timing": "wall clock, "
            "one call (the reference's own convention: host init, managed memory, kernels, copy back)",
            "bit_identical_to_ours": bool(np.array_equal(res, ours_host)), "clocks": clocks.summary()}


def run_reference_gpu(args, local_rank):
    """The reference's own CUDA path alone on the headline matrix (for a launch list of its
    kernels under ncu), beside this library's closure of the same matrix."""
    import torch

    from scalingelections_b200 import api

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if args.input == "random":
        from scalingelections_b200.ballots import random_preferences_device

        d = random_preferences_device(args.candidates, seed=args.seed, device=dev)
    else:
        d, b, o = election_matrix(args.voters, args.candidates, args.phi, args.seed, dev)
        del b, o
    ours = api._to_host_u32(api.strongest_paths_device(d, lanes=args.lanes or 16))
    line = reference_gpu_leg(api._to_host_u32(d), ours, local_rank)
    line["workload"] = f"C={args.candidates}, V={args.voters} Mallows(phi={args.phi}) ballots"
    print(json.dumps(line), flush=True)


def run_extras(args, local_rank, d, out, host_in, peak_mhz) -> dict:
    """The objects of the other configurations, added to the headline line: e2e_pipelined (the
    headline through api.ClosureStream), u32 (the headline in 32-bit lanes), c4096 (single
    election, C = V = 4096 uniform ballots), c32768 (C = 32768, V = 4096 Mallows(0.8)), batch
    (4096 mixed elections), serve (Poisson arrivals)."""
    import numpy as np
    import torch

    from scalingelections_b200 import LANES_U16, api

    dev = d.device
    C = int(d.shape[0])
    steps = max(1, args.steps)
    ex = {}
    if host_in is not None:
        cs = api.ClosureStream(C, lanes=LANES_U16)
        for _ in cs.map([host_in] * 3):  # warm: every slot and stream used once
            pass
        with ClockSampler(local_rank) as clocks:
            t0 = time.perf_counter()
            n = 0
            for res in cs.map([host_in] * steps):
                n += 1
                del res
            t = time.perf_counter() - t0
        ex["e2e_pipelined"] = {
            "value": float(C) ** 3 * n / t / 1e9, "unit": UNIT, "steps": n, "ms_per_step": t / n * 1e3,
            "h2d_bytes_per_step": C * C * 4, "d2h_bytes_per_step": C * C * 4,
            "api": "scalingelections_b200.ClosureStream.map over pinned host matrices (se_closure_enqueue: each "
                   "step's copy in and copy out overlap the neighbouring steps' closures)",
            "clocks": clocks.summary()}
        del cs
    obj, out32 = closure_object(d, 32, max(2, min(steps, 3)), 1, local_rank,
                                f"the headline election (C={C}) in 32-bit lanes")
    obj["bit_identical_to_u16"] = bool(torch.equal(out32.view(torch.int32), out.view(torch.int32)))
    ex["u32"] = obj
    del out32
    torch.cuda.empty_cache()

    # cfg2: C = V = 4096, uniform permutations (Mallows with phi = 1).
    d4, b4, o4 = election_matrix(4096, 4096, 1.0, args.seed + 4096, dev)
    del b4, o4
    obj16, o16 = closure_object(d4, 16, max(steps, 20), 3, local_rank,
                                "single election, C=4096, V=4096 uniform permutation ballots")
    obj32, o32 = closure_object(d4, 32, max(steps, 10), 2, local_rank, "the same election in 32-bit lanes")
    obj16["u32"] = obj32
    obj16["u32"]["bit_identical_to_u16"] = bool(torch.equal(o16.view(torch.int32), o32.view(torch.int32)))
    # The schedule sweep of this configuration: the 128-cell tile with the default micro-tile
    # (8 x 8 words per thread) for every tile, or the wide one (8 x 4 words, twice the warps) for
    # the panels, or for the panels and a pivot launch per round; two streams; or each round's
    # remainder and the next round's panels in one launch.
    sweep = {}
    for mode, what in ((1, "panels and pivot on 8x8 words, pivot fused"), (3, "panels on 8x4 words, pivot fused"),
                       (4, "panels and pivot on 8x4 words, pivot launched"), (5, "as 3 on two streams"),
                       (6, "remainder and next panels in one launch per round"),
                       (7, "every tile on 8x4 words, pivot fused"),
                       (8, "as 6 with every tile on 8x4 words")):
        api.set_closure_mode(mode)
        o, _ = closure_object(d4, 16, max(steps, 20), 3, local_rank, what)
        sweep[str(mode)] = {"schedule": what, "ms": o["ms"], "value": o["value"],
                            "frac_of_peak": o.get("whole_closure_frac_of_peak")}
    api.set_closure_mode(0)
    obj16["schedule_sweep"] = sweep
    obj16["tile_note"] = "tile 128 x 128 cells; micro-tile 8 x 8 or 8 x 4 words per thread (schedule_sweep)"
    ex["c4096"] = obj16
    del d4, o16, o32

    # cfg3's larger size: C = 32768, V = 4096 Mallows(0.8).
    d32, b32, o32 = election_matrix(4096, 32768, 0.8, args.seed + 32768, dev)
    tw = torch.empty(api.tally_workspace_bytes(4096, 32768), dtype=torch.uint8, device=dev)
    api.tally_device(b32.view(-1), o32, 32768, out=torch.empty_like(d32), workspace=tw)
    te0, te1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    te0.record()
    api.tally_device(b32.view(-1), o32, 32768, out=torch.empty_like(d32), workspace=tw)
    te1.record()
    torch.cuda.synchronize()
    del b32, o32, tw
    obj, S32 = closure_object(d32, 16, 2, 1, local_rank, "single election, C=32768, V=4096 Mallows(phi=0.8) ballots")
    obj["tally_ms"] = te0.elapsed_time(te1)
    wins, ranking = api.rank_device(S32)
    obj["winner"] = int(ranking[0].item())
    re0, re1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    re0.record()
    for _ in range(3):  # the 4 GiB matrix is far larger than L2
        api.rank_device(S32)
    re1.record()
    torch.cuda.synchronize()
    obj["ranking_ms"] = re0.elapsed_time(re1) / 3
    ex["c32768"] = obj
    del d32, S32, wins, ranking
    torch.cuda.empty_cache()

    if not args.no_batch:
        line = measure_batch(args, 1, 0, local_rank)
        ex["batch"] = {k: line[k] for k in ("metric", "value", "unit", "ms_per_step", "loop_elections_per_s",
                                             "speedup_vs_loop", "bit_identical_to_loop", "batched_gcells_per_s",
                                             "config", "autotune", "clocks") if k in line}
        ex["batch"]["steps"] = line["steps"]
        torch.cuda.empty_cache()
    if not args.no_serve:
        line = measure_serve(args, 1, 0, local_rank)
        ex["serve"] = {k: line[k] for k in ("metric", "value", "unit", "config", "data", "saturation", "loads",
                                             "tight_budget", "clocks") if k in line}
        ex["serve"]["saturation"].pop("engine_profile", None)
        torch.cuda.empty_cache()
    return ex


# ------------------------------------------------------------------------------------------
# Batched workload: many independent elections of uneven size
# ------------------------------------------------------------------------------------------
def batch_specs(n: int, seed: int, c_max: int = 2048):
    """C log-uniform in [8, c_max], V uniform in [50, 100000], the first half uniform ballots
    and the second half Mallows with phi uniform in [0.2, 1.0]; seeded."""
    import numpy as np

    rng = np.random.default_rng(seed)
    C = np.rint(np.exp(rng.uniform(np.log(8), np.log(c_max), size=n))).astype(int)
    V = rng.integers(50, 100001, size=n)
    phi = np.where(np.arange(n) < n // 2, 1.0, rng.uniform(0.2, 1.0, size=n))
    return [(int(C[e]), int(V[e]), float(phi[e]), seed * 1_000_003 + e) for e in range(n)]


def make_batch_inputs(specs, dev):
    """Ballots drawn and tallied on the GPU one election at a time; only the C x C tallies are
    kept (the ballots of the largest elections are 0.8 GB each)."""
    import torch

    from scalingelections_b200 import api
    from scalingelections_b200.ballots import mallows_ballots_device

    prefs = []
    for (C, V, phi, sd) in specs:
        b = mallows_ballots_device(V, C, phi, seed=sd, device=dev)
        offs = torch.arange(V + 1, dtype=torch.int64, device=dev) * C
        prefs.append(api.tally_device(b.view(-1), offs, C))
        del b, offs
    torch.cuda.synchronize()
    return prefs


def run_batch(args, world, rank, local_rank):
    line = measure_batch(args, world, rank, local_rank)
    if rank == 0:
        print(json.dumps(line), flush=True)


def measure_batch(args, world, rank, local_rank):
    """cfg4: a batch of elections of uneven size closed and ranked by one persistent launch
    (CUDA graph), against a loop of the single-election path over the same batch. Returns the
    JSON object (rank 0's view)."""
    import torch
    import torch.distributed as dist

    from scalingelections_b200 import api
    from scalingelections_b200.batch import BatchedElections, lanes_for_voters

    from scalingelections_b200.shard import election_cost, partition_by_work

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    # One global batch of elections x world, split by closure work; no collective on the
    # data path (weak scaling: the global batch grows with the number of GPUs).
    all_specs = batch_specs(args.elections * world, args.seed, args.max_candidates)
    mine = partition_by_work([election_cost(C) for (C, _, _, _) in all_specs], world)[rank]
    specs = [all_specs[i] for i in mine]
    t0 = time.perf_counter()
    prefs = make_batch_inputs(specs, dev)
    prep_s = time.perf_counter() - t0
    tuned = None
    tune_s = 0.0
    if args.no_autotune:
        lanes, order, ctas = [lanes_for_voters(V) for (_, V, _, _) in specs], 0, 0
        micro = None
    else:
        from scalingelections_b200 import autotune

        t0 = time.perf_counter()
        report_dir = os.environ.get("SE_REPORT_DIR")  # where to keep the tuning table, if anywhere
        tuned = autotune.tune(V=100000, per_bucket=32, reps=3,
                              path=Path(report_dir) / "autotune.json" if report_dir else None)
        tune_s = time.perf_counter() - t0
        lanes, order, ctas = autotune.choose(tuned, [C for (C, _, _, _) in specs], [V for (_, V, _, _) in specs])
        micro = autotune.choose_micro_tiles(tuned, [C for (C, _, _, _) in specs], lanes)
    cells = float(sum(C ** 3 for (C, _, _, _) in all_specs))
    b = BatchedElections(prefs, lanes, order=order, ctas_per_sm=ctas, micro_tiles=micro)
    b.build_graph()
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        b.launch_graph()
    b.check()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            b.launch_graph()
        e1.record(stream)
        torch.cuda.synchronize()
    b.check()
    ms = e0.elapsed_time(e1) / args.steps
    # One more run, timed alone, for the engine profile (the counters reset every run).
    pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pe0.record(stream)
    b.launch_graph()
    pe1.record(stream)
    torch.cuda.synchronize()
    prof = b.profile()
    prof["run_ms"] = pe0.elapsed_time(pe1)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())

    # The same batch through the plain single-election entry points, one election at a time,
    # checked bit for bit against the batched results.
    ws = torch.empty(max(api.closure_workspace_bytes(C, 0, dataflow=True) for (C, _, _, _) in specs),
                     dtype=torch.uint8, device=dev)
    outs = [torch.empty_like(p) for p in prefs]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ranks = []
    for p, o in zip(prefs, outs):
        api.strongest_paths_device(p, lanes=0, out=o, workspace=ws)
        ranks.append(api.rank_device(o)[1])
    torch.cuda.synchronize()
    loop_s = time.perf_counter() - t0
    identical = all(torch.equal(o.view(torch.int32), bo.view(torch.int32)) and torch.equal(r, br)
                    for o, bo, r, br in zip(outs, b.outs, ranks, b.rankings))

    n_total = len(all_specs)
    value = n_total / (ms_max * 1e-3)
    line = None
    if rank == 0:
        tasks = b.task_counts()
        line = {
            "metric": "elections/s, batched closure + ranking of mixed-size elections", "value": value,
            "unit": "elections/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u16/u32 per election", "data": "synthetic (seeded uniform and Mallows ballots, GPU-tallied)",
            "config": {"workload": f"{args.elections} elections per GPU, C log-uniform [8, {args.max_candidates}], "
                                   "V uniform [50, 100000], half uniform / half Mallows(phi~U[0.2,1])",
                       "u16_elections": sum(1 for l in lanes if l[0] == 16),
                       "u16_shifted_elections": sum(1 for l in lanes if l[0] == 16 and l[1] > 0),
                       "u32_elections": sum(1 for l in lanes if l[0] == 32),
                       "tasks": {"u16": tasks[0], "u32": tasks[1], "u16_wide_micro_tile": tasks[2]},
                       "graph": True},
            "batched_gcells_per_s": cells / (ms_max * 1e-3) / 1e9,
            "loop_elections_per_s": len(specs) / loop_s,
            "loop_seconds": loop_s,
            "speedup_vs_loop": (len(specs) / (ms * 1e-3)) / (len(specs) / loop_s),
            "bit_identical_to_loop": identical,
            "input_prep_seconds": prep_s,
            "engine_profile": prof,
            "autotune": None if tuned is None else {
                "seconds": tune_s, "order": order, "ctas_per_sm": ctas,
                "launch_ms": tuned.get("launch_ms"),
                "buckets": {k: {"C": v["range"], "lanes": v["lanes"], "micro_tile": v.get("micro_tile", 8),
                                "ms": v["ms"]} for k, v in tuned["buckets"].items()}},
            "clocks": clocks.summary(),
        }
    del b, prefs, outs, ranks, ws
    torch.cuda.empty_cache()
    return line


# ------------------------------------------------------------------------------------------
# Serving workload: Poisson arrivals on the continuous-batching server
# ------------------------------------------------------------------------------------------
def serve_specs(n: int, seed: int):
    """C log-uniform in [8, 8192], V log-uniform in [100, 100000], Mallows phi ~ U[0.2, 1]."""
    import numpy as np

    rng = np.random.default_rng(seed)
    C = np.rint(np.exp(rng.uniform(np.log(8), np.log(8192), size=n))).astype(int)
    V = np.rint(np.exp(rng.uniform(np.log(100), np.log(100000), size=n))).astype(int)
    phi = rng.uniform(0.2, 1.0, size=n)
    return [(int(V[i]), int(C[i]), float(phi[i]), seed * 7_000_003 + i) for i in range(n)]


def run_serve(args, world, rank, local_rank):
    line = measure_serve(args, world, rank, local_rank)
    if rank == 0:
        print(json.dumps(line), flush=True)


def measure_serve(args, world, rank, local_rank):
    """cfg5: saturation throughput, then p50/p99 latency under Poisson arrivals at the offered
    loads, then one load under a budget small enough that admission binds. Ballots wait in
    pinned host memory and are copied to the GPU when their request is admitted, inside its
    latency window (--serve-ballots device keeps them resident instead). Returns the JSON
    object (rank 0's view)."""
    import numpy as np
    import torch

    from scalingelections_b200.ballots import mallows_ballots_device
    from scalingelections_b200.serve import Server, run_arrivals, summarize

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    specs = serve_specs(args.requests, args.seed + 104729 * rank)
    host = args.serve_ballots == "host"
    t0 = time.perf_counter()
    reqs = []
    for (V, C, phi, sd) in specs:
        b = mallows_ballots_device(V, C, phi, seed=sd, device=dev)
        if host:
            h = torch.empty((V, C), dtype=torch.int32, pin_memory=True)
            h.copy_(b)
            b = h
        reqs.append((V, C, b))
    torch.cuda.synchronize()
    prep_s = time.perf_counter() - t0
    ballot_bytes = sum(4 * V * C for (V, C, _, _) in specs)
    server = Server(budget_bytes=int(args.budget_gb * (1 << 30)), max_slots=1024, ctas_per_sm=2, idle_ms=5,
                    priority=args.serve_priority)
    # Warm-up, then capacity: every request arrives at once (closed loop, admission-bound).
    run_arrivals(server, reqs[: min(8, len(reqs))], [0.0] * min(8, len(reqs)))
    p0 = server.stats(profile=True)
    done, makespan = run_arrivals(server, reqs, [0.0] * len(reqs))
    capacity = len(done) / makespan
    sat = summarize(done, float("inf"), makespan)
    p1 = server.stats(profile=True)
    sat_launches = p1["engine_launches"] - p0["engine_launches"]
    sat_profile = {
        "busy_cta_ms": {k: p1["busy_cta_ms"][k] - p0["busy_cta_ms"][k] for k in p1["busy_cta_ms"]},
        "tasks": {k: p1["tasks"][k] - p0["tasks"][k] for k in p1["tasks"]},
        "search_cta_ms": p1["search_cta_ms"] - p0["search_cta_ms"],
        "grid_cta_ms": p1["grid"] * makespan * 1e3,
        "host": dict(getattr(server, "last_host_stats", {})),
    }
    rng = np.random.default_rng(args.seed + 17)
    loads = []
    with ClockSampler(local_rank) as clocks:
        for frac in [float(x) for x in args.loads.split(",")]:
            rate = frac * capacity
            gaps = rng.exponential(1.0 / rate, size=len(reqs))
            arrivals = list(np.cumsum(gaps) - gaps[0])
            l0 = server.stats()["engine_launches"]
            done, span = run_arrivals(server, reqs, arrivals)
            r = summarize(done, rate, span)
            loads.append({"offered_fraction": frac, "offered_per_s": rate, "achieved_per_s": r.achieved_rate,
                          "p50_ms": r.p50_ms, "p99_ms": r.p99_ms, "mean_ms": r.mean_ms, "n": r.n,
                          "engine_launches": server.stats()["engine_launches"] - l0})
    grid = server.stats()["grid"]
    server.close()
    del server
    torch.cuda.empty_cache()
    # Admission binding: the middle load again under a budget that holds the largest request
    # but only a few at a time, so requests wait on the host for memory.
    tight = None
    if args.tight_budget_gb > 0:
        frac = [float(x) for x in args.loads.split(",")][len(loads) // 2]
        rate = frac * capacity
        gaps = rng.exponential(1.0 / rate, size=len(reqs))
        arrivals = list(np.cumsum(gaps) - gaps[0])
        with ClockSampler(local_rank) as tclocks:
            with Server(budget_bytes=int(args.tight_budget_gb * (1 << 30)), max_slots=1024, ctas_per_sm=2,
                        idle_ms=5, priority=args.serve_priority) as ts:
                done, span = run_arrivals(ts, reqs, arrivals)
                launches = ts.stats()["engine_launches"]
        r = summarize(done, rate, span)
        waited = [t.admitted - t.arrival for t in done]
        tight = {"budget_gb": args.tight_budget_gb, "offered_fraction": frac, "offered_per_s": rate,
                 "achieved_per_s": r.achieved_rate, "p50_ms": r.p50_ms, "p99_ms": r.p99_ms, "mean_ms": r.mean_ms,
                 "n": r.n, "engine_launches": launches,
                 "admission_wait_ms": {"p50": float(np.percentile(waited, 50)) * 1e3,
                                       "p99": float(np.percentile(waited, 99)) * 1e3},
                 "clocks": tclocks.summary()}
    line = None
    if rank == 0:
        V = np.array([s[0] for s in specs], float)
        C = np.array([s[1] for s in specs], float)
        line = {
            "metric": "served elections/s at saturation, and p50/p99 latency under Poisson load",
            "value": capacity * world, "unit": "elections/s", "n_gpus": world, "steps": len(loads),
            "warmup": 1, "ms_per_step": makespan * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u16 (shifted lanes above 65535 ballots)",
            "data": ("synthetic (seeded Mallows ballots in pinned host memory, copied to the GPU on admission, "
                     "inside the latency window)" if host else
                     "synthetic (seeded Mallows ballots resident on the GPU before arrival)"),
            "config": {"workload": f"{args.requests} requests, C log-uniform [8, 8192], V log-uniform [100, 100000], "
                                   f"Mallows phi ~ U[0.2, 1]; HBM budget {args.budget_gb:g} GB",
                       "ballots": "host (pinned)" if host else "device", "ballot_bytes_total": ballot_bytes,
                       "tally_pairs_total": float((V * C * C / 2).sum()), "closure_cells_total": float((C ** 3).sum()),
                       "admission_priority": args.serve_priority},
            "saturation": {"p50_ms": sat.p50_ms, "p99_ms": sat.p99_ms, "makespan_s": makespan,
                           "engine_launches": sat_launches, "grid": grid,
                           "engine_profile": sat_profile},
            "loads": loads,
            "tight_budget": tight,
            "input_prep_seconds": prep_s,
            "clocks": clocks.summary(),
        }
    del reqs
    torch.cuda.empty_cache()
    return line


TALLY_PEAK_SOURCE = ("SMs x 64 integer ALU lanes x SM clock x 32 / (B + 2): per 32 voter pairs, B lop3 "
                     "(one per bit plane, B = bits of C - 1) plus one popc and one add")


def tally_alu_peak(sms: int, mhz: float, C: int) -> float:
    """Voter pairs per second the bit-sliced counting kernel can reach on the integer ALU pipe."""
    B = max(1, (C - 1).bit_length())
    return sms * 64 * mhz * 1e6 * 32 / (B + 2)


def run_sharded(args, world, rank, local_rank):
    line = measure_sharded(args, world, rank, local_rank)
    if rank == 0:
        print(json.dumps(line), flush=True)


def measure_sharded(args, world, rank, local_rank, C=None):
    """One election closed by all ranks together (scalingelections_b200.sharded): row blocks
    split across the ranks, one pivot-row panel broadcast (NCCL) per round. Every rank draws
    and tallies the same ballots, so all hold the same preference matrix. Strong scaling: the
    work is one C^3 closure whatever the number of GPUs. Returns rank 0's JSON object."""
    import torch
    import torch.distributed as dist

    from scalingelections_b200 import LANES_U16, api
    from scalingelections_b200.ballots import mallows_ballots_device
    from scalingelections_b200.sharded import strongest_paths_sharded

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    C, V = (C or args.candidates), args.voters
    own_group = world == 1 and not dist.is_initialized()
    if own_group:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        if "MASTER_PORT" not in os.environ:
            import socket

            with socket.socket() as sk:
                sk.bind(("127.0.0.1", 0))
                os.environ["MASTER_PORT"] = str(sk.getsockname()[1])
        dist.init_process_group("nccl", rank=0, world_size=1)
    ballots = mallows_ballots_device(V, C, args.phi, seed=args.seed, device=dev)
    offs = torch.arange(V + 1, dtype=torch.int64, device=dev) * C
    d = api.tally_device(ballots.view(-1), offs, C)
    del ballots
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        rows, _ = strongest_paths_sharded(d, lanes=LANES_U16)
    torch.cuda.synchronize()
    dist.barrier()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            rows, (r0, r1) = strongest_paths_sharded(d, lanes=LANES_U16)
        e1.record(stream)
        torch.cuda.synchronize()
        dist.barrier()
    ms = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
    dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    ms_max = float(ms.item())
    # Check this rank's rows against the single-GPU closure of the same matrix.
    single = api.strongest_paths_device(d, lanes=LANES_U16)
    identical = torch.equal(rows.view(torch.int32), single[r0:r1].view(torch.int32))
    ok = torch.tensor([1 if identical else 0], device=dev)
    dist.all_reduce(ok, op=dist.ReduceOp.MIN)
    R = (C + 127) // 128
    line = None
    if rank == 0:
        line = {
            "metric": f"Gcells/s (C^3/t), one election's closure sharded over the GPUs, C={C}",
            "value": C ** 3 * args.steps / (ms_max / 1e3) / 1e9, "unit": "Gcells/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "u16", "data": "synthetic (seeded Mallows ballots)",
            "config": {"workload": f"one election, C={C}, V={V} Mallows(phi={args.phi}) ballots, row blocks split "
                                   f"over {world} GPU(s), one NCCL broadcast of the pivot-row panel per round",
                       "rounds": R, "panel_bytes": 128 * ((C + 127) // 128 * 128) * 2},
            "bit_identical_to_single_gpu": bool(ok.item()),
            "gpu_launches": (R * 2 + R * 2 * world) * args.steps,
            "clocks": clocks.summary(),
        }
    del d, rows, single
    torch.cuda.empty_cache()
    if own_group:
        dist.destroy_process_group()
    return line


def run_ingest(args, world, rank, local_rank):
    """Ballot file -> preference matrix: 2^20 incomplete ballots over C = 1024 candidates
    (lengths uniform in [1, C], Mallows(0.8) orders) in a packed file of 16-bit ids, tallied
    by streaming chunks through the GPU (ballot_file.tally_file). A step reads the file (from
    the page cache), copies it to the device and tallies it. Also timed: the tally kernels on
    the same ballots already in HBM (the roofline leg) and the C oracle's tally on a sample."""
    import tempfile

    import numpy as np
    import torch

    from scalingelections_b200 import _lib
    from scalingelections_b200 import ballot_file as bfm
    from scalingelections_b200.ballots import mallows_ballots_device

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    V, C, chunk = args.ingest_voters, args.ingest_candidates, args.ingest_chunk
    rng = np.random.default_rng(args.seed + rank)
    lens = rng.integers(1, C + 1, size=V).astype(np.int64)
    t0 = time.perf_counter()
    full = mallows_ballots_device(V, C, 0.8, seed=args.seed + 31 * rank, device=dev).to(torch.int16).cpu().numpy()
    mask = np.arange(C)[None, :] < lens[:, None]
    ids = full[mask]
    del full, mask
    offsets = np.zeros(V + 1, dtype=np.int64)
    np.cumsum(lens, out=offsets[1:])

    class _Csr:
        pass

    csr = _Csr()
    csr.ids, csr.offsets = ids, offsets
    tmp = tempfile.TemporaryDirectory(prefix="se_ingest_")
    path = os.path.join(tmp.name, "ballots.seb")
    bfm.write_ballots(path, csr, num_candidates=C)
    file_bytes = os.path.getsize(path)
    prep_s = time.perf_counter() - t0

    out = torch.zeros((C, C), dtype=torch.uint32, device=dev)
    for _ in range(args.warmup):
        bfm.tally_file(path, device=dev, chunk_ballots=chunk, out=out)
    torch.cuda.synchronize()
    stats = {}
    with ClockSampler(local_rank) as clocks:
        t1 = time.perf_counter()
        for _ in range(args.steps):
            bfm.tally_file(path, device=dev, chunk_ballots=chunk, out=out, stats=stats)
        torch.cuda.synchronize()
        e2e_s = (time.perf_counter() - t1) / args.steps
    file_result = out.view(torch.int32).cpu().numpy()

    # Kernel leg: the same ballots resident in HBM, one se_tally_ex over all of them.
    d_ids = torch.from_numpy(ids.view(np.int16)).to(dev)
    d_offs = torch.from_numpy(offsets).to(dev)
    L = _lib.lib()
    need = L.se_tally_workspace_bytes(V, C)
    work = torch.empty(need, dtype=torch.uint8, device=dev)
    d = torch.empty((C, C), dtype=torch.uint32, device=dev)
    stream = torch.cuda.current_stream()

    def tally_once():
        _lib.check(L.se_tally_ex(d_ids.data_ptr(), 2, d_offs.data_ptr(), 0, V, C, bfm.SE_TALLY_NO_SYNC, d.data_ptr(),
                                 C, work.data_ptr(), need, stream.cuda_stream))

    for _ in range(args.warmup):
        tally_once()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        tally_once()
    e1.record(stream)
    torch.cuda.synchronize()
    kernel_s = e0.elapsed_time(e1) / 1e3 / args.steps
    if int(work[:4].view(torch.int32).item()) != 0:
        raise RuntimeError("tally reported malformed ballots")
    identical = bool(np.array_equal(file_result, d.view(torch.int32).cpu().numpy()))

    # Roofline of the counting kernel (see tally_alu_peak); diagonal tiles count both halves.
    props = torch.cuda.get_device_properties(dev)
    sm_mhz = clocks.summary().get("sm_mhz") or 1965.0
    R = (C + 127) // 128
    executed_pairs = R * (R + 1) / 2 * 128 * 128 * V
    peak_pairs = tally_alu_peak(props.multi_processor_count, sm_mhz, C)
    pairs = V * C * (C - 1) / 2

    cpu = None
    if not args.no_cpu_baseline and rank == 0:
        from oracle import oracle

        n = 4000
        sample = [ids[offsets[v]:offsets[v + 1]].astype(np.int64) for v in range(n)] + [np.array([C - 1])]
        c0 = time.perf_counter()
        oracle.tally(sample, method="positions")
        cpu_s = time.perf_counter() - c0
        cpu = {"value": n / cpu_s, "unit": "ballots/s", "cores": 1, "kind": "port",
               "sample": f"{n} of the {V} ballots, C={C}, tallied by the C oracle (positions form, one thread)"}
    tmp.cleanup()
    if rank == 0:
        line = {
            "metric": "ballots/s, packed ballot file -> pairwise preference matrix (streamed GPU tally)",
            "value": V / e2e_s * world, "unit": "ballots/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": e2e_s * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32 (bit planes, integer counts)",
            "data": "synthetic (seeded Mallows(0.8) orders, truncated to uniform lengths)",
            "config": {"workload": f"ballot file ingest: V={V} incomplete ballots, C={C}, 16-bit ids, "
                                   f"{chunk} ballots per chunk", "file_bytes": file_bytes,
                       "chunks": stats.get("chunks"), "host_read_wait_s_per_step": stats.get("read_wait_s"),
                       "read_threads": stats.get("read_threads")},
            "file_gbs": file_bytes / e2e_s / 1e9,
            "kernel": {"ms": kernel_s * 1e3, "ballots_per_s": V / kernel_s, "pairs_per_s": pairs / kernel_s},
            "roofline": {"bound": "int_alu", "achieved": executed_pairs / kernel_s / 1e12,
                         "peak": peak_pairs / 1e12, "unit": "Tpairs/s", "frac": executed_pairs / kernel_s / peak_pairs,
                         "peak_source": TALLY_PEAK_SOURCE + f" ({props.multi_processor_count} SMs, {sm_mhz:.0f} MHz)",
                         "traffic": None},
            "file_equals_resident_tally": identical,
            "cpu_baseline": cpu,
            "input_prep_seconds": prep_s,
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)


def launch_ranks(n: int) -> int:
    """Runs this script once per GPU under torch.distributed.run (one node, rendezvous on
    127.0.0.1) with the same arguments, and returns its exit status. Used when --gpus N > 1 is
    given outside a torchrun launch. The ranks' process group times out a stuck collective after
    300 s; as the last bound, well above that, `timeout` ends the whole launch after 30 minutes
    (exit status 124)."""
    cmd = ["timeout", "-k", "60", "1800", sys.executable, "-m", "torch.distributed.run", "--standalone",
           "--local-addr", "127.0.0.1", "--nnodes", "1", "--nproc-per-node", str(n), str(Path(__file__).resolve()),
           *sys.argv[1:]]
    return subprocess.call(cmd)


def launch_check(world, rank):
    """Each rank joins the process group (NCCL with GPUs, else gloo), agrees on the world size
    with an all-reduce and prints one line; for testing the launcher without GPUs."""
    import datetime

    import torch
    import torch.distributed as dist

    backend = "nccl" if torch.cuda.is_available() else "gloo"
    if backend == "nccl":
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=60))
    t = torch.ones(1, device="cuda" if backend == "nccl" else "cpu")
    dist.all_reduce(t)
    # One write call per line: the ranks share stdout, and a short write to a pipe is atomic.
    line = json.dumps({"rank": rank, "world_size": world, "ranks_seen": int(t.item()), "backend": backend})
    os.write(1, (line + "\n").encode())
    dist.destroy_process_group()


def main():
    args = parse()
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        sys.exit(launch_ranks(args.gpus))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "launch-check":
        launch_check(world, rank)
        return
    if args.impl == "reference":
        run_reference_arm(args, world, rank)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        if args.workload == "batch":
            run_batch(args, world, rank, local_rank)
        elif args.workload == "serve":
            run_serve(args, world, rank, local_rank)
        elif args.workload == "ingest":
            run_ingest(args, world, rank, local_rank)
        elif args.workload == "sharded":
            run_sharded(args, world, rank, local_rank)
        elif args.workload == "reference-gpu":
            run_reference_gpu(args, local_rank)
        else:
            run_ours(args, world, rank, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
