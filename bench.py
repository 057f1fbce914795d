"""Benchmark of the MD hot path on B200: timesteps/s (and ns/day, p50/p99)
of the charged LJ melt with PME.

Workload (one GPU): 262,144 ions on a 64^3 rock-salt lattice (spacing
2.82 A, box 180.48 A), charges +-1 e, positions jittered U(-0.2, 0.2) A
(seed 2027), LJ sigma 3.0 A / eps 0.5 kJ/mol, masses 23 / 35.45 amu,
real-space cutoff 12 A + 1 A skin, alpha = 0.256412 1/A (Ewald tolerance
1e-5), PME order 4 on 192^3, Nose-Hoover 1200 K (tau 100 fs), dt 2 fs, FP64.
One step = integrate, skin-gated neighbour rebuild, LJ + real-space
Coulomb, PME (spread, FFT, influence, inverse FFT, gather), integrate +
thermostat.  Synthetic seeded inputs; the per-step working set (~0.7 GB)
is far larger than the 126 MB L2.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With N > 1 (torchrun, one rank per GPU) every rank advances its own
replica of the system (the path does not shard one system); the value is
the sum over ranks, timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "timesteps/s and ns/day (1 B200) vs plain FP64 path at stated force error; p50/p99"
UNIT = "timesteps/s"
WORKLOAD = "charged LJ melt + PME: 262,144 ions (64^3 rock salt), 192^3 grid, order 4, NVT 1200 K, dt 2 fs"
DT_FS = 2.0


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def _traffic(kernel: str):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f).get(kernel)
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return None, 0, 1, 0
    import torch
    import torch.distributed as dist
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    import datetime
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return dist, rank, ws, local


def _barrier(dist, local):
    if dist is not None:
        import torch
        dist.barrier()
        torch.cuda.synchronize(local)


def _max_over_ranks(dist, local, v: float) -> float:
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def pairs_within(system, desc, rc: float):
    """Unordered pairs closer than rc at the system's current positions
    (periodic k-d tree count on the host, outside every timed region)."""
    try:
        from scipy.spatial import cKDTree
    except ImportError:
        return None
    out, _ = system.download(keys=("x", "y", "z"))
    L = np.asarray(desc["box"][:3], dtype=np.float64)
    pts = np.mod(np.stack([out["x"], out["y"], out["z"]], axis=1), L)
    tree = cKDTree(pts, boxsize=L)
    ordered = int(tree.count_neighbors(tree, rc))
    return (ordered - len(pts)) // 2


def cpu_baseline(budget_s: float = 20.0, max_steps: int = 5):
    """The oracle (the FP64 CPU restatement of the reference path) on all
    host cores: neighbour list + forces at setup, then timed MD steps until
    `budget_s` of CPU time or `max_steps`."""
    import oracle
    from atomiverse_b200 import workloads as W
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import oracle_system
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    desc, frame = W.rocksalt_melt()
    s = oracle_system(oracle, desc, frame)
    s.build_list()
    s.compute_forces()
    n = 0
    t0 = time.perf_counter()
    while n < max_steps and (time.perf_counter() - t0) < budget_s:
        s.run(1)
        n += 1
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{n} full MD steps of the benchmark workload after a "
                      f"setup list build + force pass ({dt:.1f} s, "
                      f"OMP_NUM_THREADS={cores})"}


def run_reference(args):
    dist, rank, ws, local = _dist()
    if rank != 0:
        return 0
    steps = max(1, min(args.steps, 5))
    cb = cpu_baseline(budget_s=60.0, max_steps=steps)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": steps, "warmup": 0,
            "ms_per_step": 1e3 / cb["value"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "precision": "fp64"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": "the reference CPU path cannot be built offline (FetchContent "
                    "deps, absent molrs submodule and FFTW3); its algorithm runs as "
                    "the repository's FP64 CPU restatement"}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    dist, rank, ws, local = _dist()
    import atomiverse_b200 as A
    from atomiverse_b200 import workloads as W

    ctx = A.Context(local)
    desc, frame = W.rocksalt_melt(precision=A.FP64)
    sys_ = A.System(ctx, desc, frame)
    sys_.compute_forces()
    sys_.step(args.warmup)
    sc0 = sys_.scalars()

    # ---- timed region: K steps, CUDA events on the system's stream
    clocks = ClockSampler(local)
    _barrier(dist, local)
    clocks.start()
    total_ms, per_step = sys_.step_timed(args.steps)
    clk = clocks.stop()
    _barrier(dist, local)
    launches = sys_.launch_count()
    t_max = _max_over_ranks(dist, local, total_ms)
    sc1 = sys_.scalars()
    value = ws * args.steps / (t_max * 1e-3)

    # ---- per-kernel device times: a profiled pass of the same K steps
    sys_.profile(True)
    sys_.step(args.steps)
    prof = sys_.profile_read()
    sys_.profile(False)
    pair_ms, pair_n = prof.get("pair", (float("nan"), 1))
    pair_avg_s = pair_ms / pair_n * 1e-3
    n = desc["n_atoms"]
    p_half = sc1["list_pairs"]
    # algorithmic bytes of one pair launch (FP64): positions+charge 32 B and
    # force 24 B per atom, plus the canonical half list of int32 indices
    b_alg = n * (32 + 24) + 4 * p_half
    peak, peak_kind = _peaks()
    achieved = b_alg / pair_avg_s / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": _traffic("k_pair_fp64_config1"),
                "kernel": "k_pair<fp64>", "peak_kind": peak_kind,
                "algorithmic_bytes": b_alg, "pair_launch_ms": pair_avg_s * 1e3}
    kernels = {k: {"ms_per_launch": v[0] / v[1], "share": v[0] / sum(x[0] for x in prof.values())}
               for k, v in prof.items()}

    # ---- mixed-precision leg on the same workload (reported beside)
    d2, f2 = W.rocksalt_melt(precision=A.MIXED)
    sm = A.System(ctx, d2, f2)
    sm.compute_forces()
    sm.step(args.warmup)
    tm, _ = sm.step_timed(args.steps)
    tm = _max_over_ranks(dist, local, tm)
    mixed = ws * args.steps / (tm * 1e-3)
    sm.profile(True)
    sm.step(args.steps)
    mprof = sm.profile_read()
    sm.profile(False)
    mpair_ms, mpair_n = mprof.get("pair", (float("nan"), 1))
    mpair_s = mpair_ms / mpair_n * 1e-3
    # mixed algorithmic bytes: int4 position + float charge 16 B, force 24 B
    b_alg_m = n * (16 + 24) + 4 * sm.scalars()["list_pairs"]
    mixed_roofline = {"bound": "hbm", "achieved": b_alg_m / mpair_s / 1e9, "peak": peak,
                      "unit": "GB/s", "frac": b_alg_m / mpair_s / 1e9 / peak,
                      "traffic": _traffic("k_pair_mixed_config1"), "kernel": "k_pair<mixed>",
                      "algorithmic_bytes": b_alg_m, "pair_launch_ms": mpair_s * 1e3}
    del sm

    # ---- end to end through the C ABI with host buffers: upload from
    # pinned host memory, force pass, K steps, per-step energies (history
    # ring) and the full frame back to the host
    import torch
    pinned = {k: torch.from_numpy(np.ascontiguousarray(frame[k])).pin_memory().numpy()
              for k in A.FRAME_KEYS}
    pinned["tag"] = frame["tag"]
    e2e_sys = A.System(ctx, desc)
    _barrier(dist, local)
    t0 = time.perf_counter()
    e2e_sys.upload(pinned)
    e2e_sys.compute_forces()
    e2e_sys.step(args.steps)
    hist = e2e_sys.history(args.steps)
    out, _ = e2e_sys.download()
    t1 = time.perf_counter()
    e2e_s = _max_over_ranks(dist, local, t1 - t0)
    h2d = sum(pinned[k].nbytes for k in A.FRAME_KEYS) + pinned["tag"].nbytes
    d2h = sum(out[k].nbytes for k in out) + hist.nbytes
    del e2e_sys

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline()
    p_rc = pairs_within(sys_, desc, 12.0) if rank == 0 else None

    if rank == 0:
        steps_s = value
        ns_day = steps_s / ws * DT_FS * 1e-6 * 86400.0
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "atoms": n, "pme_grid": [192, 192, 192],
                       "cutoff_A": 12.0, "skin_A": 1.0, "precision": "fp64",
                       "l2": "inputs larger than L2 (per-step working set ~0.7 GB)",
                       "replicas": ws, "parallelism": "replicas" if ws > 1 else "1 GPU"},
            "ns_per_day_per_replica": ns_day,
            "p50_ms": float(np.percentile(per_step, 50)),
            "p99_ms": float(np.percentile(per_step, 99)),
            "pair_interactions_per_s": (p_rc if p_rc is not None else p_half) * steps_s,
            "pairs_within_cutoff": p_rc, "pairs_in_list": p_half,
            "mixed_roofline": mixed_roofline,
            "neighbor_rebuilds": sc1["rebuilds"] - sc0["rebuilds"],
            "mixed_precision_value": mixed,
            "gpu_launches": launches,
            "roofline": roofline,
            "kernels": kernels,
            "cpu_baseline": cpu,
            "e2e": {"value": ws * args.steps / e2e_s, "unit": UNIT,
                    "h2d_bytes_per_step": h2d / args.steps,
                    "d2h_bytes_per_step": d2h / args.steps,
                    "includes": "upload from pinned host SoA, force pass, K steps, "
                                "per-step energy history and frame download"},
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    del sys_
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
