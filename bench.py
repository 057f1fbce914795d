"""Benchmark of the MD hot path on B200: timesteps/s (and ns/day, p50/p99)
of the charged LJ melt with PME, beside the other workloads of the path.

Headline workload (one GPU): 262,144 ions on a 64^3 rock-salt lattice
(spacing 2.82 A, box 180.48 A), charges +-1 e, positions jittered
U(-0.2, 0.2) A (seed 2027), LJ sigma 3.0 A / eps 0.5 kJ/mol, masses 23 /
35.45 amu, real-space cutoff 12 A + 1 A skin, alpha = 0.256412 1/A (Ewald
tolerance 1e-5), PME order 4 on 192^3, Nose-Hoover 1200 K (tau 100 fs),
dt 2 fs, FP64.  One step = integrate, skin-gated neighbour rebuild, LJ +
real-space Coulomb, PME (spread, FFT, influence, inverse FFT, gather),
integrate + thermostat.  Synthetic seeded inputs; the per-step working set
(~0.7 GB) is far larger than the 126 MB L2.

Legs printed on the same JSON line (bounded so the default run ends in a
few minutes; single GPU only):
  ladder     512 LJ systems of 256-32,768 atoms (seed 2029), Langevin, mixed
             precision, one batch; aggregate timesteps/s against the same
             systems on the plain FP64 path one at a time (sampled), and the
             force RMS error of mixed against FP64 -- the >= 3x target
  precision  1,000,188-atom LJ fluid: mixed vs FP64 force / energy / virial
             error on a thermalised snapshot and timesteps/s of both builds
             (both against the CPU oracle: tests/test_gpu_fullsize.py)
  drift      the 4,000-atom LJ fluid, FP64 NVE, 1,000 steps: energy drift
  deck       the reference's published LJ deck (10,648 atoms on a simple
             cubic lattice, density 0.8, rc 2.5, dt 0.005 fs, FP64), timed as
             the reference times it (wall clock of run(frame, 80) with the
             frame download), for context beside its GH200 figure

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                  [--legs ladder,precision,drift,deck | none]
  python bench.py --form {ladder,precision,serve,drift,deck} [...]   full-size
  python bench.py --case rocksalt [--ncell 48 --steps 3 --mixed --lanes 4]
                  (a small instance of the headline for profiler captures)

With N > 1 (torchrun, one rank per GPU) every rank advances its own
replica of the headline system (the path does not shard one system); the
value is the sum over ranks, timed as the max over ranks.
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
# launches of one neighbour-list build (cell sort + rows): in the step graph
# they run only on steps that rebuild a list
REBUILD_KERNELS = 6
# FP64 instructions per evaluated list entry of k_pair<fp64> on this workload
# (ncu: 250 M FP64 warp instructions for 108 M entries, one launch)
FP64_PER_ENTRY = 74


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
    # host cores only: rank 0 runs it, the other ranks of a torchrun launch
    # exit at once (no process group, no GPU work)
    rank = int(os.environ.get("RANK", "0"))
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


# ---------------------------------------------------------------- forms

def _forces(out):
    return np.stack([out["fx"], out["fy"], out["fz"]], axis=1)


def force_errors(f, fref):
    """RMS relative error sqrt(sum |F - F_ref|^2 / sum |F_ref|^2) and the
    largest per-atom relative error over atoms whose force is not tiny."""
    d = np.linalg.norm(f - fref, axis=1)
    r = np.linalg.norm(fref, axis=1)
    rms = float(np.sqrt((d ** 2).sum() / (r ** 2).sum()))
    big = r > 1e-3 * np.sqrt((r ** 2).mean())
    mx = float((d[big] / r[big]).max()) if big.any() else 0.0
    return rms, mx


def _rel(a, b):
    return float(abs(a - b) / max(abs(b), 1e-300))


def nve_drift(hist, n_atoms, eps=1.0, dt_tau=0.005):
    """NVE drift of E_tot / (N eps): slope per tau of a linear fit, and the
    largest excursion from the first value."""
    e = (hist[:, 0] + hist[:, 1]) / (n_atoms * eps)
    t = np.arange(len(e)) * dt_tau
    slope = float(np.polyfit(t, e, 1)[0]) if len(e) > 2 else 0.0
    return slope, float(np.abs(e - e[0]).max())


def form_precision(ctx, ncell=63, steps=10000, equil=500):
    """Precision study: 4 ncell^3 LJ atoms (63 -> 1,000,188; rho* 0.8442,
    T* 0.72, rc 2.5, skin 0.3, seed 2028), FP64 and mixed builds on
    identical inputs.  Errors are taken on a thermalised snapshot (the FCC
    start has zero forces): the FP64 build run `equil` steps; then each
    build's force pass, `steps` timed NVE steps and their drift."""
    import atomiverse_b200 as A
    from atomiverse_b200 import workloads as W
    desc, frame = W.lj_fcc(ncell=ncell, t_star=0.72, seed=2028, precision=A.FP64)
    desc["history_capacity"] = max(steps, 16)
    desc["stress_required"] = 1
    n = desc["n_atoms"]
    s = A.System(ctx, desc, frame)
    s.compute_forces()
    s.step(equil)
    snap, _ = s.download()
    s.close()
    frame = dict(frame, **{k: snap[k] for k in ("x", "y", "z", "vx", "vy", "vz")})
    res = {"workload": f"LJ fluid {n} atoms (FCC {ncell}^3), rho* 0.8442, T* 0.72, "
           "rc 2.5, skin 0.3, NVE, dt 0.005 tau", "atoms": n, "steps": steps,
           "errors_at": f"snapshot after {equil} FP64 steps from the lattice "
           "(identical inputs to every build)"}
    outs = {}
    for name, prec in (("fp64", A.FP64), ("mixed", A.MIXED)):
        s = A.System(ctx, dict(desc, precision=prec), frame)
        s.compute_forces()
        outs[name] = s.download()
        ms, per = s.step_timed(steps)
        slope, excursion = nve_drift(s.history(steps), n)
        rate = steps / (ms * 1e-3)
        res[name] = {"timesteps_per_s": rate, "ms_per_step": ms / steps,
                     "p50_ms": float(np.percentile(per, 50)),
                     "p99_ms": float(np.percentile(per, 99)),
                     "nve_drift_per_tau": slope, "nve_max_excursion": excursion,
                     "tau_per_day": rate * 0.005 * 86400.0,
                     "pair_interactions_per_s": None}
        s.close()
    (o64, s64), (o32, s32) = outs["fp64"], outs["mixed"]
    rms, mx = force_errors(_forces(o32), _forces(o64))
    res["mixed_vs_fp64"] = {"force_rms_rel": rms, "force_max_rel": mx,
                            "energy_rel": _rel(s32["energy"], s64["energy"]),
                            "virial_rel": float(np.abs(s32["stress"] - s64["stress"]).max()
                                                / np.abs(s64["stress"]).max())}
    res["speedup_mixed_over_fp64"] = (res["mixed"]["timesteps_per_s"]
                                      / res["fp64"]["timesteps_per_s"])
    return res


def form_ladder(ctx, systems=512, steps=2000, warmup=5, sample=32, plain_steps=50):
    """Replica ladder: `systems` LJ systems, atom counts log-uniform in
    [256, 32768] (seed 2029), T* 0.70-1.50, Langevin damp 1 tau, mixed
    precision, one batch (one launch per kernel per step, graph-captured,
    autotuned lanes); aggregate timesteps/s against the plain FP64 path
    running the same systems one after another (an evenly spaced sample of
    `sample` systems, each timed alone over `plain_steps` steps and scaled
    to the whole ladder), and the force RMS error of mixed against FP64 on
    each sampled system's thermalised state."""
    import atomiverse_b200 as A
    from atomiverse_b200 import workloads as W
    items = W.ladder(n_systems=systems, precision=A.MIXED)
    sizes = np.array([d["n_atoms"] for d, _ in items])
    b = A.Batch(ctx, items)
    lanes = b.autotune()
    b.compute_forces()
    b.step(warmup)
    b.download(0, keys=())
    t0 = time.perf_counter()
    b.step(steps)
    b.download(0, keys=())            # synchronises the engine's stream
    dt = time.perf_counter() - t0
    launches = b.launch_count() / max(steps, 1)
    agg = systems * steps / dt
    res = {"workload": f"{systems} LJ systems, atoms log-uniform [256, 32768] (seed 2029), "
           "T* 0.70-1.50, Langevin damp 1 tau, mixed precision",
           "systems": systems, "atoms_total": int(sizes.sum()), "steps": steps,
           "batched_mixed": {"aggregate_timesteps_per_s": agg,
                             "atom_steps_per_s": float(sizes.sum()) * steps / dt,
                             "ms_per_step": dt * 1e3 / steps, "lanes_autotuned": lanes,
                             "launches_per_step": launches}}
    b.close()
    pick = np.unique(np.linspace(0, systems - 1, sample).round().astype(int))
    t_plain = 0.0
    errs = []
    for k in pick:
        d, f = items[k]
        d64 = dict(d, precision=A.FP64)
        s = A.System(ctx, d64, f)
        s.compute_forces()
        s.step(warmup)
        ms, _ = s.step_timed(plain_steps)
        t_plain += ms * 1e-3 / plain_steps
        snap, _ = s.download()
        s.close()
        f2 = dict(f, **{c: snap[c] for c in ("x", "y", "z", "vx", "vy", "vz")})
        s64 = A.System(ctx, d64, f2)
        s64.compute_forces()
        o64, _ = s64.download()
        s64.close()
        sm = A.System(ctx, d, f2)
        sm.compute_forces()
        o32, _ = sm.download()
        sm.close()
        errs.append(force_errors(_forces(o32), _forces(o64))[0])
    # the sample's mean time per system-step, scaled to the whole ladder
    plain_agg = len(pick) / t_plain
    res["plain_fp64_sequential"] = {"aggregate_timesteps_per_s": plain_agg,
                                    "sampled_systems": int(len(pick)),
                                    "steps_per_system": plain_steps}
    res["speedup_batched_mixed_over_plain_fp64"] = agg / plain_agg
    res["target_speedup"] = 3.0
    res["force_rms_rel_mixed_vs_fp64_max"] = float(max(errs))
    res["force_rms_target"] = 5e-6
    return res


def form_drift(ctx, steps=1000):
    """The plain LJ fluid: 4,000 atoms (FCC 10^3, rho* 0.8442, T* 1.44, seed
    2026), rc 2.5, skin 0.3, FP64 NVE, dt 0.005 tau, rebuild on half-skin
    displacement; the energy drift over `steps` steps.  (Its forces against
    the CPU oracle are a parity test: tests/test_gpu_parity.py.)"""
    import atomiverse_b200 as A
    from atomiverse_b200 import workloads as W
    desc, frame = W.lj_fcc(ncell=10, t_star=1.44, seed=2026, precision=A.FP64)
    desc["history_capacity"] = max(steps, 16)
    desc["stress_required"] = 1
    n = desc["n_atoms"]
    s = A.System(ctx, desc, frame)
    s.compute_forces()
    ms, per = s.step_timed(steps)
    slope, excursion = nve_drift(s.history(steps), n)
    sc = s.scalars()
    s.close()
    res = {"workload": f"LJ fluid {n} atoms (FCC 10^3), rho* 0.8442, T* 1.44, rc 2.5, "
           "skin 0.3, FP64 NVE, dt 0.005 tau", "atoms": n, "steps": steps,
           "timesteps_per_s": steps / (ms * 1e-3),
           "p50_ms": float(np.percentile(per, 50)), "p99_ms": float(np.percentile(per, 99)),
           "nve_drift_per_tau": slope, "nve_max_excursion": excursion,
           "rebuilds": sc["rebuilds"]}
    return res


def deck_frame(n_side=22, density=0.8):
    """The reference's LJ deck (benchmarks/cuda/bench_nonbonded_style.cu:
    make_lj): n_side^3 atoms on a simple cubic lattice at `density`, unit
    masses, small patterned velocities."""
    n = n_side ** 3
    L = (n / density) ** (1.0 / 3.0)
    sp = L / n_side
    ix, iy, iz = (a.ravel() for a in np.meshgrid(np.arange(n_side), np.arange(n_side),
                                                 np.arange(n_side), indexing="ij"))
    frame = {"x": (ix + 0.5) * sp, "y": (iy + 0.5) * sp, "z": (iz + 0.5) * sp,
             "vx": 0.01 * ((ix + iy + iz) % 3 - 1.0), "vy": 0.01 * ((ix + 2 * iy) % 3 - 1.0),
             "vz": 0.01 * ((2 * ix + iz) % 3 - 1.0), "mass": np.ones(n),
             "charge": np.zeros(n)}
    desc = dict(n_atoms=n, box=(L, L, L), precision=0, nl_cutoff=2.5, nl_skin=0.3,
                lj_enabled=1, lj_epsilon=1.0, lj_sigma=1.0, lj_cutoff=2.5, dt=0.005)
    return desc, frame


def form_deck(ctx, steps=80, warmup=15, repeats=5):
    """The reference's published LJ deck (benchmarks/lj/README.md:14-17:
    10,648 atoms, 80 steps after 15 warm-up, GH200 0.1098 ms/step =
    96.997 M atom-steps/s), run through System.run(frame, n) and timed as
    the reference times it: the wall clock of run(frame, 80), which ends
    with the frame download.  Best of `repeats`."""
    import atomiverse_b200 as A
    desc, frame = deck_frame()
    n = desc["n_atoms"]
    s = A.System(ctx, desc)
    fr = dict(frame)
    s.run(fr, warmup)
    best = 1e30
    for _ in range(repeats):
        t0 = time.perf_counter()
        s.run(fr, steps)
        best = min(best, time.perf_counter() - t0)
    s.close()
    ms = best * 1e3 / steps
    return {"workload": "reference LJ deck: 10,648 atoms, simple cubic 22^3, density 0.8, "
            "rc 2.5, skin 0.3, dt 0.005 fs, FP64 NVE", "atoms": n, "steps": steps,
            "ms_per_step": ms, "matom_steps_per_s": n / ms * 1e-3,
            "reference_gh200_ms_per_step": 0.1098,
            "reference_gh200_matom_steps_per_s": 96.997,
            "timing": "wall clock of run(frame, 80) including the frame download, "
                      "best of 5 (the reference's own timing of this deck)"}


def _producer(specs, q, precision):
    """Builds request frames in arrival order ahead of the serving loop."""
    from atomiverse_b200 import workloads as W
    for sp in specs:
        q.put((sp, *W.build_request(sp, precision)))
    q.put(None)


def form_serve(ctx, requests=2000, rate=200.0, seg_steps=1000, chunk=50, budget_gb=120.0,
               max_active=0, max_atoms=4e6, check=8, plain_steps=50):
    """Served request stream: Poisson arrivals of `seg_steps`-step segments
    (60 % LJ, 40 % rock-salt PME, 500-200,000 atoms, seed 2030), continuous
    batching under an HBM budget, mixed precision; p50/p99 latency
    (queueing included), offered vs achieved atom-steps/s, and each sampled
    result compared with the same request run alone (bitwise)."""
    import queue
    import threading

    import atomiverse_b200 as A
    from atomiverse_b200 import workloads as W
    specs = W.request_specs(n_requests=requests, rate=rate, steps=seg_steps)
    check_ids = set(np.unique(np.linspace(0, len(specs) - 1, check).round().astype(int)))
    q = queue.Queue(maxsize=64)
    th = threading.Thread(target=_producer, args=(specs, q, A.MIXED), daemon=True)
    th.start()
    srv = A.Server(ctx, int(budget_gb * 1e9), max_active=max_active)
    if max_atoms:
        srv.set_limits(int(max_atoms))
    live, kept = {}, {}
    lat, arrivals, done_at = [], [], []
    atom_steps = 0
    nxt = q.get()
    t0 = time.perf_counter()
    peak_running = 0
    while nxt is not None or live:
        now = time.perf_counter() - t0
        while nxt is not None and nxt[0]["t"] <= now:
            sp, d, f = nxt
            k = len(arrivals)
            rid = srv.submit(d, f, sp["steps"])
            live[rid] = k
            arrivals.append(sp["t"])
            if k in check_ids:
                kept[k] = (d, f, None)
            nxt = q.get()
        st = srv.stats()
        peak_running = max(peak_running, st["running"])
        if st["queued"] + st["running"] == 0:
            if nxt is not None:
                time.sleep(max(0.0, min(0.01, nxt[0]["t"] - (time.perf_counter() - t0))))
            continue
        srv.tick(chunk)
        for rid in list(live):
            r = srv.poll(rid)
            if r["state"] == 2:
                k = live.pop(rid)
                out, _ = srv.collect(rid)
                t_end = time.perf_counter() - t0
                lat.append(t_end - specs[k]["t"])
                done_at.append(t_end)
                atom_steps += specs[k]["n_atoms"] * specs[k]["steps"]
                if k in kept:
                    kept[k] = (kept[k][0], kept[k][1], out)
            elif r["state"] in (3, 4):
                raise RuntimeError(f"request {rid} ended in state {r['state']}")
    span = max(done_at) - min(arrivals)
    offered = sum(sp["n_atoms"] * sp["steps"] for sp in specs) / max(specs[-1]["t"], 1e-9)
    res = {"workload": f"{len(specs)} Poisson requests at {rate}/s (seed 2030), "
           f"{seg_steps}-step segments, 60% LJ / 40% rock-salt PME, 500-200,000 atoms, "
           "mixed precision", "requests": len(specs), "budget_bytes": int(budget_gb * 1e9),
           "max_resident_atoms": int(max_atoms), "chunk": chunk, "peak_running": peak_running,
           "p50_latency_s": float(np.percentile(lat, 50)),
           "p99_latency_s": float(np.percentile(lat, 99)),
           "offered_atom_steps_per_s": offered, "achieved_atom_steps_per_s": atom_steps / span,
           "aggregate_timesteps_per_s": len(specs) * seg_steps / span, "makespan_s": span}
    srv.close()
    same = True
    t64, work = 0.0, 0
    for k, (d, f, out) in sorted(kept.items()):
        s = A.System(ctx, d, f)
        s.compute_forces()
        s.step(specs[k]["steps"])
        alone, _ = s.download()
        s.close()
        same &= all(np.array_equal(alone[c], out[c]) for c in ("x", "y", "z", "vx", "vy", "vz"))
        s64 = A.System(ctx, dict(d, precision=A.FP64), f)
        s64.compute_forces()
        ms, _ = s64.step_timed(plain_steps)
        s64.close()
        t64 += ms * 1e-3 / plain_steps * specs[k]["steps"]
        work += specs[k]["n_atoms"] * specs[k]["steps"]
    res["sampled_requests"] = len(kept)
    res["served_equals_alone_bitwise"] = bool(same)
    res["plain_fp64_alone_atom_steps_per_s"] = work / t64 if t64 else None
    if t64:
        res["speedup_served_over_plain_fp64"] = res["achieved_atom_steps_per_s"] / (work / t64)
    return res


def run_form(args):
    import atomiverse_b200 as A
    ctx = A.Context(0)
    if args.form == "precision":
        res = form_precision(ctx, ncell=args.ncell or 63, steps=args.steps or 10000)
    elif args.form == "ladder":
        res = form_ladder(ctx, systems=args.systems, steps=args.steps or 2000)
    elif args.form == "drift":
        res = form_drift(ctx, steps=args.steps or 1000)
    elif args.form == "deck":
        res = form_deck(ctx)
    else:
        res = form_serve(ctx, requests=args.requests, rate=args.rate)
    res["form"] = args.form
    print(json.dumps(res), flush=True)
    return 0


def run_case(args):
    """A small instance of the headline workload for profiler captures:
    ncell^3 rock-salt ions with the headline's physics (12 A cutoff, 1 A
    skin, PME order 4 at ~0.94 A spacing, Nose-Hoover 1200 K); forces
    primed, then `steps` steps.  ncell = 48 (110,592 ions) keeps the
    working set above the 126 MB L2 and well under 1 GB on the device."""
    import atomiverse_b200 as A
    from atomiverse_b200 import workloads as W
    ncell = args.ncell or 48
    K = 192 if ncell == 64 else round(ncell * 2.82 / 0.94)
    desc, frame = W.rocksalt_melt(ncell=ncell, grid=(K, K, K),
                                  precision=A.MIXED if args.mixed else A.FP64)
    ctx = A.Context(0)
    s = A.System(ctx, desc, frame)
    if args.lanes:
        s.set_pair_lanes(args.lanes)
    s.compute_forces()
    s.step(args.steps)
    sc = s.scalars()
    print(f"ncell {ncell}: {desc['n_atoms']} ions, K={K}, step {sc['step']}, "
          f"E={sc['energy']:.6f} eV, pairs={sc['list_pairs']}")
    return 0


# --------------------------------------------------------------- headline

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--legs", default="ladder,precision,drift,deck",
                    help="comma list of extra legs on the headline line, or 'none'")
    ap.add_argument("--form", choices=["precision", "ladder", "serve", "drift", "deck"])
    ap.add_argument("--case", choices=["rocksalt"])
    ap.add_argument("--ncell", type=int, default=0)
    ap.add_argument("--mixed", action="store_true")
    ap.add_argument("--lanes", type=int, default=0)
    ap.add_argument("--systems", type=int, default=512)
    ap.add_argument("--requests", type=int, default=2000)
    ap.add_argument("--rate", type=float, default=200.0)
    args = ap.parse_args()
    if args.form:
        return run_form(args)
    if args.case:
        args.steps = args.steps or 3
        return run_case(args)
    if args.steps is None:
        args.steps = 500
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_headline(args)


def run_headline(args):
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
    t_max = _max_over_ranks(dist, local, total_ms)
    sc1 = sys_.scalars()
    value = ws * args.steps / (t_max * 1e-3)
    rebuilds = sc1["rebuilds"] - sc0["rebuilds"]
    # the list-build kernels launch only on rebuild steps (conditional graph
    # nodes, systems of >= 100,000 atoms); launch_count() counts them on
    # every step
    launches = sys_.launch_count()
    if desc["n_atoms"] >= 100000:
        launches -= REBUILD_KERNELS * (args.steps - rebuilds)
    # rebuild steps are the slowest ones: split the per-step times by count
    srt = np.sort(per_step)[::-1]
    rb_ms = float(srt[:rebuilds].mean()) if rebuilds > 0 else None
    plain_ms = float(srt[rebuilds:].mean()) if rebuilds < len(srt) else None

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
    # the pair kernel's own limit: the FP64 pipe (64 FP64 lanes per SM per
    # clock on B200).  Every listed pair is evaluated from both of its rows,
    # with FP64_PER_ENTRY FP64 instructions per evaluation (the ncu count of
    # the current kernel); the clock is the SM clock sampled during the run
    import torch
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    fp64_peak = sms * 64 * clk["sm_mhz"] * 1e6 / 1e12 if clk.get("sm_mhz") else None
    fp64_done = 2 * p_half * FP64_PER_ENTRY / pair_avg_s / 1e12
    compute_roofline = {"bound": "fp64", "kernel": "k_pair<fp64>", "unit": "T FP64 instr/s",
                        "achieved": fp64_done, "peak": fp64_peak,
                        "frac": fp64_done / fp64_peak if fp64_peak else None,
                        "fp64_instr_per_entry": FP64_PER_ENTRY, "entries": 2 * p_half,
                        "peak_kind": "nominal 64 lanes/SM/clock x SMs x sampled SM clock"}
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
    sm.close()

    # ---- end to end through the C ABI with host buffers: upload from
    # pinned host memory, force pass, K' steps, per-step energies (history
    # ring) and the full frame back to the host; K' = max(K, 500) so that
    # the one upload and force pass are spread as in a production segment
    import torch
    e2e_steps = max(args.steps, 500)
    pinned = {k: torch.from_numpy(np.ascontiguousarray(frame[k])).pin_memory().numpy()
              for k in A.FRAME_KEYS}
    pinned["tag"] = frame["tag"]
    e2e_sys = A.System(ctx, desc)
    _barrier(dist, local)
    t0 = time.perf_counter()
    e2e_sys.upload(pinned)
    e2e_sys.compute_forces()
    e2e_sys.step(e2e_steps)
    hist = e2e_sys.history(e2e_steps)
    out, _ = e2e_sys.download()
    t1 = time.perf_counter()
    e2e_s = _max_over_ranks(dist, local, t1 - t0)
    h2d = sum(pinned[k].nbytes for k in A.FRAME_KEYS) + pinned["tag"].nbytes
    d2h = sum(out[k].nbytes for k in out) + hist.nbytes
    e2e_sys.close()

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline()
    p_rc = pairs_within(sys_, desc, 12.0) if rank == 0 else None
    sys_.close()

    legs = {}
    if ws == 1 and args.legs != "none":
        for leg in args.legs.split(","):
            t_leg = time.perf_counter()
            try:
                if leg == "ladder":
                    legs[leg] = form_ladder(ctx, systems=512, steps=200, warmup=5,
                                            sample=16, plain_steps=30)
                elif leg == "precision":
                    legs[leg] = form_precision(ctx, ncell=63, steps=300, equil=300)
                elif leg == "drift":
                    legs[leg] = form_drift(ctx, steps=1000)
                elif leg == "deck":
                    legs[leg] = form_deck(ctx)
                else:
                    continue
                legs[leg]["leg_seconds"] = time.perf_counter() - t_leg
            except Exception as e:  # a failing leg is reported, not hidden
                legs[leg] = {"error": f"{type(e).__name__}: {e}"}

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
            "rebuild_step_ms": rb_ms, "non_rebuild_step_ms": plain_ms,
            "pair_interactions_per_s": (p_rc if p_rc is not None else p_half) * steps_s,
            "pairs_within_cutoff": p_rc, "pairs_in_list": p_half,
            "mixed_roofline": mixed_roofline,
            "neighbor_rebuilds": rebuilds,
            "mixed_precision_value": mixed,
            "gpu_launches": launches,
            "roofline": roofline,
            "compute_roofline": compute_roofline,
            "kernels": kernels,
            "cpu_baseline": cpu,
            "e2e": {"value": ws * e2e_steps / e2e_s, "unit": UNIT,
                    "h2d_bytes_per_step": h2d / e2e_steps,
                    "d2h_bytes_per_step": d2h / e2e_steps,
                    "steps": e2e_steps,
                    "includes": "upload from pinned host SoA, force pass, the steps, "
                                "per-step energy history and frame download"},
            "clocks": clk,
            "legs": legs,
        }
        if "ladder" in legs and "speedup_batched_mixed_over_plain_fp64" in legs["ladder"]:
            line["target_ladder_speedup"] = legs["ladder"]["speedup_batched_mixed_over_plain_fp64"]
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
