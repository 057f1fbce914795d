"""Measurements of the three forms beside the plain FP64 path (one GPU).

  python -m atomiverse_b200.forms_bench precision [--ncell 63 --steps 10000]
  python -m atomiverse_b200.forms_bench ladder    [--systems 512 --steps 2000]
  python -m atomiverse_b200.forms_bench serve     [--requests 2000 --rate 200]

precision: 1,000,188-atom LJ fluid (63^3 FCC, rho* 0.8442, T* 0.72, rc 2.5,
  skin 0.3, seed 2028); FP64 and mixed builds on identical inputs; force,
  energy and virial error at step 0 against the CPU FP64 oracle and against
  each other; NVE drift over the run; timesteps/s of each.
ladder: 512 LJ systems, atom counts log-uniform in [256, 32768] (seed
  2029), T* 0.70-1.50, Langevin, mixed precision, one batch (one launch per
  kernel per step, graph-captured, autotuned lanes); aggregate timesteps/s
  against the plain FP64 path running the same systems one after another.
serve: Poisson arrivals of 1,000-step segments (60 % LJ, 40 % rock-salt
  PME, 500-200,000 atoms, seed 2030), continuous batching under an HBM
  budget, mixed precision; p50/p99 latency (queueing included), offered vs
  achieved atom-steps/s, and each sampled result compared with the same
  request run alone.

Each prints one JSON line.  Inputs are synthetic and seeded.  The oracle is
loaded only as the checker of the precision study's step-0 errors.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import atomiverse_b200 as A  # noqa: E402
from atomiverse_b200 import workloads as W  # noqa: E402

TAU_LJ_FS = W.TAU_LJ_FS


def _forces(out):
    return np.stack([out["fx"], out["fy"], out["fz"]], axis=1)


def force_errors(f, fref):
    d = np.linalg.norm(f - fref, axis=1)
    r = np.linalg.norm(fref, axis=1)
    rms = float(np.sqrt((d ** 2).sum() / (r ** 2).sum()))
    # per-atom relative error, over atoms whose force is not tiny
    big = r > 1e-3 * np.sqrt((r ** 2).mean())
    mx = float((d[big] / r[big]).max()) if big.any() else 0.0
    return rms, mx


def rel(a, b):
    return float(abs(a - b) / max(abs(b), 1e-300))


def drift(hist, n_atoms, eps=1.0, dt_tau=0.005):
    """NVE drift of E_tot / (N eps): slope per tau of a linear fit, and the
    largest excursion from the first value."""
    e = (hist[:, 0] + hist[:, 1]) / (n_atoms * eps)
    t = np.arange(len(e)) * dt_tau
    slope = float(np.polyfit(t, e, 1)[0]) if len(e) > 2 else 0.0
    return slope, float(np.abs(e - e[0]).max())


def precision_study(args):
    ctx = A.Context(0)
    desc, frame = W.lj_fcc(ncell=args.ncell, t_star=0.72, seed=2028, precision=A.FP64)
    desc["history_capacity"] = max(args.steps, 16)
    desc["stress_required"] = 1  # the virial is one of the compared quantities
    n = desc["n_atoms"]
    # the perfect lattice has (numerically) zero forces, so errors are taken
    # on a thermalised snapshot: the FP64 build run `equil` steps from the
    # lattice; both builds and the oracle then start from that same state
    s = A.System(ctx, desc, frame)
    s.compute_forces()
    s.step(args.equil)
    snap, _ = s.download()
    s.close()
    frame = dict(frame, **{k: snap[k] for k in ("x", "y", "z", "vx", "vy", "vz")})
    res = {"form": "precision", "workload": f"LJ fluid {n} atoms (FCC {args.ncell}^3), "
           "rho* 0.8442, T* 0.72, rc 2.5, skin 0.3, NVE, dt 0.005 tau", "atoms": n,
           "steps": args.steps, "errors_at": f"snapshot after {args.equil} FP64 steps "
           "from the lattice (identical inputs to every build)"}
    outs = {}
    for name, prec in (("fp64", A.FP64), ("mixed", A.MIXED)):
        d = dict(desc, precision=prec)
        s = A.System(ctx, d, frame)
        s.compute_forces()
        o, sc = s.download()
        outs[name] = (o, sc)
        ms, per = s.step_timed(args.steps)
        hist = s.history(args.steps)
        slope, excursion = drift(hist, n)
        res[name] = {"timesteps_per_s": args.steps / (ms * 1e-3),
                     "ms_per_step": ms / args.steps,
                     "p50_ms": float(np.percentile(per, 50)),
                     "p99_ms": float(np.percentile(per, 99)),
                     "nve_drift_per_tau": slope, "nve_max_excursion": excursion,
                     "tau_per_day": args.steps / (ms * 1e-3) * 0.005 * 86400.0,
                     "ns_per_day_metal_mapping": args.steps / (ms * 1e-3) * desc["dt"]
                     * 1e-6 * 86400.0}
        s.close()
    f64, f32 = _forces(outs["fp64"][0]), _forces(outs["mixed"][0])
    s64, s32 = outs["fp64"][1], outs["mixed"][1]
    rms, mx = force_errors(f32, f64)
    res["mixed_vs_fp64"] = {"force_rms_rel": rms, "force_max_rel": mx,
                            "energy_rel": rel(s32["energy"], s64["energy"]),
                            "virial_rel": float(np.abs(s32["stress"] - s64["stress"]).max()
                                                / np.abs(s64["stress"]).max())}
    if not args.no_oracle:
        res["vs_oracle"] = _oracle_errors(desc, frame, outs)
    res["speedup_mixed_over_fp64"] = (res["mixed"]["timesteps_per_s"]
                                      / res["fp64"]["timesteps_per_s"])
    return res


def _oracle_errors(desc, frame, outs):
    """Step-0 errors of both builds against the CPU FP64 oracle (checker)."""
    import oracle
    L = desc["box"]
    od = oracle.make_desc(desc["n_atoms"], L, nl_cutoff=desc["nl_cutoff"],
                          skin=desc["nl_skin"], has_lj=1, lj_eps=desc["lj_epsilon"],
                          lj_sigma=desc["lj_sigma"], lj_rc=desc["lj_cutoff"], dt=desc["dt"])
    o = oracle.OracleSystem(od)
    o.set_state(frame["x"], frame["y"], frame["z"], frame["vx"], frame["vy"], frame["vz"],
                None, None, None, frame["mass"], frame["charge"], None)
    o.build_list()
    o.compute_forces()
    st = o.state()
    sc = o.scalars()
    fref = np.stack([st["fx"], st["fy"], st["fz"]], axis=1)
    out = {}
    for name, (ob, sb) in outs.items():
        rms, mx = force_errors(_forces(ob), fref)
        out[name] = {"force_rms_rel": rms, "force_max_rel": mx,
                     "energy_rel": rel(sb["energy"], sc["energy"]),
                     "virial_rel": float(np.abs(sb["stress"] - sc["virial"]).max()
                                         / np.abs(sc["virial"]).max())}
    o.close()
    return out


def _batch_rate(ctx, items, steps, warmup):
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
    return b, dt, lanes, launches


def ladder(args):
    ctx = A.Context(0)
    items = W.ladder(n_systems=args.systems, precision=A.MIXED)
    sizes = np.array([d["n_atoms"] for d, _ in items])
    b, dt, lanes, launches = _batch_rate(ctx, items, args.steps, args.warmup)
    agg = args.systems * args.steps / dt
    res = {"form": "ladder", "workload": f"{args.systems} LJ systems, atoms log-uniform "
           "[256, 32768] (seed 2029), T* 0.70-1.50, Langevin damp 1 tau, mixed precision",
           "systems": args.systems, "atoms_total": int(sizes.sum()), "steps": args.steps,
           "batched_mixed": {"aggregate_timesteps_per_s": agg,
                             "atom_steps_per_s": float(sizes.sum()) * args.steps / dt,
                             "ms_per_step": dt * 1e3 / args.steps, "lanes_autotuned": lanes,
                             "launches_per_step": launches}}
    # the plain FP64 path: every system alone, one after another; timed on an
    # evenly spaced sample and scaled to all systems
    pick = np.unique(np.linspace(0, args.systems - 1, args.sample).round().astype(int))
    t_plain = 0.0
    errs = []
    for k in pick:
        d, f = items[k]
        d64 = dict(d, precision=A.FP64)
        s = A.System(ctx, d64, f)
        s.compute_forces()
        s.step(args.warmup)
        ms, _ = s.step_timed(args.plain_steps)
        t_plain += ms * 1e-3 / args.plain_steps
        # force error on the thermalised state this run reached (the FCC
        # start has near-zero forces): both builds from the same snapshot
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
    plain_agg = len(pick) / t_plain
    res["plain_fp64_sequential"] = {"aggregate_timesteps_per_s": plain_agg,
                                    "sampled_systems": int(len(pick)),
                                    "steps_per_system": args.plain_steps}
    res["speedup_batched_mixed_over_plain_fp64"] = agg / plain_agg
    res["force_rms_rel_mixed_vs_fp64_max"] = float(max(errs))
    b.close()
    return res


def _producer(specs, q, precision):
    """Builds request frames in arrival order ahead of the serving loop."""
    for sp in specs:
        q.put((sp, *W.build_request(sp, precision)))
    q.put(None)


def serve(args):
    import queue
    import threading
    ctx = A.Context(0)
    specs = W.request_specs(n_requests=args.requests, rate=args.rate, steps=args.seg_steps)
    check_ids = set(np.unique(np.linspace(0, len(specs) - 1, args.check).round().astype(int)))
    q = queue.Queue(maxsize=64)
    th = threading.Thread(target=_producer, args=(specs, q, A.MIXED), daemon=True)
    th.start()
    budget = int(args.budget_gb * 1e9)
    srv = A.Server(ctx, budget, max_active=args.max_active)
    if args.max_atoms:
        srv.set_limits(int(args.max_atoms))
    live = {}        # rid -> spec index
    kept = {}        # spec index -> (desc, frame, served output)
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
        srv.tick(args.chunk)
        for rid in list(live):
            r = srv.poll(rid)
            if r["state"] == 2:
                k = live.pop(rid)
                out, res = srv.collect(rid)
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
    res = {"form": "serve", "workload": f"{len(specs)} Poisson requests at {args.rate}/s "
           f"(seed 2030), {args.seg_steps}-step segments, 60% LJ / 40% rock-salt PME, "
           "500-200,000 atoms, mixed precision", "requests": len(specs),
           "budget_bytes": budget, "max_resident_atoms": int(args.max_atoms),
           "chunk": args.chunk, "peak_running": peak_running,
           "p50_latency_s": float(np.percentile(lat, 50)),
           "p99_latency_s": float(np.percentile(lat, 99)),
           "offered_atom_steps_per_s": offered,
           "achieved_atom_steps_per_s": atom_steps / span,
           "aggregate_timesteps_per_s": len(specs) * args.seg_steps / span,
           "makespan_s": span}
    srv.close()
    # the same requests alone: mixed (must equal the served result) and the
    # plain FP64 path (throughput baseline over the sample)
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
        ms, _ = s64.step_timed(args.plain_steps)
        s64.close()
        t64 += ms * 1e-3 / args.plain_steps * specs[k]["steps"]
        work += specs[k]["n_atoms"] * specs[k]["steps"]
    res["sampled_requests"] = len(kept)
    res["served_equals_alone_bitwise"] = bool(same)
    res["plain_fp64_alone_atom_steps_per_s"] = work / t64 if t64 else None
    if t64:
        res["speedup_served_over_plain_fp64"] = res["achieved_atom_steps_per_s"] / (work / t64)
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("form", choices=["precision", "ladder", "serve"])
    ap.add_argument("--ncell", type=int, default=63)
    ap.add_argument("--steps", type=int, default=0)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--no-oracle", action="store_true")
    ap.add_argument("--equil", type=int, default=500)
    ap.add_argument("--systems", type=int, default=512)
    ap.add_argument("--sample", type=int, default=32)
    ap.add_argument("--plain-steps", type=int, default=50)
    ap.add_argument("--requests", type=int, default=2000)
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--seg-steps", type=int, default=1000)
    ap.add_argument("--chunk", type=int, default=50)
    ap.add_argument("--budget-gb", type=float, default=120.0)
    ap.add_argument("--max-active", type=int, default=0)
    ap.add_argument("--check", type=int, default=8)
    ap.add_argument("--max-atoms", type=float, default=4e6,
                    help="serve: resident-atom admission limit (0 = memory budget only)")
    ap.add_argument("--out", default=None, help="also append the JSON line to this file")
    args = ap.parse_args(argv)
    if args.form == "precision":
        args.steps = args.steps or 10000
        res = precision_study(args)
    elif args.form == "ladder":
        args.steps = args.steps or 2000
        res = ladder(args)
    else:
        res = serve(args)
    line = json.dumps(res)
    print(line, flush=True)
    if args.out:
        with open(args.out, "a") as f:
            f.write(line + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
