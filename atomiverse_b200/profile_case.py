"""Run a small instance of the benchmark workload for profiler captures.

    python -m atomiverse_b200.profile_case [--ncell 48] [--steps 3] [--mixed]

Builds an ncell^3 rock-salt melt with the benchmark's physics (12 A cutoff,
1 A skin, PME order 4 at ~0.94 A spacing, Nose-Hoover 1200 K), primes
forces, then advances `steps` steps.  ncell = 48 (110,592 ions, a 255 MB
neighbour list) keeps the working set above the 126 MB L2 while holding
well under 1 GB of device memory.
"""
import argparse
import sys

import atomiverse_b200 as A
from atomiverse_b200 import workloads as W


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ncell", type=int, default=48)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--mixed", action="store_true")
    ap.add_argument("--lanes", type=int, default=0)
    a = ap.parse_args(argv)
    K = 192 if a.ncell == 64 else round(a.ncell * 2.82 / 0.94)
    desc, frame = W.rocksalt_melt(ncell=a.ncell, grid=(K, K, K),
                                  precision=A.MIXED if a.mixed else A.FP64)
    ctx = A.Context(0)
    s = A.System(ctx, desc, frame)
    if a.lanes:
        s.set_pair_lanes(a.lanes)
    s.compute_forces()
    s.step(a.steps)
    sc = s.scalars()
    print(f"ncell {a.ncell}: {desc['n_atoms']} ions, K={K}, step {sc['step']}, "
          f"E={sc['energy']:.6f} eV, pairs={sc['list_pairs']}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
