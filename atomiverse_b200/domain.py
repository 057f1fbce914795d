"""Domain decomposition of one MD system over the ranks of one node.

The reference splits one system across GPUs with a brick decomposition:
each rank owns the atoms of its sub-box, receives ghost atoms within the
cutoff of its faces in a per-axis cascade (``CommBrick``;
``src/cuda/communication/multi_gpu.cu:480-700``, positions forwarded every
step over the same plan, forces sent back), migrates atoms that left its
sub-box between steps, and, for PME, all-reduces a replicated charge grid,
transforms it on rank 0 and broadcasts it back (``src/cpu/longrange/
pme.cpp:191-216``).

Here the same decomposition is made for slabs along x, the axis the PME mesh
is also split along, so each rank holds the mesh planes inside its slab and
the 3D transform needs two all-to-all transposes instead of a replicated
grid:

* ownership: rank r owns x in [r L/P, (r+1) L/P); a slab at least
  ``rlist`` wide gets all its ghosts from its two neighbours (shifted by
  +-L across the periodic boundary), so the cascade has one axis;
* halo (``halo_plan``, ``exchange``, ``forward``): the owned atoms within
  ``rlist`` of a neighbour's face, with the shift that places them next to
  that neighbour; the plan is kept and replayed with new positions until
  the next list build (the reference's forward_comm);
* forces: each rank evaluates its owned atoms against owned + ghost atoms
  (a full shell), so no force travels back; the pair energy of a rank is
  half of its owned-ghost pairs plus its owned-owned pairs;
* migration (``migrate``): atoms whose x left the slab move to their new
  owner, in one exchange;
* PME mesh: rank r owns the planes p with p h in its slab (h = L/K0);
  ``to_pencils`` / ``to_slabs`` transpose between x-slabs and y-pencils of
  the half-complex spectrum, ``lower_planes`` brings the ``order`` planes
  below the slab that the force interpolation of the slab's atoms reads.

Host logic only: the per-rank arithmetic (pair forces, spreading, the
transforms along each axis, interpolation) is the single-GPU library's.  All
exchanges are ``torch.distributed.all_to_all_single`` (NCCL on GPUs, gloo
on CPU; every rank makes the same calls in the same order), with the row
counts exchanged first; nothing reads another GPU's memory directly.
Tested on two gloo ranks on CPU (``tests/test_dist_domain.py``); unmeasured
on hardware.
"""
from __future__ import annotations

import math

import numpy as np


def _dist():
    import torch.distributed as dist
    return dist


class Slabs:
    """x-slab decomposition of an orthorhombic box over ``world_size`` ranks.

    ``box``: the three edges; ``rlist``: cutoff + skin (the ghost shell);
    ``K``, ``order``: the PME mesh and spline order, when the system has PME.
    Raises ValueError when a slab is narrower than ``rlist`` (ghosts would
    come from beyond the neighbours), or when the mesh is too coarse for the
    shell to hold every atom whose splines reach a slab's planes."""

    def __init__(self, box, rlist: float, world_size: int, rank: int, K=None, order: int = 4):
        self.L = np.array([float(b) for b in box[:3]])
        self.rlist = float(rlist)
        self.P = int(world_size)
        self.r = int(rank)
        if self.P < 1 or not 0 <= self.r < self.P:
            raise ValueError("rank must be in [0, world_size)")
        self.width = self.L[0] / self.P
        self.lo = self.r * self.width
        self.hi = (self.r + 1) * self.width if self.r < self.P - 1 else self.L[0]
        if self.P > 1 and self.width < self.rlist:
            raise ValueError(f"slab width {self.width:.3f} is below cutoff + skin {self.rlist}: "
                             f"use fewer ranks")
        self.K = None if K is None else tuple(int(k) for k in K)
        self.order = int(order)
        if self.K is not None:
            K0 = self.K[0]
            if K0 < self.P:
                raise ValueError("fewer mesh planes than ranks")
            self.h = self.L[0] / K0
            # the splines of an atom at x cover planes floor(x/h)-order+1 ..
            # floor(x/h): the slab's planes draw on atoms up to
            # (P1 + order) h, which the shell must reach
            if (self.order + 1) * self.h > self.rlist:
                raise ValueError("PME mesh too coarse for the ghost shell")
            # planes p with p h in [lo, hi)
            self.P0 = (self.r * K0 + self.P - 1) // self.P
            self.P1 = ((self.r + 1) * K0 + self.P - 1) // self.P
            # the K1 rows of the spectrum held after the transpose
            K1 = self.K[1]
            self.M1 = [(s * K1) // self.P for s in range(self.P + 1)]
            self.planes = [((s * K0 + self.P - 1) // self.P, ((s + 1) * K0 + self.P - 1) // self.P)
                           for s in range(self.P)]

    # ---- ownership -----------------------------------------------------------
    def owner(self, x) -> np.ndarray:
        """Rank owning each x (wrapped into [0, L))."""
        xw = np.mod(np.asarray(x, dtype=np.float64), self.L[0])
        return np.minimum((xw / self.width).astype(np.int64), self.P - 1)

    def take_owned(self, rows: dict) -> dict:
        """The owned part of a full frame (dict of per-atom arrays with at
        least x and tag), ordered by tag."""
        mine = self.owner(rows["x"]) == self.r
        out = {k: np.asarray(v)[mine] for k, v in rows.items()}
        o = np.argsort(out["tag"], kind="stable")
        return {k: v[o] for k, v in out.items()}

    # ---- the exchange primitive ----------------------------------------------
    def alltoallv(self, parts: list) -> np.ndarray:
        """Send parts[d] (a float64 array of shape (k_d, C)) to rank d and
        return what every rank sent here, stacked by source rank."""
        import torch
        dist = _dist()
        C = parts[0].shape[1] if parts and parts[0].ndim == 2 else 1
        counts = torch.tensor([p.shape[0] for p in parts], dtype=torch.int64)
        rcounts = torch.empty(self.P, dtype=torch.int64)
        dist.all_to_all_single(rcounts, counts)
        send = torch.from_numpy(np.ascontiguousarray(
            np.concatenate([p.reshape(-1, C) for p in parts], axis=0).reshape(-1)))
        recv = torch.empty(int(rcounts.sum()) * C, dtype=torch.float64)
        dist.all_to_all_single(recv, send, output_split_sizes=(rcounts * C).tolist(),
                               input_split_sizes=(counts * C).tolist())
        return recv.numpy().reshape(-1, C)

    # ---- halo -------------------------------------------------------------------
    def halo_plan(self, x) -> list:
        """Send plan for the ghosts of the owned atoms at x: one entry per
        neighbour face, (destination rank, owned indices, x shift).  The
        lower neighbour gets the atoms within rlist above this slab's lower
        face, the upper neighbour those within rlist below its upper face."""
        x = np.asarray(x, dtype=np.float64)
        dn, up = (self.r - 1) % self.P, (self.r + 1) % self.P
        plan = []
        low = np.nonzero(x < self.lo + self.rlist)[0]
        plan.append((dn, low, self.L[0] if self.r == 0 else 0.0))
        high = np.nonzero(x >= self.hi - self.rlist)[0]
        plan.append((up, high, -self.L[0] if self.r == self.P - 1 else 0.0))
        return plan

    def exchange(self, plan: list, cols: np.ndarray) -> np.ndarray:
        """Ghost rows for this rank: cols is (n_owned, C) with x in column 0;
        every planned row is sent with its x shifted.  Rows arrive by source
        rank, then in plan order."""
        C = cols.shape[1]
        parts = [np.zeros((0, C)) for _ in range(self.P)]
        for dest, idx, shift in plan:
            rows = cols[idx].copy()
            rows[:, 0] += shift
            parts[dest] = np.concatenate([parts[dest], rows], axis=0)
        return self.alltoallv(parts)

    def forward(self, plan: list, cols: np.ndarray) -> np.ndarray:
        """The same exchange with the current values (positions between list
        builds): the ghosts keep their order."""
        return self.exchange(plan, cols)

    # ---- migration -------------------------------------------------------------
    def migrate(self, cols: np.ndarray) -> np.ndarray:
        """Rows (x in column 0, wrapped here into [0, L)) whose atom left the
        slab go to its new owner; returns this rank's rows, the kept ones
        first, then the arrivals by source rank."""
        cols = cols.copy()
        cols[:, 0] = np.mod(cols[:, 0], self.L[0])
        dest = self.owner(cols[:, 0])
        keep = dest == self.r
        parts = [cols[(dest == d) & ~keep] for d in range(self.P)]
        parts[self.r] = np.zeros((0, cols.shape[1]))
        return np.concatenate([cols[keep], self.alltoallv(parts)], axis=0)

    # ---- PME mesh slabs ----------------------------------------------------------
    def to_pencils(self, slab: np.ndarray) -> np.ndarray:
        """(P1-P0, K1, Kh) complex, this rank's x planes of the spectrum
        transformed along y and z -> (K0, M1b-M1a, Kh): every x plane of
        this rank's rows m1 in [M1a, M1b)."""
        import torch
        dist = _dist()
        n_p, K1, Kh = slab.shape
        parts = [np.ascontiguousarray(slab[:, self.M1[s]:self.M1[s + 1], :]).view(np.float64)
                 .reshape(-1) for s in range(self.P)]
        rows = self.M1[self.r + 1] - self.M1[self.r]
        rsz = [(self.planes[s][1] - self.planes[s][0]) * rows * Kh * 2 for s in range(self.P)]
        recv = torch.empty(sum(rsz), dtype=torch.float64)
        dist.all_to_all_single(recv, torch.from_numpy(np.concatenate(parts)),
                               output_split_sizes=rsz, input_split_sizes=[p.size for p in parts])
        out = np.empty((self.K[0], rows, Kh), dtype=np.complex128)
        off = 0
        for s in range(self.P):
            a, b = self.planes[s]
            k = (b - a) * rows * Kh
            out[a:b] = recv.numpy()[off:off + 2 * k].view(np.complex128).reshape(b - a, rows, Kh)
            off += 2 * k
        return out

    def to_slabs(self, pencils: np.ndarray) -> np.ndarray:
        """The inverse of ``to_pencils``: (K0, M1b-M1a, Kh) -> (P1-P0, K1, Kh)."""
        import torch
        dist = _dist()
        K0, rows, Kh = pencils.shape
        parts = [np.ascontiguousarray(pencils[a:b]).view(np.float64).reshape(-1)
                 for a, b in self.planes]
        n_p = self.P1 - self.P0
        rsz = [n_p * (self.M1[s + 1] - self.M1[s]) * Kh * 2 for s in range(self.P)]
        recv = torch.empty(sum(rsz), dtype=torch.float64)
        dist.all_to_all_single(recv, torch.from_numpy(np.concatenate(parts)),
                               output_split_sizes=rsz, input_split_sizes=[p.size for p in parts])
        out = np.empty((n_p, self.K[1], Kh), dtype=np.complex128)
        off = 0
        for s in range(self.P):
            m = self.M1[s + 1] - self.M1[s]
            k = n_p * m * Kh
            out[:, self.M1[s]:self.M1[s + 1], :] = \
                recv.numpy()[off:off + 2 * k].view(np.complex128).reshape(n_p, m, Kh)
            off += 2 * k
        return out

    def lower_planes(self, slab: np.ndarray, n: int) -> np.ndarray:
        """The n mesh planes just below this rank's first plane (held by the
        lower neighbours; periodic), for the interpolation of this slab's
        atoms: each rank sends its top planes up."""
        K0 = self.K[0]
        want = [(self.P0 - n + j) % K0 for j in range(n)]
        # every rank asks for the planes below it; serve the requests that
        # fall in this rank's planes (identical bookkeeping on all ranks)
        parts = []
        for d in range(self.P):
            p0 = self.planes[d][0]
            rows = [(p0 - n + j) % K0 for j in range(n)]
            mine = [p - self.P0 for p in rows if self.P0 <= p < self.P1]
            parts.append(slab[mine].reshape(len(mine), -1) if mine
                         else np.zeros((0, slab[0].size)))
        got = self.alltoallv(parts)
        # arrivals by source rank: map them back to the requested planes
        out = np.empty((n,) + slab.shape[1:])
        k = 0
        for s in range(self.P):
            a, b = self.planes[s]
            for j, p in enumerate(want):
                if a <= p < b:
                    out[j] = got[k].reshape(slab.shape[1:])
                    k += 1
        return out


def slab_widths_ok(box, rlist: float, world_size: int) -> bool:
    """True when x slabs of this box for world_size ranks are at least
    cutoff + skin wide (the condition ``Slabs`` checks)."""
    return world_size == 1 or float(box[0]) / world_size >= rlist - 1e-12


def max_ranks(box, rlist: float) -> int:
    """The most ranks an x-slab decomposition of this box supports."""
    return max(1, int(math.floor(float(box[0]) / rlist)))
