"""Multi-GPU placement for the batched and served forms.

One MD system of the sizes this library targets does not shard without
domain decomposition, so a single system runs on one GPU and N GPUs run
independent work.  The replica ladder and the request stream partition by
system: each rank owns whole systems, its step has no collective, and the
only exchange is a host gather of per-system scalars at the end of a
segment (``gather_scalars``).  One process per GPU, ``torch.distributed``
for the plumbing (NCCL on GPUs; gloo works the same for these host objects).
"""
from __future__ import annotations

import heapq


def assign(sizes: list[int], world_size: int) -> list[list[int]]:
    """Greedy longest-first placement of systems on ranks by atom count.

    Returns, for every rank, the sorted indices of the systems it owns.  The
    result depends only on ``sizes`` and ``world_size`` (ties broken by
    index, then by rank), so every rank computes the same placement without
    communicating.  The heaviest rank carries at most the lightest rank's
    load plus one system.
    """
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k))
    heap = [(0, r) for r in range(world_size)]
    owned: list[list[int]] = [[] for _ in range(world_size)]
    for k in order:
        load, r = heapq.heappop(heap)
        owned[r].append(k)
        heapq.heappush(heap, (load + int(sizes[k]), r))
    return [sorted(o) for o in owned]


def owned_by(rank: int, sizes: list[int], world_size: int) -> list[int]:
    """Indices of the systems that ``rank`` owns."""
    return assign(sizes, world_size)[rank]


def route_request(request_index: int, n_atoms: int, loads: list[int]) -> int:
    """Rank for a newly arrived request: the one with the fewest resident
    atoms (ties to the lowest rank).  ``loads`` is updated in place."""
    r = min(range(len(loads)), key=lambda q: (loads[q], q))
    loads[r] += int(n_atoms)
    return r


def gather_scalars(local: dict, group=None, dst: int = 0) -> dict | None:
    """Host gather of ``{system index: scalars}`` from every rank to ``dst``.

    The one exchange of the sharded forms; returns the merged dict on
    ``dst`` and None elsewhere.  Every rank must call it (collective)."""
    import torch.distributed as dist
    ws = dist.get_world_size(group)
    rank = dist.get_rank(group)
    parts = [None] * ws if rank == dst else None
    dist.gather_object(local, parts, dst=dst, group=group)
    if rank != dst:
        return None
    merged: dict = {}
    for p in parts:
        for k, v in p.items():
            if k in merged:
                raise RuntimeError(f"system {k} reported by two ranks")
            merged[k] = v
    return merged


def run_ladder_rank(ctx, items: list, n_steps: int, rank: int, world_size: int,
                    autotune: bool = True) -> dict:
    """Advance this rank's share of a replica ladder as one batch on its GPU
    and return ``{system index: scalars}`` for ``gather_scalars``."""
    import atomiverse_b200 as A
    mine = owned_by(rank, [d["n_atoms"] for d, _ in items], world_size)
    if not mine:
        return {}
    b = A.Batch(ctx, [items[k] for k in mine])
    if autotune:
        b.autotune()
    b.compute_forces()
    b.step(n_steps)
    out = {}
    for j, k in enumerate(mine):
        _, sc = b.download(j, keys=())
        out[k] = {key: (v.tolist() if hasattr(v, "tolist") else v) for key, v in sc.items()}
    b.close()
    return out
