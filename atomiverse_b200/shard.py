"""Multi-GPU placement for the batched and served forms.

One MD system of the sizes this library targets does not shard without
domain decomposition, so a single system runs on one GPU and N GPUs run
independent work.  The replica ladder and the request stream partition by
system: each rank owns whole systems, its step has no collective, and the
only exchange is a host gather of per-system scalars at the end of a
segment (``gather_scalars``).  Served requests can move between ranks
between ticks as checkpoints (``rebalance``, ``exchange_checkpoints``).  One
process per GPU, ``torch.distributed`` for the plumbing (NCCL on GPUs; gloo
works the same for these host objects).
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


def rebalance(held: list[list[tuple[int, int]]]) -> list[tuple[int, int, int]]:
    """Moves that even out the resident atoms of the served form.

    ``held[r]`` lists ``(request id, atoms)`` resident on rank r.  Returns
    ``(request id, from rank, to rank)`` moves: repeatedly the largest request
    of the heaviest rank that lowers the larger of the two loads goes to the
    lightest rank.  Deterministic (ties by id, then rank), so every rank
    computes the same plan from the same ``held``.  A request moves as its
    checkpoint (``Server.checkpoint`` -> ``exchange_checkpoints`` ->
    ``Server.submit_checkpoint``) and continues bit for bit on its new rank.
    """
    loads = [sum(a for _, a in h) for h in held]
    where = {rid: r for r, h in enumerate(held) for rid, _ in h}
    atoms = {rid: a for h in held for rid, a in h}
    moves = []
    for _ in range(sum(len(h) for h in held)):
        hi = max(range(len(loads)), key=lambda q: (loads[q], -q))
        lo = min(range(len(loads)), key=lambda q: (loads[q], q))
        best = None
        for rid in sorted((rid for rid, r in where.items() if r == hi), key=lambda x: (-atoms[x], x)):
            if max(loads[hi] - atoms[rid], loads[lo] + atoms[rid]) < loads[hi]:
                best = rid
                break
        if best is None:
            break
        loads[hi] -= atoms[best]
        loads[lo] += atoms[best]
        where[best] = lo
        moves.append((best, hi, lo))
    return moves


def exchange_checkpoints(moves: list[tuple[int, int, int]], blobs: dict, group=None) -> dict:
    """Carry the checkpoints of ``moves`` to their new ranks.

    ``blobs`` maps this rank's outgoing request ids to their checkpoint
    bytes; returns ``{request id: bytes}`` for the requests that move to this
    rank.  Every rank must call it (collective; any backend, the blobs travel
    as byte tensors of a size agreed first)."""
    import torch
    import torch.distributed as dist
    rank = dist.get_rank(group)
    incoming = {}
    for rid, src, dst in moves:
        if src == dst:
            continue
        if rank == src:
            data = torch.frombuffer(bytearray(blobs[rid]), dtype=torch.uint8)
            dist.send(torch.tensor([data.numel()], dtype=torch.int64), dst=dst, group=group)
            dist.send(data, dst=dst, group=group)
        elif rank == dst:
            n = torch.zeros(1, dtype=torch.int64)
            dist.recv(n, src=src, group=group)
            data = torch.empty(int(n.item()), dtype=torch.uint8)
            dist.recv(data, src=src, group=group)
            incoming[rid] = data.numpy().tobytes()
    return incoming


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
