"""Host logic of the sharded forms, on CPU: placement of systems on ranks and
the end-of-segment scalar gather, run as two gloo ranks (no GPU)."""
import os
import socket

import numpy as np
import pytest

from atomiverse_b200 import shard


def test_assign_is_complete_disjoint_and_balanced():
    rng = np.random.default_rng(2029)
    sizes = np.round(np.exp(rng.uniform(np.log(256), np.log(32768), 512))).astype(int).tolist()
    for ws in (1, 2, 3, 8):
        owned = shard.assign(sizes, ws)
        flat = sorted(k for o in owned for k in o)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[k] for k in o) for o in owned]
        assert max(loads) <= min(loads) + max(sizes)
        assert owned == shard.assign(sizes, ws)      # same on every rank


def test_assign_edge_cases():
    assert shard.assign([], 4) == [[], [], [], []]
    assert shard.assign([5], 3) == [[0], [], []]
    with pytest.raises(ValueError):
        shard.assign([1, 2], 0)


def test_route_request_least_loaded():
    loads = [0, 0]
    ranks = [shard.route_request(k, n, loads) for k, n in enumerate([100, 50, 60, 10])]
    assert ranks == [0, 1, 1, 0]
    assert loads == [110, 110]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, sizes, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    try:
        mine = shard.owned_by(rank, sizes, ws)
        # stand-in for the per-system scalars a rank's batch would report
        local = {k: {"energy": -float(sizes[k]), "rank": rank} for k in mine}
        merged = shard.gather_scalars(local)
        if rank == 0:
            q.put(merged)
    finally:
        dist.destroy_process_group()


def test_gather_scalars_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    sizes = [300, 1200, 800, 256, 5000, 40, 777]
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(merged) == list(range(len(sizes)))
    owned = shard.assign(sizes, 2)
    for k, v in merged.items():
        assert v["energy"] == -float(sizes[k])
        assert k in owned[v["rank"]]


def test_rebalance_plan():
    held = [[(1, 5000), (2, 3000), (3, 2000)], [(4, 500)], []]
    moves = shard.rebalance(held)
    loads = [sum(a for _, a in h) for h in held]
    atoms = {rid: a for h in held for rid, a in h}
    for rid, src, dst in moves:
        loads[src] -= atoms[rid]
        loads[dst] += atoms[rid]
    assert max(loads) - min(loads) <= 5000
    assert max(loads) < 10000
    assert moves == shard.rebalance(held)            # same plan on every rank
    assert shard.rebalance([[(1, 100)], [(2, 100)]]) == []


def _migrate_worker(rank, ws, port, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank 0 holds three requests, rank 1 none; blobs stand in for checkpoints
        held = [[(10, 4000), (11, 3000), (12, 2500)], []]
        rng = np.random.default_rng(rank + 7)
        mine = {rid: bytes(rng.integers(0, 256, size=1000 + rid, dtype=np.uint8))
                for rid, _ in held[rank]}
        moves = shard.rebalance(held)
        outgoing = {rid: mine[rid] for rid, src, _ in moves if src == rank}
        got = shard.exchange_checkpoints(moves, outgoing)
        q.put((rank, moves, {k: v.hex() for k, v in got.items()},
               {k: v.hex() for k, v in mine.items()}))
    finally:
        dist.destroy_process_group()


def test_checkpoint_migration_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_migrate_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        rank, moves, got, mine = q.get(timeout=120)
        res[rank] = (moves, got, mine)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    moves = res[0][0]
    assert moves and all(src == 0 and dst == 1 for _, src, dst in moves)
    for rid, _, _ in moves:
        assert res[1][1][rid] == res[0][2][rid]        # the bytes arrived intact
    assert res[0][1] == {}
