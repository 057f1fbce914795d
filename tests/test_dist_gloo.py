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
