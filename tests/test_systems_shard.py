"""Independent systems split over several GPUs (the uneven workload under torchrun), on the CPU.

Each rank computes the split from the systems' estimated costs alone (no exchange), so two gloo ranks must arrive at
complementary shards: together every system exactly once, with balanced totals.
"""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from pargemslr_b200.systems import shard_systems  # noqa: E402


def _costs():
    rng = np.random.default_rng(11)
    g = np.exp(rng.uniform(np.log(32), np.log(512), size=512)).astype(int)
    return [float(v) ** 3 for v in g]


def test_shards_cover_every_system_once_and_balance():
    costs = _costs()
    for world in (1, 2, 3, 8):
        parts = shard_systems(costs, world)
        flat = sorted(k for part in parts for k in part)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[k] for k in part) for part in parts]
        # greedy largest-first: no GPU exceeds another by more than the largest single system
        assert max(loads) - min(loads) <= max(costs)
        assert shard_systems(costs, world) == parts  # deterministic


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    mine = shard_systems(_costs(), world)[rank]
    got = [None] * world
    dist.all_gather_object(got, mine)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, got))


def test_two_ranks_agree_on_complementary_shards():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, got in res:
        assert sorted(got[0] + got[1]) == list(range(512))
        assert not set(got[0]) & set(got[1])
    assert res[0][1] == res[1][1]
