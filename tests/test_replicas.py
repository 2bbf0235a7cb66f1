"""Multi-GPU mode of bench.py on CPU: replicas with MAX-over-ranks timing.

The solve does not shard (one system per GPU), so N > 1 runs independent
replicas and the only exchange is the reduction of the timed region to its
maximum over ranks.  Here two gloo ranks check that reduction and that the
reference arm prints from rank 0 only.
"""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    got = bench.max_over_ranks(10.0 + 5.0 * rank, "cpu")
    # the reference arm runs on rank 0 only; other ranks leave without work or output
    buf = io.StringIO()
    if rank != 0:
        with redirect_stdout(buf):
            bench.run_reference(None)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, got, buf.getvalue()))


def test_max_over_ranks_and_rank0_reference_arm():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.0, 15.0]
    assert res[1][2] == ""


def test_max_over_ranks_without_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, "cpu") == 3.5
