"""bench.py --gpus N runs N independent replicas (one system per rank, no
collective on the data path): the timing is the max over ranks and the
value the whole job's steps/s.  The host side of that path on two gloo
ranks on the CPU (the GPU runs use NCCL with the same calls)."""
import datetime
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, local_ms, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        m = bench.reduce_max(local_ms[rank], dist, "cpu")
        v = bench.replica_throughput(m, world)
        # the reference arm: rank 0 alone works and prints, the others return at once
        ref = bench.run_reference(None, rank, world) if rank != 0 else "rank0"
        dist.barrier()
        out.put((rank, m, v, ref))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_take_the_max_and_sum_the_replicas():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    local_ms = [3.0, 5.0]
    procs = [ctx.Process(target=_worker, args=(r, 2, port, local_ms, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=100) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for rank, m, v, ref in res:
        assert m == 5.0                    # the slowest rank sets the step time
        assert v == pytest.approx(400.0)   # 2 replicas x 1000 / 5 ms
    assert res[1][3] is None               # rank 1 of the reference arm does no work


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max(2.5) == 2.5
    assert bench.replica_throughput(2.5, 1) == pytest.approx(400.0)
