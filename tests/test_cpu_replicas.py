"""The multi-GPU form of the PIC step is "replicas only": each rank runs an
independent copy and the job time is the slowest rank's. These checks run
the bench's reduction with two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms = [10.0, 25.0][rank]
    m = bench.max_over_ranks(ms, world, "cpu")
    v = bench.replica_throughput(m, world)
    q.put((rank, m, v))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, m, v in out:
        assert m == 25.0
        assert v == pytest.approx(2 * 1000.0 / 25.0)


def test_single_rank_passthrough():
    import bench
    assert bench.max_over_ranks(12.5, 1, "cpu") == 12.5
    assert bench.replica_throughput(20.0, 1) == pytest.approx(50.0)
