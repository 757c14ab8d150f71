"""Multi-process (world size 2, gloo, CPU) tests of the replica host logic
used by bench.py --gpus N: timing aggregation (max over ranks), whole-job
throughput, request sharding."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "MASTER_ADDR": "127.0.0.1",
                       "MASTER_PORT": str(port)})
    import torch.distributed as dist
    from vqcb200 import replicas
    try:
        r, w = replicas.init_from_env("gloo")
        assert (r, w) == (rank, world)
        replicas.barrier()
        ms_local = 10.0 * (rank + 1)  # rank 1 is the slowest
        thr, ms = replicas.whole_job_throughput(units_per_rank=5, ms_local=ms_local)
        share = replicas.shard(list(range(11)), rank, world)
        q.put((rank, thr, ms, share))
    finally:
        if dist.is_initialized():
            dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_replica_aggregation():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=90) for _ in range(world))
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for rank, thr, ms, share in res:
        assert ms == 20.0                       # max over ranks
        assert abs(thr - 10 / 0.020) < 1e-9     # 2 ranks x 5 units / slowest 20 ms
    shares = [share for _, _, _, share in res]
    assert sorted(shares[0] + shares[1]) == list(range(11))
    assert not set(shares[0]) & set(shares[1])


def test_single_process_needs_no_group():
    from vqcb200 import replicas
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.shard([1, 2, 3], 0, 1) == [1, 2, 3]
