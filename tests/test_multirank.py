"""The N > 1 path on CPU: two gloo ranks each build their own (T, P) batch
(weak scaling, independent objects, no data-path collective) and agree on
the max-over-ranks step time, as bench.py does over NCCL on GPUs."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import torch

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        _, _, conds, _ = bench.sweep_workload(2000, 1000, rank)
        mine = torch.tensor([100.0 + 7.0 * rank], dtype=torch.float64)  # this rank's time
        dist.all_reduce(mine, op=dist.ReduceOp.MAX)
        q.put((rank, conds[0]["temperature"], float(mine.item()), len(conds)))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_independent_batches_and_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    # each rank has its own 40-condition batch (shifted temperatures)
    assert res[0][1] != res[1][1] and res[0][3] == res[1][3] == 40
    # both see the max over ranks
    assert res[0][2] == res[1][2] == pytest.approx(107.0)
