"""The N > 1 path on CPU: two gloo ranks each build their own (T, P) batch
(weak scaling, independent objects, no data-path collective) and agree on
the max-over-ranks step time, as bench.py does over NCCL on GPUs."""
import os
import socket

import numpy as np
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


def _split_case():
    from gpu_cross_b200 import synth

    lines = synth.random_lines(6000, 1000.0, 1200.0, 2500.0, 1e-6, 1e2, seed=77, pressure_atm=0.5)
    # denser lines in one part of the band, so that equal work is not equal points
    more = synth.random_lines(6000, 1040.0, 1060.0, 2500.0, 1e-6, 1e2, seed=78, pressure_atm=0.5)
    both = synth.LineList(*(np.concatenate([getattr(lines, f), getattr(more, f)])
                            for f in ("nu", "energies", "aif", "gns", "gamma", "n")))
    order = np.argsort(both.nu, kind="stable")
    both = synth.LineList(*(getattr(both, f)[order] for f in ("nu", "energies", "aif", "gns",
                                                               "gamma", "n")))
    grid = synth.Grid(990.0, 1210.0, 22000)
    cond = dict(temperature=900.0, partition=synth.partition_poly(900.0), mean_mass=17.03,
                pressure=1.0, ref_temp=296.0)
    return both, grid, cond


def _split_worker(rank, world, port, q):
    import torch

    import oracle
    from gpu_cross_b200 import multigpu

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        lines, grid, cond = _split_case()
        fr = grid.freq()
        part = multigpu.split(lines.nu, fr[0], grid.dfreq, grid.npoints, 25.0, world, rank)
        s, p = part["start"], part["points"]
        # The oracle restates the reference kernel's summation order, which
        # hands line i to thread i mod 128 (cross_kernal.cu:924-997): a slice
        # that starts on a multiple of 128 keeps every point's order.
        l0 = part["l0"] - part["l0"] % 128
        full = oracle.gpu_convention(oracle.VOIGT, fr, np.zeros_like(fr),
                                     lines.slice(l0, part["l1"]), cond, grid.dfreq,
                                     points=p, start_idx=s)
        local = torch.from_numpy(np.ascontiguousarray(full[s:s + p]))[None, :]
        gathered = multigpu.gather_slices(local, part, grid.npoints)
        q.put((rank, part, gathered.numpy()[0]))
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_grid_split_gathers_the_one_rank_result(built_libs, world):
    """Grid-range split over gloo ranks: each rank evaluates only its tiles
    with only the lines that reach them (here through the oracle), one
    all-gather concatenates the slices, and every rank holds exactly the
    1-rank result -- bit for bit, since each point sums the same lines in
    the same order."""
    import oracle

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_split_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    lines, grid, cond = _split_case()
    fr = grid.freq()
    want = oracle.gpu_convention(oracle.VOIGT, fr, np.zeros_like(fr), lines, cond, grid.dfreq)
    parts = [r[1] for r in res]
    # contiguous whole tiles in rank order, covering the grid
    pos = 0
    for part in parts:
        assert part["start"] == pos and part["start"] % 256 == 0
        pos += part["points"]
        assert part["l1"] - part["l0"] < len(lines)  # a line subset, not the whole list
    assert pos == grid.npoints
    # balanced by work, not by points: the dense band shifts the boundaries
    work = [part["pairs"] for part in parts]
    assert max(work) < 1.25 * (sum(work) / world)
    for _, _, got in res:
        assert np.array_equal(got, want)
