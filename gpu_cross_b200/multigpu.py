"""Several GPUs on one cross-section: the grid-range split.

Grid points are independent sums over the lines within the cut, so N ranks
(one process per GPU) each take a contiguous range of whole 256-point tiles,
balanced by estimated line-evals (xs_split_grid), and only the lines whose
window can reach that range.  Each rank computes its slice with the engine --
no reduction, no data-path exchange during the computation -- and the slices
are concatenated by one all-gather over torch.distributed (NCCL between GPUs,
gloo on CPU).  The reference instead splits the transitions over GPUs and
sums whole grids on the host (MultiGPUManager.cpp:61-83).

  part = split(nu_host, grid_f0, df, npoints, cut, world, rank)
  local = execute_slice(engine, opts, conds, dev_lines, dev_freq, part)
  sigma = gather_slices(local, part, npoints)       # every rank, (ncond, npoints)
"""
from __future__ import annotations

from . import capi


def split(nu, f0: float, df: float, npoints: int, cut: float, world: int, rank: int) -> dict:
    """This rank's grid points [start, start + points) and lines [l0, l1)."""
    return capi.split_grid(nu, f0, df, npoints, cut, world, rank)


def execute_slice(engine: "capi.Engine", opts, conds, dev_lines: dict, dev_freq, part: dict):
    """The rank's slice for every condition: a (ncond, points) float64 tensor
    on the lines' device (the full grid array is passed; the engine evaluates
    the chunk [start, start + points) of it with the lines [l0, l1))."""
    import torch

    ncond = len(conds)
    out = torch.zeros((ncond, max(part["points"], 1)), dtype=torch.float64, device=dev_freq.device)
    if part["points"] == 0 or part["l1"] <= part["l0"]:
        return out[:, :part["points"]]
    sub = {k: v[part["l0"]:part["l1"]] for k, v in dev_lines.items()}
    # the engine writes out[c][start + j]: shift the output pointer back by
    # start so that the rank's buffer holds just its slice
    base = out.data_ptr() - 8 * part["start"]
    engine.execute(opts, conds, capi.make_lines(sub),
                   capi.make_grid(dev_freq, part["start"], part["points"]), base,
                   out.shape[1] if ncond > 1 else None)
    engine.sync()
    return out


def gather_slices(local, part: dict, npoints: int, group=None):
    """All-gather of every rank's (ncond, points) slice into the whole
    (ncond, npoints) grid on every rank."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    ncond = local.shape[0]
    meta = torch.tensor([part["start"], part["points"]], dtype=torch.int64, device=local.device)
    metas = [torch.zeros_like(meta) for _ in range(world)]
    dist.all_gather(metas, meta, group=group)
    spans = [(int(m[0]), int(m[1])) for m in metas]
    width = max(1, max(p for _, p in spans))
    buf = torch.zeros((ncond, width), dtype=local.dtype, device=local.device)
    buf[:, :part["points"]] = local[:, :part["points"]]
    bufs = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(bufs, buf, group=group)
    full = torch.zeros((ncond, npoints), dtype=local.dtype, device=local.device)
    covered = 0
    for (s, p), b in zip(spans, bufs):
        if p:
            full[:, s:s + p] = b[:, :p]
            covered += p
    if covered != npoints:
        raise RuntimeError(f"grid split covers {covered} of {npoints} points")
    return full
