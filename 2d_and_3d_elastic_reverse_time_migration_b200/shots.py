"""Shot-parallel RTM over several GPUs: one process per GPU, torch.distributed.

Shots are independent (the reference migrates them one after another, one
image file per shot, 3D_elastic_RTM/3D_output_file.cu:339-365).  Here each
rank migrates its share of the shot list on its own GPU with
`Context.rtm_batch` (images stacked on the device) and the per-rank stacks are
summed with one collective per image (NCCL over NVLink; gloo in the CPU tests).
A single grid is never split across GPUs.

Before the image collective every rank contributes a status word, so a rank
whose shots failed makes every rank raise `ShotFailure` (naming the failed
ranks) instead of leaving the others blocked in the reduction.
"""
from __future__ import annotations

import heapq
from dataclasses import dataclass
from typing import Callable, Sequence


class ShotFailure(RuntimeError):
    def __init__(self, failed_ranks: list[int], message: str = ""):
        super().__init__(f"shot migration failed on rank(s) {failed_ranks}: {message}")
        self.failed_ranks = failed_ranks


def shot_cost(cells: int, nt: int, src_steps: int = 0) -> float:
    """Work of one RTM shot in cell-updates (source pass + receiver pass)."""
    return float(cells) * ((src_steps or 2 * nt // 3) + nt)


def plan(costs: Sequence[float], world: int) -> list[list[int]]:
    """Longest-processing-time assignment of shots to `world` ranks: every shot
    exactly once, the most expensive first onto the least loaded rank; ties go to
    the lower rank, so every rank computes the same plan."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0.0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    for lst in out:
        lst.sort()
    return out


@dataclass
class StackResult:
    pp: object
    ps: object
    tp: object
    my_shots: list


def migrate(local: Callable[[list[int]], tuple], nshots: int, costs: Sequence[float] | None = None,
            group=None, dst: int | None = None) -> StackResult:
    """Migrate `nshots` shots across the ranks of `group`.

    `local(indices)` migrates the given shots on this rank and returns its
    stacked (pp, ps, tp) tensors (e.g. a closure over `Context.rtm_batch`).  The
    stacks are summed with all_reduce (or reduce to `dst`).  Raises ShotFailure
    on every rank if any rank's `local` raised."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    costs = list(costs) if costs is not None else [1.0] * nshots
    if len(costs) != nshots:
        raise ValueError("one cost per shot")
    mine = plan(costs, world)[rank]
    err = ""
    imgs = None
    try:
        imgs = local(mine)
    except Exception as e:  # reported to every rank below
        err = f"{type(e).__name__}: {e}"
    if world > 1:
        dev = imgs[0].device if imgs is not None else (
            torch.device("cuda", torch.cuda.current_device())
            if dist.get_backend(group) == "nccl" else torch.device("cpu"))
        flags = torch.zeros(world, dtype=torch.int32, device=dev)
        flags[rank] = 1 if err else 0
        dist.all_reduce(flags, group=group)
        failed = [r for r in range(world) if int(flags[r]) != 0]
        if failed:
            raise ShotFailure(failed, err)
        for t in imgs:
            if dst is None:
                dist.all_reduce(t, group=group)
            else:
                dist.reduce(t, dst=dst, group=group)
    elif err:
        raise ShotFailure([0], err)
    return StackResult(*imgs, my_shots=mine)


def context_local(ctx, shots: list, data: list) -> Callable[[list[int]], tuple]:
    """`local` callable for `migrate` over a Context: stacks on the context's GPU."""
    import torch

    def run(idx: list[int]):
        dev = torch.device("cuda", ctx.cfg.device)
        outs = [torch.zeros(ctx.cfg.shape, dtype=torch.float32, device=dev) for _ in range(3)]
        if idx:
            ctx.rtm_batch([shots[i] for i in idx], [data[i] for i in idx], *outs)
        return tuple(outs)

    return run
