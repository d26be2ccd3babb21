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

`migrate_shots` runs shot by shot: with a `ShotCache` every finished shot's
images go to their own file (the reference's restart unit is also the per-shot
image file), so a run that stopped resumes at the shots that have no file yet;
with `skip_failed` a shot that raises is left out of the stack and reported
(shot index and message, gathered from every rank) instead of failing the run.
"""
from __future__ import annotations

import heapq
import os
from dataclasses import dataclass, field
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
    failed: list = field(default_factory=list)   # (shot, message), every rank's (migrate_shots)


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


class ShotCache:
    """Per-shot images (pp, ps, tp) on disk, one `.npz` file per shot, written to a
    temporary name and renamed, so a file that exists is complete."""

    def __init__(self, directory: str):
        self.dir = directory
        os.makedirs(directory, exist_ok=True)

    def path(self, shot: int) -> str:
        return os.path.join(self.dir, f"shot{shot:06d}.npz")

    def has(self, shot: int) -> bool:
        return os.path.exists(self.path(shot))

    def load(self, shot: int):
        import numpy as np
        with np.load(self.path(shot)) as f:
            return f["pp"], f["ps"], f["tp"]

    def save(self, shot: int, imgs) -> None:
        import numpy as np
        host = [x.detach().cpu().numpy() if hasattr(x, "detach") else np.asarray(x) for x in imgs]
        tmp = self.path(shot) + ".tmp.npz"
        np.savez(tmp, pp=host[0], ps=host[1], tp=host[2])
        os.replace(tmp, self.path(shot))


def migrate_shots(one_shot: Callable[[int], tuple], nshots: int, shape, costs: Sequence[float] | None = None,
                  group=None, dst: int | None = None, cache: ShotCache | None = None,
                  skip_failed: bool = False, device=None) -> StackResult:
    """`migrate` shot by shot: `one_shot(i)` returns shot i's (pp, ps, tp) tensors of
    `shape`; cached shots are loaded instead of migrated and new ones are saved;
    with `skip_failed` a shot that raises is reported in `StackResult.failed` (on
    every rank) and left out of the stack, otherwise the run fails as in `migrate`."""
    import torch
    import torch.distributed as dist

    if device is None:
        device = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() \
            else torch.device("cpu")
    failed_here: list = []

    def local(idx):
        acc = [torch.zeros(tuple(shape), dtype=torch.float32, device=device) for _ in range(3)]
        for i in idx:
            if cache is not None and cache.has(i):
                imgs = [torch.from_numpy(x).to(device) for x in cache.load(i)]
            else:
                try:
                    imgs = one_shot(i)
                except Exception as e:
                    if not skip_failed:
                        raise
                    failed_here.append((i, f"{type(e).__name__}: {e}"))
                    continue
                if cache is not None:
                    cache.save(i, imgs)
            for a, x in zip(acc, imgs):
                a += torch.as_tensor(x, device=device).reshape(a.shape)
        return tuple(acc)

    res = migrate(local, nshots, costs, group=group, dst=dst)
    failed = list(failed_here)
    if dist.is_initialized() and dist.get_world_size(group) > 1:
        lists = [None] * dist.get_world_size(group)
        dist.all_gather_object(lists, failed_here, group=group)
        failed = [tuple(f) for lst in lists for f in lst]
    res.failed = sorted(failed)
    return res


def context_shot(ctx, shots: list, data: list) -> Callable[[int], tuple]:
    """`one_shot` callable for `migrate_shots` over a Context (images on its GPU)."""
    import torch

    def run(i: int):
        dev = torch.device("cuda", ctx.cfg.device)
        outs = [torch.zeros(ctx.cfg.shape, dtype=torch.float32, device=dev) for _ in range(3)]
        ctx.rtm_shot(shots[i], data[i], *outs)
        return tuple(outs)

    return run
