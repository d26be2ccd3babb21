"""Least-squares RTM: conjugate gradients on the Born normal equations.

Solves  min_m 0.5 sum_shots |F_s m - d_s|^2  for the relative perturbations
m = (r_vp, r_vs, r_rho) of the migration model, with F_s the Born operator of
shot s (`Context.born_forward`) and F_s^T its exact adjoint
(`Context.born_adjoint`).  The reference's LSRTM driver loop is absent from its
tree; its kernels (Born "demig", adjoint, gradient) are what these operators
restate.

`precond` (optional) maps a gradient (3 volumes) to a search direction; it is
used as in preconditioned CGLS, and a preconditioned step is accepted only if
the Born-modelled data misfit falls, otherwise the plain CG step of the same
iteration is taken instead (plain CG is the fallback).

`state` (optional) is a path prefix for the iteration state (model, residual,
gradient, direction, scalars and history), written after every iteration —
one file per rank, replaced atomically — and read back at the start, so an
interrupted run continues from its last finished iteration with the same
numbers as an uninterrupted one.  `log` (optional) is a JSON-lines file that
gets one record per iteration (misfit, step kind, seconds).
"""
from __future__ import annotations

import json
import os
import time
from dataclasses import dataclass, field
from typing import Callable, Sequence

import numpy as np


@dataclass
class CGResult:
    m: tuple                      # (r_vp, r_vs, r_rho), numpy arrays or CUDA tensors like the data
    misfit: list = field(default_factory=list)   # relative data misfit |r|^2/|d|^2 per iteration
    accepted: list = field(default_factory=list)  # per iteration: "precond" or "plain"


def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


def _sq(x) -> float:
    """sum of squares in float64"""
    if _is_torch(x):
        return float((x.double() ** 2).sum())
    return float(np.sum(x.astype(np.float64) ** 2))


def _dot(a: Sequence, b: Sequence) -> float:
    if a and _is_torch(a[0]):
        return float(sum((x.double() * y.double()).sum() for x, y in zip(a, b)))
    return float(sum(np.sum(x.astype(np.float64) * y) for x, y in zip(a, b)))


def _lin(alpha: float, x, y):
    """y + alpha x in float32"""
    if _is_torch(x):
        return y + alpha * x
    return (y + alpha * x).astype(np.float32)


def _to_numpy(x):
    return x.detach().cpu().numpy() if _is_torch(x) else x


class _Sum:
    """Sums over the ranks of `group` (torch.distributed; identity on one process):
    the gradient (three volumes) and the scalar norms of CGLS, so every rank holds
    the same model, direction and step after each iteration."""

    def __init__(self, group):
        import torch.distributed as dist
        self.on = dist.is_available() and dist.is_initialized() and \
            dist.get_world_size(group) > 1
        self.group = group

    def scalar(self, v: float) -> float:
        if not self.on:
            return v
        import torch
        import torch.distributed as dist
        t = torch.tensor([v], dtype=torch.float64)
        dist.all_reduce(t, group=self.group)
        return float(t.item())

    def volumes(self, g):
        if not self.on:
            return g
        import torch
        import torch.distributed as dist
        if _is_torch(g[0]):
            t = torch.stack([x.float() for x in g]).contiguous()
            if t.is_cuda and dist.get_backend(self.group) != "nccl":
                h = t.cpu()
                dist.all_reduce(h, group=self.group)
                t = h.to(g[0].device)
            else:
                dist.all_reduce(t, group=self.group)
            return tuple(t[q].clone() for q in range(len(g)))
        t = torch.from_numpy(np.stack([x.astype(np.float32) for x in g]))
        dist.all_reduce(t, group=self.group)
        return tuple(t[q].numpy().copy() for q in range(len(g)))


def _axpy(alpha: float, x, y):
    return tuple(_lin(alpha, xx, yy) for xx, yy in zip(x, y))


def _stack(arrs):
    if arrs and _is_torch(arrs[0]):
        import torch
        return torch.stack(list(arrs)).contiguous()
    return np.ascontiguousarray(np.stack(arrs), np.float32)


def born_all(ctx, shots, m):
    """Born data of every shot, stacked (nshots, 3, nt, nrec): one batched call when the
    context offers it (all shots share each step's kernel launches), else one per shot."""
    if not shots:
        return None
    if hasattr(ctx, "born_forward_shots"):
        if _is_torch(m[0]):
            import torch
            out = torch.zeros((len(shots), 3, ctx.cfg.nt, shots[0].nrec), device=m[0].device)
            # the library works on its own stream: the inputs must be complete first
            torch.cuda.current_stream(m[0].device).synchronize()
            return ctx.born_forward_shots(shots, *m, out=out)
        return ctx.born_forward_shots(shots, *m)
    return _stack([ctx.born_forward(s, *m) for s in shots])


def adjoint_all(ctx, shots, res):
    """Gradient summed over the shots for stacked residuals (nshots, 3, nt, nrec)."""
    if not shots:                      # a rank without shots contributes zero
        return tuple(np.zeros(ctx.cfg.shape, np.float32) for _ in range(3))
    if isinstance(res, (list, tuple)):
        res = _stack(res)
    if hasattr(ctx, "born_adjoint_shots"):
        if _is_torch(res):
            import torch
            g = [torch.zeros(ctx.cfg.shape, device=res.device) for _ in range(3)]
            torch.cuda.current_stream(res.device).synchronize()
            return ctx.born_adjoint_shots(shots, res, *g)
        return ctx.born_adjoint_shots(shots, res)
    g = None
    for s, r in zip(shots, res):
        gs = ctx.born_adjoint(s, r)
        g = gs if g is None else tuple(a + b for a, b in zip(g, gs))
    return tuple(x.astype(np.float32) for x in g)


def _state_file(prefix: str, group) -> str:
    import torch.distributed as dist
    rank = dist.get_rank(group) if dist.is_available() and dist.is_initialized() else 0
    return f"{prefix}.rank{rank}.npz"


def _save_state(path: str, it: int, m, r, s, p, gamma, rnorm, dnorm, out: "CGResult"):
    tmp = path + ".tmp.npz"
    arrs = {"it": np.int64(it), "gamma": np.float64(gamma), "rnorm": np.float64(rnorm),
            "dnorm": np.float64(dnorm), "misfit": np.asarray(out.misfit, np.float64),
            "accepted": np.asarray(out.accepted, dtype="U8"), "nres": np.int64(len(r))}
    for q in range(3):
        arrs[f"m{q}"], arrs[f"s{q}"], arrs[f"p{q}"] = _to_numpy(m[q]), _to_numpy(s[q]), _to_numpy(p[q])
    for k, x in enumerate(r):
        arrs[f"r{k}"] = _to_numpy(x)
    np.savez(tmp, **arrs)
    os.replace(tmp, path)


def _load_state(path: str):
    with np.load(path) as f:
        st = {k: f[k] for k in f.files}
    vol = lambda key: tuple(st[f"{key}{q}"].astype(np.float32) for q in range(3))
    return (int(st["it"]), vol("m"), [st[f"r{k}"].astype(np.float32) for k in range(int(st["nres"]))],
            vol("s"), vol("p"), float(st["gamma"]), float(st["rnorm"]), float(st["dnorm"]),
            [float(x) for x in st["misfit"]], [str(x) for x in st["accepted"]])


def cgls(ctx, shots: list, data: list, niter: int,
         precond: Callable[[tuple], tuple] | None = None,
         callback: Callable[[int, float], None] | None = None, group=None,
         state: str | None = None, log: str | None = None) -> CGResult:
    """CGLS on this rank's shots; with torch.distributed initialised, the ranks of
    `group` each pass their own shots and data, and the gradient (one all-reduce of
    three volumes per iteration) and the norms are summed over them.  The data may be
    numpy arrays or CUDA tensors: with CUDA tensors every CG vector (model, residual,
    gradient, direction) stays on the device.  `state` and `log`: see the module
    docstring."""
    red = _Sum(group)
    shape = ctx.cfg.shape
    on_dev = bool(data) and _is_torch(data[0])
    if on_dev:
        import torch
        dev = data[0].device
        zeros = lambda: torch.zeros(shape, device=dev)
        asarr = lambda x: torch.as_tensor(x, device=dev).float()
    else:
        zeros = lambda: np.zeros(shape, np.float32)
        asarr = lambda x: np.asarray(x, np.float32)
    out = CGResult(m=None)
    path = _state_file(state, group) if state else None
    start = 0
    have = path is not None and os.path.exists(path)
    # every rank resumes, or none does (the ranks must take the same steps)
    if state and red.on and red.scalar(1.0 if have else 0.0) not in (0.0, float(_world(group))):
        raise RuntimeError(f"CG state {state!r}: some ranks have a state file and some do not")
    if have:
        start, m, r, s, p, gamma, rnorm, dnorm, out.misfit, out.accepted = _load_state(path)
        if len(r) != len(data):
            raise RuntimeError(f"CG state {path!r} holds {len(r)} residuals for {len(data)} shots")
        if red.on and red.scalar(float(start)) != float(start) * _world(group):
            raise RuntimeError(f"CG state {state!r}: ranks stopped at different iterations")
        m, s, p = (tuple(asarr(x) for x in v) for v in (m, s, p))
        r = _stack([asarr(x) for x in r]) if r else None
    else:
        m = tuple(zeros() for _ in range(3))
        r = _stack([d.float().clone() if on_dev else d.astype(np.float32).copy() for d in data]) \
            if data else None                                    # r = d - F m, (nshots, 3, nt, nrec)
        dnorm = red.scalar(sum(_sq(d) for d in data))
        s = red.volumes(adjoint_all(ctx, shots, r))
        z = precond(s) if precond else s
        p = z
        gamma = _dot(s, z)
        rnorm = dnorm
    out.m = m
    for it in range(start, niter):
        t0 = time.perf_counter()
        q = born_all(ctx, shots, p)
        qq = red.scalar(_sq(q) if q is not None else 0.0)
        if qq == 0.0 or gamma == 0.0:
            break
        alpha = gamma / qq
        r_new = _lin(-alpha, q, r) if r is not None else None
        rn = red.scalar(_sq(r_new) if r_new is not None else 0.0)
        kind = "precond" if precond else "plain"
        if precond and rn >= rnorm:
            # safeguard: the preconditioned direction did not lower the misfit;
            # restart from the plain gradient direction
            p = s
            gamma = _dot(s, s)
            q = born_all(ctx, shots, p)
            qq = red.scalar(_sq(q) if q is not None else 0.0)
            alpha = gamma / qq
            r_new = _lin(-alpha, q, r) if r is not None else None
            rn = red.scalar(_sq(r_new) if r_new is not None else 0.0)
            kind = "plain"
        m = _axpy(alpha, p, m)
        r, rnorm = r_new, rn
        s = red.volumes(adjoint_all(ctx, shots, r))
        z = precond(s) if (precond and kind == "precond") else s
        gamma_new = _dot(s, z)
        beta = gamma_new / gamma if gamma else 0.0
        p = _axpy(beta, p, z)
        gamma = gamma_new
        out.misfit.append(rnorm / dnorm)
        out.accepted.append(kind)
        if path:
            _save_state(path, it + 1, m, list(r) if r is not None else [], s, p, gamma, rnorm, dnorm, out)
        if log:
            with open(log, "a") as f:
                f.write(json.dumps({"event": "cg_iteration", "iteration": it, "misfit": rnorm / dnorm,
                                    "step": kind, "seconds": round(time.perf_counter() - t0, 6)}) + "\n")
        if callback:
            callback(it, rnorm / dnorm)
    out.m = m
    return out


def _world(group) -> int:
    import torch.distributed as dist
    return dist.get_world_size(group)
