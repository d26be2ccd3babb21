"""CGLS across ranks (world_size 2 over gloo on CPU): each rank holds part of the
shots, the gradient and the norms are all-reduced, and the result equals one
process running CGLS over every shot.  A linear stand-in replaces the Born
operators (no GPU)."""
import importlib
import os
import socket
import sys

import numpy as np
import torch
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = "2d_and_3d_elastic_reverse_time_migration_b200"
SHAPE = (6, 1, 7)
NSHOTS, NT, NREC = 5, 9, 4


def _lsrtm():
    if REPO not in sys.path:
        sys.path.insert(0, REPO)
    return importlib.import_module(PKG + ".lsrtm")


class FakeCfg:
    shape = SHAPE


class FakeBorn:
    """d_s = A_s m for shot s (A_s: random dense maps), with the exact transpose."""

    def __init__(self):
        rng = np.random.default_rng(5)
        n = 3 * int(np.prod(SHAPE))
        self.A = [rng.standard_normal((3 * NT * NREC, n)) for _ in range(NSHOTS)]
        self.cfg = FakeCfg()

    def born_forward(self, s, *m):
        x = np.concatenate([a.ravel() for a in m]).astype(np.float64)
        return (self.A[s] @ x).reshape(3, NT, NREC).astype(np.float32)

    def born_adjoint(self, s, r):
        g = self.A[s].T @ r.astype(np.float64).ravel()
        n = int(np.prod(SHAPE))
        return tuple(g[q * n:(q + 1) * n].reshape(SHAPE).astype(np.float32) for q in range(3))


def _data(ctx):
    true = [np.random.default_rng(9 + q).standard_normal(SHAPE).astype(np.float32) for q in range(3)]
    return [ctx.born_forward(s, *true) for s in range(NSHOTS)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    L = _lsrtm()
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ctx = FakeBorn()
        data = _data(ctx)
        mine = [s for s in range(NSHOTS) if s % world == rank]
        res = L.cgls(ctx, mine, [data[s] for s in mine], niter=6)
        torch.save({"misfit": res.misfit, "m": [torch.from_numpy(x) for x in res.m]},
                   f"{out}/r{rank}.pt")
    finally:
        dist.destroy_process_group()


def test_distributed_cgls_equals_single_process(tmp_path):
    L = _lsrtm()
    ctx = FakeBorn()
    data = _data(ctx)
    ref = L.cgls(ctx, list(range(NSHOTS)), data, niter=6)
    assert ref.misfit[-1] < 0.5 * ref.misfit[0]
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        got = torch.load(f"{tmp_path}/r{r}.pt")
        assert np.allclose(got["misfit"], ref.misfit, rtol=1e-4)
        for a, b in zip(got["m"], ref.m):
            assert np.allclose(a.numpy(), b, rtol=1e-3, atol=1e-5 * np.abs(b).max())


def _avg_worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    if REPO not in sys.path:
        sys.path.insert(0, REPO)
    nn = importlib.import_module(PKG + ".nn")
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        g = [torch.full((3, 4), float(rank + 1)), torch.arange(5, dtype=torch.float32) * (rank + 1)]
        nn.average_gradients(g)
        torch.save(g, f"{out}/g{rank}.pt")
    finally:
        dist.destroy_process_group()


def test_unet_gradient_averaging_over_two_ranks(tmp_path):
    mp.spawn(_avg_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        g = torch.load(f"{tmp_path}/g{r}.pt")
        assert torch.allclose(g[0], torch.full((3, 4), 1.5))
        assert torch.allclose(g[1], torch.arange(5, dtype=torch.float32) * 1.5)
