"""CG iteration state: an LSRTM run stopped after some iterations and started
again from its state files gives the same model and misfit history as one run
straight through — in one process, and with the shots split over two gloo ranks
(linear stand-in for the Born operators, no GPU).  Also the JSON-lines log."""
import datetime
import json
import os

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from test_lsrtm_dist import NSHOTS, FakeBorn, _data, _free_port, _lsrtm


def test_resume_equals_uninterrupted(tmp_path):
    L = _lsrtm()
    ctx = FakeBorn()
    data = _data(ctx)
    shots = list(range(NSHOTS))
    ref = L.cgls(ctx, shots, data, niter=6)
    state, log = str(tmp_path / "cg"), str(tmp_path / "run.jsonl")
    first = L.cgls(ctx, shots, data, niter=3, state=state, log=log)
    assert len(first.misfit) == 3 and os.path.exists(state + ".rank0.npz")
    again = L.cgls(ctx, shots, data, niter=6, state=state, log=log)
    assert again.misfit == ref.misfit and again.accepted == ref.accepted
    for a, b in zip(again.m, ref.m):
        assert np.array_equal(a, b)
    recs = [json.loads(x) for x in open(log)]
    assert [r["iteration"] for r in recs] == list(range(6))
    assert [r["misfit"] for r in recs] == ref.misfit
    # a finished state is a no-op for the same iteration count
    done = L.cgls(ctx, shots, data, niter=6, state=state)
    assert done.misfit == ref.misfit
    # a state written for other shots is refused
    with pytest.raises(RuntimeError):
        L.cgls(ctx, shots[:2], data[:2], niter=6, state=state)


def _worker(rank, world, port, out, stop):
    import torch.distributed as dist
    L = _lsrtm()
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ctx = FakeBorn()
        data = _data(ctx)
        mine = [s for s in range(NSHOTS) if s % world == rank]
        res = L.cgls(ctx, mine, [data[s] for s in mine], niter=stop, state=f"{out}/cg")
        torch.save({"misfit": res.misfit, "m": [torch.from_numpy(x) for x in res.m]},
                   f"{out}/r{rank}_{stop}.pt")
    finally:
        dist.destroy_process_group()


def test_distributed_resume(tmp_path):
    L = _lsrtm()
    ctx = FakeBorn()
    data = _data(ctx)
    ref = L.cgls(ctx, list(range(NSHOTS)), data, niter=6)
    for stop in (2, 6):
        mp.spawn(_worker, args=(2, _free_port(), str(tmp_path), stop), nprocs=2, join=True)
    for r in range(2):
        assert os.path.exists(f"{tmp_path}/cg.rank{r}.npz")
        got = torch.load(f"{tmp_path}/r{r}_6.pt")
        assert np.allclose(got["misfit"], ref.misfit, rtol=1e-4)
        for a, b in zip(got["m"], ref.m):
            assert np.allclose(a.numpy(), b, rtol=1e-3, atol=1e-5 * np.abs(b).max())
