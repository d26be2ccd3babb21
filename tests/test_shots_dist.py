"""Shot-parallel migration across ranks: plan, stacking and failure reporting
(world_size 2 over gloo on CPU; the GPU work is replaced by a stand-in)."""
import importlib
import os
import socket
import sys

import pytest
import torch
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = "2d_and_3d_elastic_reverse_time_migration_b200"


def _shots():
    if REPO not in sys.path:
        sys.path.insert(0, REPO)
    return importlib.import_module(PKG + ".shots")


def test_plan_covers_every_shot_once_and_balances():
    S = _shots()
    costs = [S.shot_cost(cells, nt) for cells, nt in
             [(10_000 * (1 + i % 5), 2000 + 100 * i) for i in range(23)]]
    for world in (1, 2, 3, 8):
        p = S.plan(costs, world)
        flat = sorted(i for lst in p for i in lst)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in lst) for lst in p]
        assert max(loads) - min(loads) <= max(costs) + 1e-6
        assert p == S.plan(costs, world)     # deterministic on every rank


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, mode, out_dir):
    import datetime
    import torch.distributed as dist
    S = _shots()
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    nshots = 7

    def local(idx):
        if mode == "fail" and rank == 1:
            raise RuntimeError("simulated device error on shot %s" % idx)
        base = float(sum(i + 1 for i in idx))
        return tuple(torch.full((4, 1, 5), base * (k + 1)) for k in range(3))

    try:
        res = S.migrate(local, nshots, costs=[1.0 + (i % 3) for i in range(nshots)])
        torch.save({"pp": res.pp, "ps": res.ps, "mine": res.my_shots}, f"{out_dir}/r{rank}.pt")
    except S.ShotFailure as e:
        torch.save({"failed": e.failed_ranks}, f"{out_dir}/r{rank}.pt")
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("mode", ["ok", "fail"])
def test_two_ranks_over_gloo(tmp_path, mode):
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), mode, str(tmp_path)), nprocs=world, join=True)
    res = [torch.load(f"{tmp_path}/r{r}.pt") for r in range(world)]
    if mode == "fail":
        assert all(r["failed"] == [1] for r in res)
        return
    total = float(sum(i + 1 for i in range(7)))
    for r in res:
        assert torch.allclose(r["pp"], torch.full((4, 1, 5), total))
        assert torch.allclose(r["ps"], torch.full((4, 1, 5), 2 * total))
    assert sorted(res[0]["mine"] + res[1]["mine"]) == list(range(7))
