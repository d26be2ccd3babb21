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


def _cache_worker(rank, world, port, out_dir, phase):
    """phase "crash": shot 4 raises (the run fails, the shots migrated before it stay
    cached); "resume": nothing raises; "skip": shot 4 always raises, skip_failed."""
    import datetime
    import torch.distributed as dist
    S = _shots()
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    nshots = 7

    def one_shot(i):
        with open(f"{out_dir}/calls_{phase}_{rank}.txt", "a") as f:
            f.write(f"{i}\n")
        if i == 4 and phase in ("crash", "skip"):
            raise RuntimeError(f"simulated device error on shot {i}")
        return tuple(torch.full((4, 1, 5), float((i + 1) * (k + 1))) for k in range(3))

    try:
        cache = S.ShotCache(f"{out_dir}/cache") if phase != "skip" else None
        res = S.migrate_shots(one_shot, nshots, (4, 1, 5), costs=[1.0] * nshots, cache=cache,
                              skip_failed=(phase == "skip"), device=torch.device("cpu"))
        torch.save({"pp": res.pp, "tp": res.tp, "failed": res.failed}, f"{out_dir}/{phase}{rank}.pt")
    except S.ShotFailure as e:
        torch.save({"failed_ranks": e.failed_ranks}, f"{out_dir}/{phase}{rank}.pt")
    finally:
        dist.destroy_process_group()


def _calls(out_dir, phase):
    out = []
    for r in range(2):
        p = f"{out_dir}/calls_{phase}_{r}.txt"
        if os.path.exists(p):
            out += [int(x) for x in open(p).read().split()]
    return sorted(out)


def test_shot_cache_resumes_and_failed_shots_are_skipped(tmp_path):
    d = str(tmp_path)
    full = float(sum(range(1, 8)))
    mp.spawn(_cache_worker, args=(2, _free_port(), d, "crash"), nprocs=2, join=True)
    for r in range(2):
        assert torch.load(f"{d}/crash{r}.pt")["failed_ranks"]          # every rank learns of it
    cached = sorted(int(f[4:10]) for f in os.listdir(f"{d}/cache") if f.endswith(".npz"))
    assert 4 not in cached and cached
    mp.spawn(_cache_worker, args=(2, _free_port(), d, "resume"), nprocs=2, join=True)
    # only the shots without a file were migrated again
    assert _calls(d, "resume") == sorted(set(range(7)) - set(cached))
    for r in range(2):
        got = torch.load(f"{d}/resume{r}.pt")
        assert torch.allclose(got["pp"], torch.full((4, 1, 5), full))
        assert torch.allclose(got["tp"], torch.full((4, 1, 5), 3 * full))
        assert got["failed"] == []
    mp.spawn(_cache_worker, args=(2, _free_port(), d, "skip"), nprocs=2, join=True)
    for r in range(2):
        got = torch.load(f"{d}/skip{r}.pt")
        assert torch.allclose(got["pp"], torch.full((4, 1, 5), full - 5.0))
        assert len(got["failed"]) == 1 and got["failed"][0][0] == 4
        assert "simulated device error" in got["failed"][0][1]
