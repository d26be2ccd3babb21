"""What the trained network gains: on a held-out layered-and-faulted model, CG
preconditioned by a U-Net trained (on the library's tensor-core kernels) on
pairs from other models reaches a lower data misfit than plain CG in the same
number of iterations (GPU, reduced scale)."""
import importlib

import pytest

pytestmark = pytest.mark.gpu

PKG = "2d_and_3d_elastic_reverse_time_migration_b200"


def test_learned_preconditioner_beats_plain_cg_on_a_held_out_model():
    import torch
    nn = importlib.import_module(PKG + ".nn")
    L = importlib.import_module(PKG + ".learned")
    dev = torch.device("cuda", 0)
    geo = L.Geometry(nt=400, nshots=4)
    pairs = []
    for k in range(10):
        case = L.make_case(1000 + k, geo)
        pairs.append(L.training_pair(case, cg_iters=10))
        case.ctx.close()
    net = nn.UNet(dev, seed=0)
    log = L.train(net, pairs, steps=400, batch=16, patch=(64, 128), lr=1e-3)
    assert log.loss[-1][1] < 0.5 * log.loss[0][1], log.loss
    case = L.make_case(7777, geo)
    r = L.compare(case, net, niter=6, target=1e-2)
    case.ctx.close()
    # every preconditioned step lowered the misfit, and the curve sits below plain CG
    assert all(b <= a * (1 + 1e-4) for a, b in zip(r["learned_misfit"], r["learned_misfit"][1:]))
    assert r["learned_misfit"][2] < 0.7 * r["plain_misfit"][2], (r["plain_misfit"], r["learned_misfit"])
    assert r["learned_misfit"][-1] < r["plain_misfit"][-1], (r["plain_misfit"], r["learned_misfit"])
