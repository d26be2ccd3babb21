"""Least-squares RTM by CGLS on the CUDA Born operators (GPU)."""
import importlib

import numpy as np
import pytest

from _born_case import VISCO, born_case
from _cases import rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("visco", [False, True])
def test_cgls_lowers_the_misfit_monotonically(ertm, orc, visco):
    lsrtm = importlib.import_module("2d_and_3d_elastic_reverse_time_migration_b200.lsrtm")
    c = born_case(orc, nz=60, nx=90, nt=350)
    nz, _, nx = c["shape"]
    v = dict(zip(("visco_nmech", "visco_qp", "visco_qs", "visco_f0"), VISCO)) if visco else {}
    cfg = ertm.Config(nx=nx, ny=1, nz=nz, dx=10, dy=10, dz=10, dt_ms=1.0, nt=c["nt"],
                      order=8, boundary=ertm.BOUNDARY_SPONGE_CUBIC, pml=c["pml"],
                      sponge_coef=150.0, checkpoint_every=50, **v)
    ctx = ertm.Context(cfg)
    ctx.set_model(ertm.MIGRATION_MODEL, c["vp"], c["vs"], c["rho"])
    shots = [ertm.Shot(sx, 0, 12, wavelet=c["w"], rx0=10, nrx=nx - 20, rz=12)
             for sx in (20, 45, 70)]
    # a reflector: relative perturbations on two interfaces
    true = [np.zeros(c["shape"], np.float32) for _ in range(3)]
    true[0][35:38] = 0.08
    true[1][35:38] = -0.05
    true[2][45:47] = 0.04
    data = [ctx.born_forward(s, *true) for s in shots]
    res = lsrtm.cgls(ctx, shots, data, niter=8)
    mis = res.misfit
    assert all(b <= a * (1 + 1e-4) for a, b in zip(mis, mis[1:])), mis
    assert mis[-1] < 0.3, mis
    # the inverted r_vp correlates with the true one
    corr = np.corrcoef(res.m[0].ravel(), true[0].ravel())[0, 1]
    assert corr > 0.3, corr


def test_cgls_with_device_vectors_matches_host_vectors(ertm, orc):
    """CUDA tensors in: every CG vector stays on the device (batched operators, no
    host copies); the misfit history equals the host-vector run to float rounding."""
    import torch
    lsrtm = importlib.import_module("2d_and_3d_elastic_reverse_time_migration_b200.lsrtm")
    c = born_case(orc, nz=50, nx=80, nt=300)
    nz, _, nx = c["shape"]
    cfg = ertm.Config(nx=nx, ny=1, nz=nz, dx=10, dy=10, dz=10, dt_ms=1.0, nt=c["nt"],
                      order=8, boundary=ertm.BOUNDARY_SPONGE_CUBIC, pml=c["pml"],
                      sponge_coef=150.0, checkpoint_every=60)
    ctx = ertm.Context(cfg)
    ctx.set_model(ertm.MIGRATION_MODEL, c["vp"], c["vs"], c["rho"])
    shots = [ertm.Shot(sx, 0, 12, wavelet=c["w"], rx0=10, nrx=nx - 20, rz=12) for sx in (20, 40, 60)]
    true = [np.zeros(c["shape"], np.float32) for _ in range(3)]
    true[0][30:33] = 0.08
    true[2][40:42] = 0.04
    data = list(ctx.born_forward_shots(shots, *true))
    host = lsrtm.cgls(ctx, shots, data, niter=5)
    dev = lsrtm.cgls(ctx, shots, [torch.from_numpy(d).cuda() for d in data], niter=5)
    assert all(torch.is_tensor(x) and x.is_cuda for x in dev.m)
    np.testing.assert_allclose(dev.misfit, host.misfit, rtol=1e-4)
    for a, b in zip(dev.m, host.m):
        assert rel(a.cpu().numpy(), b) < 1e-4
