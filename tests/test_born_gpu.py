"""CUDA Born operators (elastic and GSLS-3 viscoelastic) against the oracle, adjointness
in FP32, checkpoint independence."""
import numpy as np
import pytest

from _born_case import VISCO, born_case, oracle_shot, visco_case
from _cases import rel

pytestmark = pytest.mark.gpu


def _ctx(ertm, c, K=0, visco=False):
    nz, _, nx = c["shape"]
    v = dict(zip(("visco_nmech", "visco_qp", "visco_qs", "visco_f0"), VISCO)) if visco else {}
    cfg = ertm.Config(nx=nx, ny=1, nz=nz, dx=10, dy=10, dz=10, dt_ms=1.0, nt=c["nt"],
                      order=2 * c["R"], boundary=ertm.BOUNDARY_SPONGE_CUBIC, pml=c["pml"],
                      sponge_coef=150.0, checkpoint_every=K, **v)
    ctx = ertm.Context(cfg)
    ctx.set_model(ertm.MIGRATION_MODEL, c["vp"], c["vs"], c["rho"])
    shot = ertm.Shot(*c["geo"]["src"], wavelet=c["w"], **c["geo"]["rec"])
    return ctx, shot


@pytest.mark.parametrize("R,visco", [(4, False), (6, False), (4, True)])
def test_born_forward_and_adjoint_match_oracle(ertm, orc, R, visco):
    c = (visco_case if visco else born_case)(orc, R=R)
    s = oracle_shot(orc, c)
    rng = c["rng"]
    m = [(0.05 * rng.standard_normal(c["shape"])).astype(np.float32) for _ in range(3)]
    ref = orc.born_forward(c["g"], c["vp"], c["vs"], c["rho"], s, c["nt"], *m)
    r32 = orc.born_forward(c["g"], c["vp"], c["vs"], c["rho"], s, c["nt"], *m, bits=32)
    ctx, shot = _ctx(ertm, c, K=40, visco=visco)
    gpu = ctx.born_forward(shot, *m)
    for q in (0, 2):
        assert rel(gpu[q], ref[q]) <= max(1e-5, 3 * rel(r32[q], ref[q])), q
    dh = rng.standard_normal(ref.shape).astype(np.float32)
    dh[1] = 0
    gref = orc.born_adjoint(c["g"], c["vp"], c["vs"], c["rho"], s, c["nt"], dh)
    g32 = orc.born_adjoint(c["g"], c["vp"], c["vs"], c["rho"], s, c["nt"], dh, bits=32)
    ggpu = ctx.born_adjoint(shot, dh)
    for a, b, f in zip(ggpu, gref, g32):
        assert rel(a, b) <= max(1e-5, 3 * rel(f, b))


@pytest.mark.parametrize("visco", [False, True])
def test_gpu_dot_product_and_checkpoint_independence(ertm, orc, visco):
    c = born_case(orc, nz=64, nx=80, nt=400)
    rng = c["rng"]
    m = [(0.05 * rng.standard_normal(c["shape"])).astype(np.float32) for _ in range(3)]
    ctx, shot = _ctx(ertm, c, K=0, visco=visco)
    d = ctx.born_forward(shot, *m)
    dh = rng.standard_normal(d.shape).astype(np.float32)
    dh[1] = 0
    g_default = ctx.born_adjoint(shot, dh)
    lhs = float(np.sum(d.astype(np.float64) * dh))
    rhs = sum(float(np.sum(a.astype(np.float64) * b)) for a, b in zip(m, g_default))
    assert abs(lhs - rhs) <= 1e-4 * abs(lhs), (lhs, rhs)
    ctx7, shot7 = _ctx(ertm, c, K=7, visco=visco)
    g7 = ctx7.born_adjoint(shot7, dh)
    for a, b in zip(g7, g_default):
        assert np.array_equal(a, b)       # the rebuilt background is bit-identical


def test_born_rejects_cpml_and_3d(ertm):
    cfg = ertm.Config(nx=40, ny=1, nz=40, dx=5, dy=5, dz=5, dt_ms=0.5, nt=10, pml=(8, 8, 0, 0, 8, 8))
    ctx = ertm.Context(cfg)
    z = np.zeros((40, 1, 40), np.float32) + 2000
    ctx.set_model(ertm.MIGRATION_MODEL, z, z / 2, z / 2)
    shot = ertm.Shot(20, 0, 10, wavelet=np.ones(3, np.float32), rx0=0, nrx=4, rz=10)
    with pytest.raises(ertm.ErtmError) as ei:
        ctx.born_forward(shot, z * 0, z * 0, z * 0)
    assert ei.value.code == -5


@pytest.mark.parametrize("visco", [False, True])
def test_shot_batch_matches_single_shots(ertm, orc, visco):
    """Several shots in one launch per step (ertm_born_*_shots) against one call per
    shot: the traces are bit-identical (the per-shot arithmetic is the same), the
    summed gradient agrees to float rounding (the batch sums the accumulators before
    scaling), and the batched pair passes the dot test."""
    c = born_case(orc, nz=48, nx=72, nt=300)
    rng = c["rng"]
    m = [(0.05 * rng.standard_normal(c["shape"])).astype(np.float32) for _ in range(3)]
    ctx, _ = _ctx(ertm, c, K=60, visco=visco)
    nx = c["shape"][2]
    rec = c["geo"]["rec"]
    shots = [ertm.Shot(int(x), 0, 12, wavelet=c["w"] * (1.0 + 0.1 * k), **rec)
             for k, x in enumerate((15, 30, 41, nx - 16))]
    single = np.stack([ctx.born_forward(s, *m) for s in shots])
    batch = ctx.born_forward_shots(shots, *m)
    assert np.array_equal(batch, single)
    dh = rng.standard_normal(batch.shape).astype(np.float32)
    dh[:, 1] = 0
    g_single = [ctx.born_adjoint(s, d) for s, d in zip(shots, dh)]
    g_sum = [sum(g[q].astype(np.float64) for g in g_single) for q in range(3)]
    g_batch = ctx.born_adjoint_shots(shots, dh)
    for a, b in zip(g_batch, g_sum):
        assert rel(a, b) <= 1e-6
    lhs = float(np.sum(batch.astype(np.float64) * dh))
    rhs = sum(float(np.sum(a.astype(np.float64) * b)) for a, b in zip(m, g_batch))
    assert abs(lhs - rhs) <= 1e-4 * abs(lhs), (lhs, rhs)


def test_shot_batch_device_arrays(ertm, orc):
    import torch
    c = born_case(orc, nz=40, nx=64, nt=200)
    rng = c["rng"]
    m = [(0.05 * rng.standard_normal(c["shape"])).astype(np.float32) for _ in range(3)]
    ctx, _ = _ctx(ertm, c, K=50)
    shots = [ertm.Shot(int(x), 0, 12, wavelet=c["w"], **c["geo"]["rec"]) for x in (20, 44)]
    host = ctx.born_forward_shots(shots, *m)
    dev = torch.zeros(host.shape, device="cuda")
    ctx.born_forward_shots(shots, *[torch.from_numpy(a).cuda() for a in m], out=dev)
    assert np.array_equal(dev.cpu().numpy(), host)
    gh = ctx.born_adjoint_shots(shots, host)
    gd = [torch.zeros(c["shape"], device="cuda") for _ in range(3)]
    ctx.born_adjoint_shots(shots, dev, *gd)
    for a, b in zip(gd, gh):
        assert np.array_equal(a.cpu().numpy(), b)


def test_chunk_length_does_not_change_the_results(ertm, orc):
    """The step kernels march each warp down a chunk of rows whose length follows the
    size of the launch (32, 16 or 8 rows, the longest that still gives about two
    waves of blocks): 8 shots on a 1000 x 1100 grid run in 32-row chunks, one shot
    in 8-row chunks.  The traces are bit-identical (the per-cell arithmetic does not
    depend on the chunk), the batched gradient equals the sum of the single-shot
    ones to float rounding."""
    c = born_case(orc, nz=1100, nx=1000, nt=100)
    rng = c["rng"]
    m = [(0.05 * rng.standard_normal(c["shape"])).astype(np.float32) for _ in range(3)]
    ctx, _ = _ctx(ertm, c, K=20)
    rec = c["geo"]["rec"]
    shots = [ertm.Shot(int(x), 0, 12, wavelet=c["w"], **rec) for x in np.linspace(20, 979, 8).astype(int)]
    batch = ctx.born_forward_shots(shots, *m)
    for k in (0, 5):
        assert np.array_equal(batch[k], ctx.born_forward(shots[k], *m)), k
    dh = rng.standard_normal(batch.shape).astype(np.float32)
    dh[:, 1] = 0
    g_batch = ctx.born_adjoint_shots(shots, dh)
    g_single = [ctx.born_adjoint(s, d) for s, d in zip(shots, dh)]
    for q in range(3):
        assert rel(g_batch[q], sum(g[q].astype(np.float64) for g in g_single)) <= 1e-6, q
