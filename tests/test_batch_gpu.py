"""Multi-shot RTM with on-device stacking (ertm_rtm_batch) and the shot-parallel
driver on one rank (GPU).  The stack is checked against the sum of single-shot
migrations (ertm_rtm_shot), the call that test_parity_gpu.py pins to the FP64
oracle on the same kind of grid; the batched windows of test_windows_gpu.py are
also checked against the oracle directly."""
import importlib

import numpy as np
import pytest

from _cases import CASES, DT_MS, geometry, model, product_config, rel

pytestmark = pytest.mark.gpu


def test_rtm_batch_equals_sum_of_shots(ertm, orc):
    case = "3d_r4_cpml"
    c = CASES[case]
    vp, vs, rho = model(c["shape"], seed=3)
    nz, ny, nx = c["shape"]
    src, rec = geometry(c["shape"], c["pml"])
    w = orc.ricker(25.0, DT_MS / 1000.0)
    ctx = ertm.Context(product_config(ertm, case, nt=160, src_steps=120))
    ctx.set_model(ertm.TRUE_MODEL, vp, vs, rho)
    ctx.set_model(ertm.MIGRATION_MODEL, vp, vs, rho)
    shots, data = [], []
    for dx in (-6, 0, 5):
        sh = ertm.Shot(src[0] + dx, src[1], src[2], wavelet=w, **rec)
        shots.append(sh)
        data.append(ctx.forward_together_using_real_model(sh))
    per = [ctx.rtm_shot(sh, d) for sh, d in zip(shots, data)]
    stack = ctx.rtm_batch(shots, data)
    for k in range(3):
        ref = np.sum([p[k].astype(np.float64) for p in per], axis=0)
        ok = np.isfinite(ref)
        assert rel(stack[k][ok], ref[ok]) < 1e-6

    shots_mod = importlib.import_module("2d_and_3d_elastic_reverse_time_migration_b200.shots")
    res = shots_mod.migrate(shots_mod.context_local(ctx, shots, data), len(shots))
    for k, t in enumerate((res.pp, res.ps, res.tp)):
        a = t.cpu().numpy()
        ok = np.isfinite(a) & np.isfinite(stack[k])
        assert rel(a[ok], stack[k][ok]) < 1e-6
