"""The device-error path of the step kernels (GPU): a staged copy that never lands.

Every wait of the step kernels on a shared-memory stage is bounded.  The test
hook `Context.set_wait_fault(plane, polls)` makes the first CTA of every
step-kernel launch skip the staged copy of one z plane, so its consumers' wait
runs out after `polls` polls; the kernel stops writing, its producer waits for
the copies it did issue, and the pass reports ERTM_EDEVICE.  Nothing faults or
hangs: the wait that runs out is on a copy that was never issued.  The next
pass on the same context, with the hook off, must give exactly the result of a
context that never saw the error (the reference simply aborts on a CUDA error,
3D_elastic_RTM/3D_forward_or_back_together.cu:34).
"""
import numpy as np
import pytest

from _cases import CASES, DT_MS, FREQ, geometry, model, product_config

pytestmark = pytest.mark.gpu

EDEVICE = -6


@pytest.mark.parametrize("case", ["3d_r4_cpml", "2d_r6_sponge"])
def test_wait_runs_out_then_context_recovers(ertm, orc, case):
    nt = 12
    c = CASES[case]
    vp, vs, rho = model(c["shape"], seed=11)
    src, rec = geometry(c["shape"], c["pml"])
    w = orc.ricker(FREQ, DT_MS / 1000.0)
    cfg = product_config(ertm, case, nt)
    shot = ertm.Shot(*src, wavelet=w, **rec)
    with ertm.Context(cfg) as fresh:
        fresh.set_model(ertm.TRUE_MODEL, vp, vs, rho)
        want = fresh.forward_together_using_real_model(shot)
    with ertm.Context(cfg) as ctx:
        ctx.set_model(ertm.TRUE_MODEL, vp, vs, rho)
        ctx.set_wait_fault(plane=1, polls=2000)
        with pytest.raises(ertm.ErtmError) as ei:
            ctx.forward_together_using_real_model(shot)
        assert ei.value.code == EDEVICE, str(ei.value)
        assert "bounded wait" in str(ei.value)
        ctx.set_wait_fault(-1)
        got = ctx.forward_together_using_real_model(shot)
        assert np.array_equal(got, want)
        # and once more, to show that no error word was left behind
        again = ctx.forward_together_using_real_model(shot)
        assert np.array_equal(again, want)


def test_wait_fault_argument_checked(ertm):
    cfg = ertm.Config(nx=40, ny=1, nz=40, dx=5, dy=5, dz=5, dt_ms=0.5, nt=4)
    with ertm.Context(cfg) as ctx:
        with pytest.raises(ertm.ErtmError) as ei:
            ctx.set_wait_fault(plane=-2)
        assert ei.value.code == -1
