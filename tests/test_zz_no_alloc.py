"""The no-allocation modelling entry point against the context entry point (GPU).

The no-allocation variant serves callers that cannot allocate GPU memory when
they call into the library — a plugin host whose execute step forbids it, a
real-time pipeline whose memory is fixed at start-up, a framework whose own
allocator owns the device.  They pass device buffers for every input and the
output, and the library keeps its wavefields in one fixed device array.  This
file runs last (pytest collects it after the others), in a fresh process or
after the rest of the suite, and checks two calls in a row against
ertm_forward_together_using_real_model through the C ABI.
"""
import ctypes as C

import numpy as np
import pytest

from _cases import CASES, DT_MS, FREQ, geometry, model, product_config, rel

pytestmark = pytest.mark.gpu

TOL = 1e-5     # relative L2, the traces tolerance of the parity tests


@pytest.mark.parametrize("case", ["2d_r4_cpml", "3d_r4_cpml", "3d_r6_sponge"])
def test_noalloc_matches_context_path_twice(ertm, orc, case):
    import torch
    nt = 200
    c = CASES[case]
    vp, vs, rho = model(c["shape"], seed=5)
    src, rec = geometry(c["shape"], c["pml"])
    w = orc.ricker(FREQ, DT_MS / 1000.0)
    cfg = product_config(ertm, case, nt)
    with ertm.Context(cfg) as ctx:
        ctx.set_model(ertm.TRUE_MODEL, vp, vs, rho)
        ref = ctx.forward_together_using_real_model(ertm.Shot(*src, wavelet=w, **rec))
    dev = [torch.from_numpy(a).cuda() for a in (vp, vs, rho)]
    shot = ertm.Shot(*src, wavelet=torch.from_numpy(w).cuda(), **rec)
    for call in range(2):
        out = torch.full((3, nt, shot.nrec), float("nan"), device="cuda")
        ertm.forward_together_using_real_model_noalloc(cfg, *dev, shot, out)
        got = out.cpu().numpy()
        for q in range(3):
            assert rel(got[q], ref[q]) <= TOL, (case, call, q, rel(got[q], ref[q]))


def test_noalloc_rejects_oversize_and_host_pointers(ertm):
    import torch
    big = ertm.Config(nx=600, ny=600, nz=400, dx=10, dy=10, dz=10, dt_ms=0.8, nt=10,
                      pml=(20,) * 6)
    n = big.nx * big.ny * big.nz
    t = torch.zeros(1, device="cuda")
    shot = ertm.Shot(300, 300, 30, wavelet=torch.zeros(4, device="cuda"), rx0=0, nrx=4, rz=30)
    buf = C.create_string_buffer(512)
    cs, ss = big.struct(), shot.struct()
    rc = ertm.lib().ertm_forward_together_using_real_model_noalloc(
        C.byref(cs), t.data_ptr(), t.data_ptr(), t.data_ptr(), C.byref(ss), t.data_ptr(), None,
        buf, len(buf))
    assert rc == -1 and b"MiB" in buf.value, buf.value
    small = ertm.Config(nx=40, ny=1, nz=40, dx=5, dy=5, dz=5, dt_ms=0.5, nt=10)
    host = np.ones(40 * 40, np.float32)
    shot2 = ertm.Shot(20, 0, 5, wavelet=np.ones(3, np.float32), rx0=0, nrx=4, rz=5)
    with pytest.raises(ertm.ErtmError) as ei:
        ertm.forward_together_using_real_model_noalloc(small, host, host, host, shot2,
                                                       torch.zeros((3, 10, 4), device="cuda"))
    assert ei.value.code == -1 and "memory of device 0" in str(ei.value)
    # buffers of device 0 handed to a call configured for device 1: refused before any
    # work is queued, whether or not a second GPU exists
    other = ertm.Config(nx=40, ny=1, nz=40, dx=5, dy=5, dz=5, dt_ms=0.5, nt=10, device=1)
    d = torch.ones(40 * 40, device="cuda:0")
    shot3 = ertm.Shot(20, 0, 5, wavelet=torch.ones(3, device="cuda:0"), rx0=0, nrx=4, rz=5)
    with pytest.raises(ertm.ErtmError) as ei:
        ertm.forward_together_using_real_model_noalloc(other, d, d, d, shot3,
                                                       torch.zeros((3, 10, 4), device="cuda:0"))
    assert ei.value.code == -1 and "memory of device 1" in str(ei.value)
    del n
