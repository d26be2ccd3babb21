"""The two 3D step-kernel variants compute the same numbers (GPU).

The default 3D kernels update two x-adjacent cells per thread with packed FP32
pairs; the single-cell kernels one cell per thread.  Per cell both evaluate the
same operations in the same order (a difference as one rounding, each stencil tap
as one fused multiply-add), so modelling traces, wavefields, excitation state and
images of a full RTM shot must agree to the last bit, on grids with partial tiles
(odd nx: a thread whose second cell lies outside the grid) in both stencil radii
and boundary kinds.
"""
import numpy as np
import pytest

from _cases import CASES, DT_MS, geometry, model, product_config

pytestmark = pytest.mark.gpu


def _run(ertm, orc, case, variant):
    c = CASES[case]
    nt, nsrc = 220, 160
    vp, vs, rho = model(c["shape"], seed=3)
    src, rec = geometry(c["shape"], c["pml"])
    w = orc.ricker(25.0, DT_MS / 1000.0)
    with ertm.Context(product_config(ertm, case, nt, nsrc)) as ctx:
        ctx.set_step_variant(variant)
        ctx.set_model(ertm.TRUE_MODEL, vp, vs, rho)
        ctx.set_model(ertm.MIGRATION_MODEL, vp, vs, rho)
        shot = ertm.Shot(*src, wavelet=w, **rec)
        data = ctx.forward_together_using_real_model(shot)
        fields = {n: ctx.get_wavefield(n) for n in ("vx", "vy", "vz", "txx", "tyz")}
        imgs = ctx.rtm_shot(shot, data)
        ex = ctx.get_excitation()
    return data, fields, imgs, ex


@pytest.mark.parametrize("case", ["3d_r4_cpml", "3d_r6_sponge"])
def test_pair_and_single_cell_kernels_agree_bitwise(ertm, orc, case):
    assert CASES[case]["shape"][2] % 2 == 1        # odd nx: a half-active pair at the edge
    a = _run(ertm, orc, case, ertm.STEP_PAIRS)
    b = _run(ertm, orc, case, ertm.STEP_SINGLE)
    assert np.array_equal(a[0], b[0]), "traces"
    for k in a[1]:
        assert np.array_equal(a[1][k], b[1][k]), k
    for q in range(3):
        assert np.array_equal(a[2][q], b[2][q], equal_nan=True), f"image {q}"
    for k in ("time", "amp", "evx", "evy", "evz", "etp"):
        assert np.array_equal(a[3][k], b[3][k]), k


def test_step_variant_argument_checked(ertm):
    cfg = ertm.Config(nx=40, ny=30, nz=20, dx=5, dy=5, dz=5, dt_ms=0.5, nt=4)
    with ertm.Context(cfg) as ctx:
        with pytest.raises(ertm.ErtmError):
            ctx.set_step_variant(2)
