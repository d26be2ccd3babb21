"""The two 3D step-kernel variants compute the same numbers (GPU).

The default 3D kernels update one cell per thread; the pair kernels two
x-adjacent cells per thread with packed FP32 pairs.  Per cell both evaluate the
stencils with the same operations in the same order; the compiler may fuse the
products of the update formulas differently, so the results agree to float
rounding.  Checked on a full RTM shot (modelling traces, wavefields, excitation
state and images) on grids with partial tiles (odd nx: a thread whose second
cell lies outside the grid), both stencil radii and both boundary kinds.
Tolerances: relative L2 1e-5 on traces and wavefields (the bound both variants
meet against the FP64 oracle; measured 1e-6 to 4e-6 between them after 220
steps), the excitation time equal on at least 99.9 % of the excited cells, the
PP and PS images 1e-5 on those cells, the TP image (r_tp / e_tp, ill-conditioned
where the excitation P stress crosses zero: 9.7e-4 measured over all excited
cells) 1e-4, the image bound of the parity tests, on those whose |e_tp| is above
1e-3 of its 99th percentile.
"""
import numpy as np
import pytest

from _cases import CASES, DT_MS, geometry, model, product_config, rel

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
def test_pair_and_single_cell_kernels_agree(ertm, orc, case):
    assert CASES[case]["shape"][2] % 2 == 1        # odd nx: a half-active pair at the edge
    a = _run(ertm, orc, case, ertm.STEP_PAIRS)
    b = _run(ertm, orc, case, ertm.STEP_SINGLE)
    for q in (0, 1, 2):
        assert rel(a[0][q], b[0][q]) <= 1e-5, ("trace", q, rel(a[0][q], b[0][q]))
    for k in a[1]:
        assert rel(a[1][k], b[1][k]) <= 1e-5, (k, rel(a[1][k], b[1][k]))
    amp = b[3]["amp"].astype(np.float64)
    excited = amp > 1e-2 * np.percentile(amp, 99)
    same = a[3]["time"] == b[3]["time"]
    assert same[excited].mean() > 0.999, same[excited].mean()
    m = excited & same
    etp = np.abs(b[3]["etp"].astype(np.float64))
    tp_ok = m & (etp > 1e-3 * np.percentile(etp[m], 99))
    for q, mask, tol in ((0, m, 1e-5), (1, m, 1e-5), (2, tp_ok, 1e-4)):
        assert rel(a[2][q][mask], b[2][q][mask]) <= tol, ("image", q, rel(a[2][q][mask], b[2][q][mask]))


def test_step_variant_argument_checked(ertm):
    cfg = ertm.Config(nx=40, ny=30, nz=20, dx=5, dy=5, dz=5, dt_ms=0.5, nt=4)
    with ertm.Context(cfg) as ctx:
        with pytest.raises(ertm.ErtmError):
            ctx.set_step_variant(2)
