"""Shared 2D Born case: heterogeneous model, reference cubic sponge, one shot."""
import numpy as np

SPONGE_CUBIC = 2


def born_case(orc, nz=50, nx=60, nt=250, R=4, seed=0):
    rng = np.random.default_rng(seed)
    vp = (2500 + 300 * rng.random((nz, 1, nx))).astype(np.float32)
    vs = (vp / 1.8).astype(np.float32)
    rho = (310 * vp.astype(np.float64) ** 0.25).astype(np.float32)
    pml = (10, 10, 0, 0, 10, 10)
    g = orc.make_grid(nx, 1, nz, 10.0, 10.0, 10.0, 1.0, R=R, boundary=SPONGE_CUBIC, pml=pml,
                      sponge_coef=150.0)
    w = orc.ricker(20.0, 1e-3)
    geo = dict(src=(nx // 2, 0, 12), rec=dict(rx0=10, nrx=nx - 20, drx=1, rz=12))
    return dict(g=g, vp=vp, vs=vs, rho=rho, w=w, nt=nt, pml=pml, shape=(nz, 1, nx), R=R, geo=geo,
                rng=rng)


def oracle_shot(orc, c):
    return orc.make_shot(*c["geo"]["src"], c["w"], **c["geo"]["rec"])


VISCO = (3, 100.0, 50.0, 15.0)   # GSLS-3, Qp 100, Qs 50, reference 15 Hz


def visco_case(orc, **kw):
    """The Born case with GSLS-3 attenuation (Qp 100, Qs 50 around 15 Hz)."""
    c = born_case(orc, **kw)
    c["g"].visco_nmech, c["g"].visco_qp, c["g"].visco_qs, c["g"].visco_f0 = VISCO
    return c
