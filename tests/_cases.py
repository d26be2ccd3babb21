"""Shared parity cases: seeded heterogeneous models on small odd-sized grids that
exercise partial tiles, both stencil radii and both boundary kinds."""
from __future__ import annotations

import numpy as np

CPML, SPONGE_COS, SPONGE_CUBIC = 0, 1, 2


def model(shape, seed=7, vmin=2200.0, vmax=3300.0):
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    z = np.arange(nz)[:, None, None]
    layers = vmin + (vmax - vmin) * np.floor(z / max(1, nz // 4)) / 4.0
    vp = layers + 0.04 * vmin * rng.standard_normal(shape)
    vp = np.broadcast_to(vp, shape).astype(np.float32).copy()
    vs = (vp / np.sqrt(3)).astype(np.float32)
    rho = (310.0 * vp.astype(np.float64) ** 0.25).astype(np.float32)
    return vp, vs, rho


CASES = {
    # name: grid (nz, ny, nx), order, boundary, widths, coefficient kind (0 Taylor, 1 reference)
    "3d_r4_cpml": dict(shape=(33, 38, 45), order=8, boundary=CPML, pml=(8, 7, 6, 8, 7, 6), coef=0),
    "3d_r6_sponge": dict(shape=(31, 36, 41), order=12, boundary=SPONGE_COS, pml=(7, 7, 6, 6, 6, 8),
                         coef=1, sponge=180.0),
    "2d_r4_cpml": dict(shape=(83, 1, 97), order=8, boundary=CPML, pml=(12, 10, 0, 0, 11, 12), coef=0),
    "2d_r6_sponge": dict(shape=(79, 1, 91), order=12, boundary=SPONGE_CUBIC, pml=(10, 10, 0, 0, 10, 10),
                         coef=1, sponge=250.0),
}

DX, DT_MS, FREQ = 10.0, 0.8, 15.0


def geometry(shape, pml):
    nz, ny, nx = shape
    src = (nx // 2, ny // 2, pml[4] + 3)
    rec = dict(rx0=pml[0], nrx=nx - pml[0] - pml[1], drx=1,
               ry0=(pml[2] if ny > 1 else 0), nry=(max(1, (ny - pml[2] - pml[3]) // 3) if ny > 1 else 1),
               dry=(3 if ny > 1 else 1), rz=pml[4] + 3)
    return src, rec


def oracle_grid(orc, case, vp):
    c = CASES[case]
    nz, ny, nx = c["shape"]
    coef = orc.coef_reference12() if c["coef"] == 1 else None
    return orc.make_grid(nx, ny, nz, DX, DX, DX, DT_MS, R=c["order"] // 2, coef=coef,
                         boundary=c["boundary"], pml=c["pml"], pml_r=1e-3, pml_f0=10.0,
                         pml_vmax=float(vp.max()), sponge_coef=c.get("sponge", 0.0))


def product_config(ertm, case, nt, src_steps=0):
    c = CASES[case]
    nz, ny, nx = c["shape"]
    return ertm.Config(nx=nx, ny=ny, nz=nz, dx=DX, dy=DX, dz=DX, dt_ms=DT_MS, nt=nt,
                       src_steps=src_steps, order=c["order"], coef_kind=c["coef"],
                       boundary=c["boundary"], pml=c["pml"], pml_r=1e-3, pml_f0=10.0,
                       sponge_coef=c.get("sponge", 0.0))


def rel(a, b):
    """Relative L2 error of a against the reference b."""
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a.astype(np.float64) - b)) / (nb if nb > 0 else 1.0)
