"""Record outputs of the reference's own 2D CUDA kernels as fixtures (needs a GPU).

Loads oracle/_ref/libref2d.so — built here from the reference tree by
oracle/ref_kernels/Makefile (`__graft_entry__.build()` does it when the tree is
present) — runs four reference kernels on seeded inputs and writes
tests/golden/ref_kernels_2d.npz (inputs and outputs in the x-fastest [nz][nx]
layout used by the oracle):
  fwd_txxzzxzpp_viscoelastic_and_memory_3parameterization (elastic: tao=strain=1)
  decom_new, imaging_inner_product_ex_2D, cuda_cal_dem_parameter_viscoelastic_media_new

    python tests/golden/make_golden_kernels.py
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
LIB = os.path.join(REPO, "oracle", "_ref", "libref2d.so")
NX, NZ, RAD = 32, 32, 6                  # interior of the reference kernels; radius halo
DT_MS, DX = 1.0, 10.0
PML = (6, 7, 0, 0, 5, 6)                 # x0, x1, (y), z0, z1 sponge widths
SPONGE = 200.0
COE = np.array([0.0, 1.2213363647, -0.096931457519, 0.017447662353, -0.0029672895159,
                0.00035900539822, -0.00002184781161], np.float32)


def to_ref(a):
    """[nz][nx] -> radius-padded ix-major reference layout"""
    out = np.zeros((NX + 2 * RAD, NZ + 2 * RAD), np.float32)
    out[RAD:RAD + NX, RAD:RAD + NZ] = a.T
    return np.ascontiguousarray(out)


def from_ref(a):
    return np.ascontiguousarray(a.reshape(NX + 2 * RAD, NZ + 2 * RAD)[RAD:RAD + NX, RAD:RAD + NZ].T)


def fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def main():
    import sys
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as orc
    L = C.CDLL(LIB)
    rng = np.random.default_rng(20261203)
    vp = (2000 + 1000 * rng.random((NZ, NX))).astype(np.float32)
    vs = (vp / np.sqrt(3) * (1 + 0.05 * rng.standard_normal((NZ, NX)))).astype(np.float32)
    rho = (310 * vp.astype(np.float64) ** 0.25).astype(np.float32)
    # the reference sponge: per-cell damping = z profile + x profile
    px = orc.sponge_profile(orc.SPONGE_CUBIC, NX, PML[0], PML[1], SPONGE).astype(np.float32)
    pz = orc.sponge_profile(orc.SPONGE_CUBIC, NZ, PML[4], PML[5], SPONGE).astype(np.float32)
    att = (pz[:, None] + px[None, :]).astype(np.float32)
    f = {k: rng.standard_normal((NZ, NX)).astype(np.float32) for k in ("vx", "vz", "txx", "tzz", "txz")}
    out = {"vp": vp, "vs": vs, "rho": rho, "att": att, **{"in_" + k: v for k, v in f.items()}}
    n = (NX + 2 * RAD) * (NZ + 2 * RAD)
    o = [np.zeros(n, np.float32) for _ in range(3)]
    rc = L.ref_stress_step(NX, NZ, C.c_float(DT_MS), C.c_float(DX), C.c_float(DX), fp(COE),
                           fp(to_ref(vp)), fp(to_ref(vs)), fp(to_ref(rho)), fp(to_ref(att)),
                           *[fp(to_ref(f[k])) for k in ("vx", "vz", "txx", "tzz", "txz")],
                           *[fp(x) for x in o])
    assert rc == 0, rc
    out.update(stress_txx=from_ref(o[0]), stress_tzz=from_ref(o[1]), stress_txz=from_ref(o[2]))

    p, s = np.zeros(n, np.float32), np.zeros(n, np.float32)
    rc = L.ref_decom_new(NX, NZ, C.c_float(DX), C.c_float(DX), fp(COE), fp(to_ref(f["vx"])),
                         fp(to_ref(f["vz"])), fp(to_ref(vp)), fp(to_ref(vs)), fp(p), fp(s))
    assert rc == 0, rc
    out.update(decom_p=from_ref(p), decom_s=from_ref(s))

    e = [rng.standard_normal((NZ, NX)).astype(np.float32) for _ in range(4)]
    e[0][0, :3] = 0.0
    e[1][0, :3] = 0.0        # three cells with a zero excitation vector
    img = np.zeros(NX * NZ, np.float32)
    ix = [np.ascontiguousarray(a.T) for a in e]           # ix-major, no padding
    rc = L.ref_imaging(NX, NZ, *[fp(a) for a in ix], fp(img))
    assert rc == 0, rc
    out.update(img_ex=e[0], img_ez=e[1], img_rx=e[2], img_rz=e[3],
               img_pp=np.ascontiguousarray(img.reshape(NX, NZ).T))

    g = {k: (rng.standard_normal((NZ, NX)) * (0.05 if k.startswith("r") else 1.0)).astype(np.float32)
         for k in ("rvp", "rvs", "rrho", "vx_x", "vx_z", "vz_x", "vz_z", "vx_t", "vz_t")}
    dem = np.zeros(5 * n, np.float32)
    rc = L.ref_dem_sources(NX, NZ, C.c_float(DT_MS), fp(to_ref(vp)), fp(to_ref(vs)), fp(to_ref(rho)),
                           *[fp(to_ref(g[k])) for k in ("rvp", "rvs", "rrho", "vx_x", "vx_z", "vz_x",
                                                        "vz_z", "vx_t", "vz_t")], fp(dem))
    assert rc == 0, rc
    out.update({"dem_" + k: v for k, v in g.items()})
    for q, name in enumerate(("dem_p1", "dem_p2", "dem_sxx", "dem_szz", "dem_sxz")):
        out[name] = from_ref(dem[q * n:(q + 1) * n])
    np.savez_compressed(os.path.join(HERE, "ref_kernels_2d.npz"),
                        meta=np.array([NX, NZ, RAD, DT_MS, DX, SPONGE] + list(PML), np.float64), **out)
    print("wrote ref_kernels_2d.npz")


if __name__ == "__main__":
    main()
