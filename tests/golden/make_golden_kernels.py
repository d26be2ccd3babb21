"""Record outputs of the reference's own 2D CUDA kernels as fixtures (needs a GPU).

Loads oracle/_ref/libref2d.so — built here from the reference tree by
oracle/ref_kernels/Makefile (`__graft_entry__.build()` does it when the tree is
present) — runs reference kernels on seeded inputs and writes, with inputs and
outputs in the x-fastest [nz][nx] layout used by the oracle:
  tests/golden/ref_kernels_2d.npz:
    fwd_txxzzxzpp_viscoelastic_and_memory_3parameterization (elastic: tao=strain=1)
    decom_new, imaging_inner_product_ex_2D, cuda_cal_dem_parameter_viscoelastic_media_new
  tests/golden/ref_kernels_2d_post.npz (the post-imaging products):
    sum_poynting + caculate_ex_angle_pp_only_RTM / caculate_ex_angle_rp_only_RTM,
    imaging_pp/ps_compensate_dependent_angle_2D and their _new (sign) variants,
    cuda_bell_smoothz_new / cuda_bell_smoothx_new / cuda_bell_smooth_2d,
    cuda_attenuation_truncation, cauda_zero_and_attenuation_truncation

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


def ix_major(a):
    """[nz][nx] -> the reference's plain ix-major layout"""
    return np.ascontiguousarray(a.T)


def from_ix(a, nx, nz):
    return np.ascontiguousarray(a.reshape(nx, nz).T)


def main_post():
    L = C.CDLL(LIB)
    rng = np.random.default_rng(20261204)
    out = {}
    # propagation angles: P stress and P velocity fields, excitation step 0..3 per cell
    nx, nz, it = 32, 32, 1
    tp = rng.standard_normal((nz, nx)).astype(np.float32)
    vxp = rng.standard_normal((nz, nx)).astype(np.float32)
    vzp = rng.standard_normal((nz, nx)).astype(np.float32)
    tp[:12, :12] = 0.0                   # windows with no P energy keep their input value
    et = rng.integers(0, 4, (nz, nx)).astype(np.int32)
    out.update(ang_tp=tp, ang_vxp=vxp, ang_vzp=vzp, ang_time=et,
               ang_meta=np.array([nx, nz, it], np.int64))
    for mode, name in ((0, "ang_pp"), (1, "ang_rp")):
        a = np.full(((nx + 2 * RAD) * (nz + 2 * RAD)), -999.0, np.float32)
        rc = L.ref_angle(nx, nz, mode, it, fp(to_ref(tp)), fp(to_ref(vxp)), fp(to_ref(vzp)),
                         fp(to_ref(et.astype(np.float32))), fp(a))
        assert rc == 0, rc
        out[name] = from_ref(a)
    # angle-dependent compensation, the four variants
    nx, nz = 40, 30
    img = rng.standard_normal((nz, nx)).astype(np.float32)
    src = rng.uniform(-80, 80, (nz, nx)).astype(np.float32)
    rcv = rng.uniform(-80, 80, (nz, nx)).astype(np.float32)
    src[0, :10], rcv[0, :10] = 90.0, 0.0           # the clamped band near 90 degrees
    src[1, :10], rcv[1, :10] = 1.0, 0.0            # small open angles (PS clamp)
    src[2, :10], rcv[2, :10] = 30.0, 120.0         # cos < 0 (the sign variant)
    out.update(comp_img=img, comp_src=src, comp_rcv=rcv)
    for kind in range(4):
        o = np.zeros(nx * nz, np.float32)
        r2 = np.zeros(nx * nz, np.float32)
        rc = L.ref_compensate(nx, nz, kind, fp(ix_major(src)), fp(ix_major(rcv)), fp(ix_major(img)),
                              fp(o), fp(r2))
        assert rc == 0, rc
        out[f"comp_out{kind}"] = from_ix(o, nx, nz)
        if kind < 2:
            out[f"comp_open{kind}"] = from_ix(r2, nx, nz)
    # truncated Gaussian smoothing
    nx, nz = 48, 40
    g = rng.standard_normal((nz, nx)).astype(np.float32)
    out["bell_in"] = g
    for mode, rb, name in ((0, 5, "bell_z5"), (1, 5, "bell_x5"), (2, 3, "bell_2d3")):
        o = np.zeros(nx * nz, np.float32)
        rc = L.ref_bell(nx, nz, rb, mode, fp(ix_major(g)), fp(o))
        assert rc == 0, rc
        out[name] = from_ix(o, nx, nz)
    # edge tapers and aperture mutes of a gradient
    nx, nz = 96, 20
    g = rng.standard_normal((nz, nx)).astype(np.float32)
    out["trunc_in"] = g
    cases = {"trunc_a": (0, 30, 24, 10, 0), "trunc_b": (1, 40, 50, 20, 4), "trunc_c": (1, 30, 5, 8, 4)}
    for name, (zm, ol, orr, ro, oa) in cases.items():
        a = ix_major(g).copy()
        rc = L.ref_truncation(nx, nz, zm, ol, orr, ro, oa, fp(a))
        assert rc == 0, rc
        out[name] = from_ix(a, nx, nz)
        out[name + "_args"] = np.array([zm, ol, orr, ro, oa], np.int64)
    np.savez_compressed(os.path.join(HERE, "ref_kernels_2d_post.npz"), **out)
    print("wrote ref_kernels_2d_post.npz")


if __name__ == "__main__":
    import sys as _sys
    if "--post" not in _sys.argv:
        main()
    main_post()
