"""ctypes front end of the CPU oracle — TEST INFRASTRUCTURE ONLY.

Loaded only by tests/, the smoke check and bench.py's CPU-baseline leg, as
the checker.  The product library never imports this module.

`Grid` and `Shot` mirror ``orc_grid`` / ``orc_shot`` in ertm_oracle.h.  All
arrays are float32 numpy arrays in x-fastest order, shape (nz, ny, nx).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "build")

MODEL, SOURCE, RECEIVER = 0, 1, 2
CPML, SPONGE_COS, SPONGE_CUBIC = 0, 1, 2
FIELD_NAMES = ("vx", "vy", "vz", "txx", "tyy", "tzz", "txy", "txz", "tyz",
               "tp", "vxp", "vyp", "vzp")


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("dt_ms", C.c_double), ("R", C.c_int), ("coef", C.c_double * 8),
                ("boundary", C.c_int), ("pml", C.c_int * 6), ("pml_r", C.c_double),
                ("pml_f0", C.c_double), ("pml_vmax", C.c_double),
                ("sponge_coef", C.c_double), ("visco_nmech", C.c_int), ("visco_qp", C.c_double),
                ("visco_qs", C.c_double), ("visco_f0", C.c_double)]


class Shot(C.Structure):
    _fields_ = [("sx", C.c_int), ("sy", C.c_int), ("sz", C.c_int), ("nw", C.c_int),
                ("wavelet", C.POINTER(C.c_float)),
                ("rx0", C.c_int), ("nrx", C.c_int), ("drx", C.c_int),
                ("ry0", C.c_int), ("nry", C.c_int), ("dry", C.c_int),
                ("rz", C.c_int), ("inject_mode", C.c_int)]


class Excitation(C.Structure):
    _fields_ = [("amp2", C.POINTER(C.c_float)), ("second2", C.POINTER(C.c_float)),
                ("time", C.POINTER(C.c_int)), ("evx", C.POINTER(C.c_float)),
                ("evy", C.POINTER(C.c_float)), ("evz", C.POINTER(C.c_float)),
                ("etp", C.POINTER(C.c_float)), ("src_angle", C.POINTER(C.c_float)),
                ("rcv_angle", C.POINTER(C.c_float)), ("src_energy", C.POINTER(C.c_float)),
                ("rcv_energy", C.POINTER(C.c_float))]


_libs: dict[int, C.CDLL] = {}


def build() -> None:
    """Compile both oracle builds with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib(bits: int = 64) -> C.CDLL:
    if bits not in _libs:
        path = os.path.join(_BUILD, f"liboracle{bits}.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        P = C.POINTER
        f = P(C.c_float)
        L.orc_ricker.argtypes = [C.c_double, C.c_double, f, C.c_int]
        L.orc_ricker.restype = C.c_int
        L.orc_coef_taylor.argtypes = [C.c_int, P(C.c_double)]
        L.orc_coef_reference12.argtypes = [P(C.c_double)]
        L.orc_sponge_profile.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                         P(C.c_double)]
        L.orc_cpml_profile.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                       C.c_double, C.c_double, C.c_double, C.c_int,
                                       P(C.c_double), P(C.c_double)]
        L.orc_run_pass.argtypes = [P(Grid), f, f, f, P(Shot), C.c_int, C.c_int, f,
                                   P(Excitation), f, f, f, f]
        L.orc_run_pass.restype = C.c_int
        L.orc_divcurl.argtypes = [P(Grid), f, f, f, f, f, f, f, f, f]
        L.orc_divcurl.restype = C.c_int
        L.orc_state_create.argtypes = [P(Grid), f, f, f]
        L.orc_state_create.restype = C.c_void_p
        L.orc_state_step.argtypes = [C.c_void_p, P(Shot), C.c_int, C.c_int, C.c_int, f,
                                     P(Excitation), f, f, f]
        L.orc_state_destroy.argtypes = [C.c_void_p]
        L.orc_state_fields.argtypes = [C.c_void_p, f]
        L.orc_born_forward.argtypes = [P(Grid), f, f, f, P(Shot), C.c_int, f, f, f, f]
        L.orc_born_forward.restype = C.c_int
        L.orc_born_adjoint.argtypes = [P(Grid), f, f, f, P(Shot), C.c_int, f, f, f, f]
        L.orc_born_adjoint.restype = C.c_int
        L.orc_stress_step_given.argtypes = [P(Grid)] + [f] * 11
        L.orc_stress_step_given.restype = C.c_int
        L.orc_born_sources_given.argtypes = [C.c_long, C.c_double] + [f] * 16
        L.orc_born_sources_given.restype = C.c_int
        L.orc_image_given.argtypes = [C.c_long] + [f] * 8
        L.orc_image_given.restype = C.c_int
        L.orc_visco_model.argtypes = [P(Grid), f, f, f, P(Shot), C.c_int, f]
        L.orc_visco_model.restype = C.c_int
        L.orc_visco_fit.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, P(C.c_double),
                                    P(C.c_double), P(C.c_double)]
        L.orc_angle_given.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, f, f, f, P(C.c_int), f]
        L.orc_angle_given.restype = C.c_int
        L.orc_threads.restype = C.c_int
        L.orc_real_size.restype = C.c_int
        _libs[bits] = L
    return _libs[bits]


def _fp(a):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_float))


def ricker(freq_hz: float, dt_s: float, bits: int = 64) -> np.ndarray:
    L = lib(bits)
    n = L.orc_ricker(freq_hz, dt_s, None, 0)
    out = np.zeros(n, np.float32)
    L.orc_ricker(freq_hz, dt_s, _fp(out), n)
    return out


def coef_taylor(R: int) -> np.ndarray:
    c = (C.c_double * 8)()
    lib().orc_coef_taylor(R, c)
    return np.array(c[:R + 1])


def coef_reference12() -> np.ndarray:
    c = (C.c_double * 8)()
    lib().orc_coef_reference12(c)
    return np.array(c[:7])


def sponge_profile(kind: int, n: int, w0: int, w1: int, coe: float) -> np.ndarray:
    out = (C.c_double * n)()
    lib().orc_sponge_profile(kind, n, w0, w1, coe, out)
    return np.array(out[:])


def cpml_profile(n, w0, w1, h, dt_s, vmax, rc, f0, stagger):
    a = (C.c_double * n)()
    b = (C.c_double * n)()
    lib().orc_cpml_profile(n, w0, w1, h, dt_s, vmax, rc, f0, stagger, a, b)
    return np.array(a[:]), np.array(b[:])


def make_grid(nx, ny, nz, dx, dy, dz, dt_ms, R=4, coef=None, boundary=CPML, pml=(0,) * 6,
              pml_r=1e-3, pml_f0=10.0, pml_vmax=4000.0, sponge_coef=0.0, visco=None) -> Grid:
    """visco: None (elastic) or (nmech, qp, qs, f0) for the Born operators."""
    g = Grid()
    g.nx, g.ny, g.nz = nx, ny, nz
    g.dx, g.dy, g.dz = dx, dy, dz
    g.dt_ms = dt_ms
    g.R = R
    c = coef_taylor(R) if coef is None else np.asarray(coef, np.float64)
    for i in range(8):
        g.coef[i] = float(c[i]) if i < len(c) else 0.0
    g.boundary = boundary
    for i in range(6):
        g.pml[i] = int(pml[i])
    g.pml_r, g.pml_f0, g.pml_vmax, g.sponge_coef = pml_r, pml_f0, pml_vmax, sponge_coef
    if visco:
        g.visco_nmech, g.visco_qp, g.visco_qs, g.visco_f0 = visco
    return g


def visco_fit(nmech, qp, qs, f0):
    ts = (C.c_double * 3)()
    tp, tsh = C.c_double(), C.c_double()
    lib().orc_visco_fit(nmech, qp, qs, f0, ts, C.byref(tp), C.byref(tsh))
    return np.array(ts[:nmech]), tp.value, tsh.value


def make_shot(sx, sy, sz, wavelet, rx0=0, nrx=1, drx=1, ry0=0, nry=1, dry=1, rz=0,
              inject_mode=1):
    s = Shot()
    s.sx, s.sy, s.sz = sx, sy, sz
    w = np.ascontiguousarray(wavelet, np.float32)
    s.nw = len(w)
    s.wavelet = _fp(w)
    s.rx0, s.nrx, s.drx, s.ry0, s.nry, s.dry, s.rz = rx0, nrx, drx, ry0, nry, dry, rz
    s.inject_mode = inject_mode
    s._keep = w  # keep the wavelet buffer alive
    return s


class ExcitationArrays:
    """Excitation state; with angles=True (2D) also the source and receiver P-wave
    propagation angles at the excitation time."""

    def __init__(self, shape, angles: bool = False):
        self.src_angle = np.zeros(shape, np.float32) if angles else None
        self.rcv_angle = np.zeros(shape, np.float32) if angles else None
        self.src_energy = np.zeros(shape, np.float32) if angles else None
        self.rcv_energy = np.zeros(shape, np.float32) if angles else None
        self.amp2 = np.zeros(shape, np.float32)
        self.second2 = np.zeros(shape, np.float32)
        self.time = np.zeros(shape, np.int32)
        self.evx = np.zeros(shape, np.float32)
        self.evy = np.zeros(shape, np.float32)
        self.evz = np.zeros(shape, np.float32)
        self.etp = np.zeros(shape, np.float32)

    def struct(self) -> Excitation:
        e = Excitation()
        e.amp2, e.second2 = _fp(self.amp2), _fp(self.second2)
        e.time = self.time.ctypes.data_as(C.POINTER(C.c_int))
        e.evx, e.evy, e.evz, e.etp = _fp(self.evx), _fp(self.evy), _fp(self.evz), _fp(self.etp)
        e.src_angle, e.rcv_angle = _fp(self.src_angle), _fp(self.rcv_angle)
        e.src_energy, e.rcv_energy = _fp(self.src_energy), _fp(self.rcv_energy)
        return e


def run_pass(g: Grid, vp, vs, rho, shot: Shot, mode: int, nsteps: int, data=None,
             ex: ExcitationArrays | None = None, want_fields=False, bits=64):
    """Run one pass; returns dict with 'data', 'ex', 'pp', 'ps', 'tp', 'fields'."""
    shape = (g.nz, g.ny, g.nx)
    nrec = shot.nrx * shot.nry
    out = {}
    if mode == MODEL:
        data = np.zeros((3, nsteps, nrec), np.float32)
    if mode == SOURCE and ex is None:
        ex = ExcitationArrays(shape)
    pp = ps = tp = None
    if mode == RECEIVER:
        pp, ps, tp = (np.zeros(shape, np.float32) for _ in range(3))
        data = np.ascontiguousarray(data, np.float32)
    fields = np.zeros((13,) + shape, np.float32) if want_fields else None
    exs = ex.struct() if ex is not None else None
    rc = lib(bits).orc_run_pass(C.byref(g), _fp(vp), _fp(vs), _fp(rho), C.byref(shot), mode,
                                nsteps, _fp(data) if data is not None else None,
                                C.byref(exs) if exs is not None else None,
                                _fp(pp), _fp(ps), _fp(tp), _fp(fields))
    if rc != 0:
        raise RuntimeError(f"orc_run_pass failed: {rc}")
    out.update(data=data, ex=ex, pp=pp, ps=ps, tp=tp)
    if want_fields:
        out["fields"] = {n: fields[i] for i, n in enumerate(FIELD_NAMES)}
    return out


def angle_given(tp, vxp, vzp, ex_time, it: int, hw: int, init: float = 0.0):
    """Window propagation angle on given 2D (nz, nx) arrays at the cells whose
    excitation step is `it` (hw 2: the source window, 4: the receiver window);
    other cells keep `init`."""
    nz, nx = tp.shape
    out = np.full((nz, nx), init, np.float32)
    a = [np.ascontiguousarray(v, np.float32) for v in (tp, vxp, vzp)]
    t = np.ascontiguousarray(ex_time, np.int32)
    rc = lib().orc_angle_given(nx, nz, hw, it, *[_fp(v) for v in a],
                               t.ctypes.data_as(C.POINTER(C.c_int)), _fp(out))
    if rc != 0:
        raise RuntimeError(f"orc_angle_given failed: {rc}")
    return out


def divcurl(g: Grid, vp, vs, vx, vy, vz):
    shape = (g.nz, g.ny, g.nx)
    p, sx, sy, sz = (np.zeros(shape, np.float32) for _ in range(4))
    two_d = g.ny == 1
    rc = lib().orc_divcurl(C.byref(g), _fp(vp), _fp(vs), _fp(vx),
                           None if two_d else _fp(vy), _fp(vz), _fp(p),
                           None if two_d else _fp(sx), _fp(sy), None if two_d else _fp(sz))
    if rc != 0:
        raise RuntimeError(f"orc_divcurl failed: {rc}")
    return p, sx, sy, sz


def born_forward(g: Grid, vp, vs, rho, shot: Shot, nt: int, r_vp, r_vs, r_rho, bits=64):
    """Born data [3][nt][nrec] for relative perturbations of (vp, vs, rho); 2D sponge only."""
    data = np.zeros((3, nt, shot.nrx * shot.nry), np.float32)
    args = [np.ascontiguousarray(a, np.float32) for a in (r_vp, r_vs, r_rho)]
    rc = lib(bits).orc_born_forward(C.byref(g), _fp(vp), _fp(vs), _fp(rho), C.byref(shot), nt,
                                    *[_fp(a) for a in args], _fp(data))
    if rc != 0:
        raise RuntimeError(f"orc_born_forward failed: {rc}")
    return data


def born_adjoint(g: Grid, vp, vs, rho, shot: Shot, nt: int, residual, bits=64):
    """Exact transpose of born_forward applied to residual; returns (g_vp, g_vs, g_rho)."""
    shape = (g.nz, g.ny, g.nx)
    out = [np.zeros(shape, np.float32) for _ in range(3)]
    res = np.ascontiguousarray(residual, np.float32)
    rc = lib(bits).orc_born_adjoint(C.byref(g), _fp(vp), _fp(vs), _fp(rho), C.byref(shot), nt,
                                    _fp(res), *[_fp(o) for o in out])
    if rc != 0:
        raise RuntimeError(f"orc_born_adjoint failed: {rc}")
    return tuple(out)


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def stress_step_given(g: Grid, vp, vs, rho, vx, vz, txx, tzz, txz):
    """One 2D stress half-step from given [nz][nx] fields -> (txx, tzz, txz)."""
    shape = (g.nz, g.nx)
    out = [np.zeros(shape, np.float32) for _ in range(3)]
    ins = [_f32(a) for a in (vp, vs, rho, vx, vz, txx, tzz, txz)]
    rc = lib().orc_stress_step_given(C.byref(g), *[_fp(a) for a in ins], *[_fp(o) for o in out])
    if rc != 0:
        raise RuntimeError(f"orc_stress_step_given failed: {rc}")
    return tuple(out)


def born_sources_given(dt_ms, vp, vs, rho, rvp, rvs, rrho, exx, ezz, exz, ax, az):
    """Per-cell Born secondary sources -> (sxx, szz, sxz, svx, svz) increments."""
    ins = [_f32(a).ravel() for a in (vp, vs, rho, rvp, rvs, rrho, exx, ezz, exz, ax, az)]
    n = ins[0].size
    out = [np.zeros(n, np.float32) for _ in range(5)]
    lib().orc_born_sources_given(n, dt_ms, *[_fp(a) for a in ins], *[_fp(o) for o in out])
    return tuple(out)


def image_given(ex, ez, rpx, rpz, rsx, rsz):
    """Per-cell PP and PS excitation-amplitude images (0 where e == 0)."""
    ins = [_f32(a).ravel() for a in (ex, ez, rpx, rpz, rsx, rsz)]
    n = ins[0].size
    pp, ps = np.zeros(n, np.float32), np.zeros(n, np.float32)
    lib().orc_image_given(n, *[_fp(a) for a in ins], _fp(pp), _fp(ps))
    return pp, ps


def visco_model(g: Grid, vp, vs, rho, shot: Shot, nt: int, bits=64):
    """Data [3][nt][nrec] of the Born background scheme (2D; viscoelastic if g.visco_nmech)."""
    data = np.zeros((3, nt, shot.nrx * shot.nry), np.float32)
    rc = lib(bits).orc_visco_model(C.byref(g), _fp(vp), _fp(vs), _fp(rho), C.byref(shot), nt, _fp(data))
    if rc != 0:
        raise RuntimeError(f"orc_visco_model failed: {rc}")
    return data
