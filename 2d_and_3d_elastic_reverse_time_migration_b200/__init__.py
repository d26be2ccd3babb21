"""B200-native elastic reverse-time migration: Python front end of libertm.so.

The C ABI (include/ertm.h) is the product boundary; this module is a thin
ctypes mirror of it whose method names follow the reference's per-shot calls
(3D_elastic_RTM/3D_forward_or_back_together.cu):

    ctx = Context(Config(nx=..., ny=..., nz=..., dx=..., dy=..., dz=..., dt_ms=..., nt=...))
    ctx.set_model(TRUE_MODEL, vp, vs, rho)
    ctx.set_model(MIGRATION_MODEL, svp, svs, srho)
    data = ctx.forward_together_using_real_model(shot)             # observed data
    ctx.forward_together_using_smoothed_model(shot)                 # source pass
    pp, ps, tp = ctx.backward_together_using_smoothed_model(shot, data)  # receiver pass

Arrays are float32 with shape (nz, ny, nx) (x fastest).  Inputs and outputs
may be numpy arrays (host) or CUDA torch tensors (passed by pointer, no copy).
There is no CPU fallback: if libertm.so is missing or no GPU is present the
calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libertm.so")

TRUE_MODEL, MIGRATION_MODEL = 0, 1
BOUNDARY_CPML, BOUNDARY_SPONGE_COS, BOUNDARY_SPONGE_CUBIC = 0, 1, 2
COEF_TAYLOR, COEF_REFERENCE12, COEF_USER = 0, 1, 2
INJECT_ADD, INJECT_REPLACE = 1, 2
STEP_SINGLE, STEP_PAIRS = 0, 1
MULTI_MAX = 10          # shots per ertm_rtm_multi call (ERTM_MULTI_MAX)
FIELDS = ("vx", "vy", "vz", "txx", "tyy", "tzz", "txy", "txz", "tyz", "tp", "vxp", "vyp", "vzp")
ERRORS = {0: "OK", -1: "EINVAL", -2: "ENOMEM", -3: "ECUDA", -4: "ESTATE", -5: "ENOTSUP",
          -6: "EDEVICE"}


class ErtmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class _Config(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("dx", C.c_float), ("dy", C.c_float), ("dz", C.c_float),
                ("dt_ms", C.c_float), ("nt", C.c_int), ("src_steps", C.c_int),
                ("order", C.c_int), ("coef_kind", C.c_int), ("coef", C.c_float * 8),
                ("boundary", C.c_int), ("pml", C.c_int * 6), ("pml_r", C.c_float),
                ("pml_f0", C.c_float), ("pml_vmax", C.c_float), ("sponge_coef", C.c_float),
                ("device", C.c_int), ("checkpoint_every", C.c_int), ("autotune", C.c_int),
                ("visco_nmech", C.c_int), ("visco_qp", C.c_float), ("visco_qs", C.c_float),
                ("visco_f0", C.c_float), ("reserved", C.c_int * 1)]


class _Shot(C.Structure):
    _fields_ = [("sx", C.c_int), ("sy", C.c_int), ("sz", C.c_int), ("nw", C.c_int),
                ("wavelet", C.c_void_p),
                ("rx0", C.c_int), ("nrx", C.c_int), ("drx", C.c_int),
                ("ry0", C.c_int), ("nry", C.c_int), ("dry", C.c_int),
                ("rz", C.c_int), ("inject_mode", C.c_int)]


class _Window(C.Structure):
    _fields_ = [("x0", C.c_int), ("y0", C.c_int), ("wx", C.c_int), ("wy", C.c_int),
                ("nt", C.c_int), ("src_steps", C.c_int)]


class _NnAct(C.Structure):
    _fields_ = [("data", C.c_void_p), ("n", C.c_int), ("h", C.c_int), ("w", C.c_int),
                ("cstride", C.c_int), ("coff", C.c_int), ("c", C.c_int)]


# every entry point of include/ertm.h: name -> (restype, argtypes)
_P = C.c_void_p
SIGNATURES = {
    "ertm_abi_version": (C.c_int, []),
    "ertm_create": (C.c_int, [C.POINTER(_Config), C.POINTER(_P)]),
    "ertm_destroy": (C.c_int, [_P]),
    "ertm_last_error": (C.c_int, [_P, C.c_char_p, C.c_size_t]),
    "ertm_set_stream": (C.c_int, [_P, _P]),
    "ertm_set_model": (C.c_int, [_P, C.c_int, _P, _P, _P]),
    "ertm_set_grid": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int]),
    "ertm_rtm_windows": (C.c_int, [C.POINTER(_Config), _P, _P, _P, C.c_int, C.POINTER(_Window),
                                   C.POINTER(_Shot), C.POINTER(_P), C.c_int, _P, _P, _P,
                                   C.c_char_p, C.c_size_t]),
    "ertm_forward_together_using_real_model": (C.c_int, [_P, C.POINTER(_Shot), _P]),
    "ertm_forward_together_using_smoothed_model": (C.c_int, [_P, C.POINTER(_Shot)]),
    "ertm_backward_together_using_smoothed_model": (C.c_int, [_P, C.POINTER(_Shot), _P, _P, _P, _P]),
    "ertm_rtm_shot": (C.c_int, [_P, C.POINTER(_Shot), _P, _P, _P, _P]),
    "ertm_rtm_batch": (C.c_int, [_P, C.POINTER(_Shot), C.c_int, C.POINTER(_P), _P, _P, _P]),
    "ertm_rtm_multi": (C.c_int, [C.POINTER(_P), C.c_int, C.POINTER(_Shot), C.POINTER(_P), C.POINTER(_P),
                                 C.POINTER(_P), C.POINTER(_P)]),
    "ertm_get_wavefield": (C.c_int, [_P, C.c_int, _P]),
    "ertm_get_excitation": (C.c_int, [_P, _P, _P, _P, _P, _P, _P]),
    "ertm_set_angles": (C.c_int, [_P, C.c_int]),
    "ertm_get_angles": (C.c_int, [_P, _P, _P]),
    "ertm_angle_compensate": (C.c_int, [_P, _P, _P, _P, C.c_longlong, C.c_int, _P]),
    "ertm_adcig_bin": (C.c_int, [_P, _P, _P, _P, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int,
                                 C.c_int, C.c_float, _P]),
    "ertm_divcurl": (C.c_int, [_P, C.c_int, _P, _P, _P, _P]),
    "ertm_propagate": (C.c_int, [_P, C.c_int, C.POINTER(_Shot), C.c_int]),
    "ertm_time_kernels": (C.c_int, [_P, C.POINTER(_Shot), C.c_int, C.POINTER(C.c_float)]),
    "ertm_kernel_launches": (C.c_int64, [_P]),
    "ertm_set_wait_fault": (C.c_int, [_P, C.c_int, C.c_uint32]),
    "ertm_set_step_variant": (C.c_int, [_P, C.c_int]),
    "ertm_born_forward": (C.c_int, [_P, C.POINTER(_Shot), _P, _P, _P, _P]),
    "ertm_born_adjoint": (C.c_int, [_P, C.POINTER(_Shot), _P, _P, _P, _P]),
    "ertm_born_forward_shots": (C.c_int, [_P, C.POINTER(_Shot), C.c_int, _P, _P, _P, _P]),
    "ertm_born_adjoint_shots": (C.c_int, [_P, C.POINTER(_Shot), C.c_int, _P, _P, _P, _P]),
    "ertm_write_volume_xyz": (C.c_int, [C.c_char_p, _P] + [C.c_int] * 9),
    "ertm_read_volume_xyz": (C.c_int, [C.c_char_p, _P] + [C.c_int] * 9),
    "ertm_laplace_filter": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                      C.c_float]),
    "ertm_hilbert_z": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int]),
    "ertm_bell_smooth": (C.c_int, [_P, _P, _P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _P]),
    "ertm_taper_x": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _P]),
    "ertm_aperture_taper": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                      _P]),
    "ertm_mute_direct": (C.c_int, [C.POINTER(_Shot), _P, C.c_int, C.c_float, C.c_float, C.c_float,
                                   C.c_float, C.c_float, C.c_int, _P]),
    "ertm_nn_gemm": (C.c_int, [_P, _P, _P, C.c_int, C.c_int, C.c_int, _P, _P]),
    "ertm_nn_conv3x3": (C.c_int, [C.POINTER(_NnAct), _P, _P, C.POINTER(_NnAct), C.c_int, _P, _P, _P]),
    "ertm_nn_conv3x3_dgrad": (C.c_int, [C.POINTER(_NnAct), _P, C.POINTER(_NnAct), C.POINTER(_NnAct),
                                        _P, _P]),
    "ertm_nn_conv3x3_wgrad": (C.c_int, [C.POINTER(_NnAct), C.POINTER(_NnAct), _P, C.c_int, _P, _P]),
    "ertm_nn_up2": (C.c_int, [C.POINTER(_NnAct), _P, _P, C.POINTER(_NnAct), C.c_int, _P, _P]),
    "ertm_nn_up2_dgrad": (C.c_int, [C.POINTER(_NnAct), _P, C.POINTER(_NnAct), C.POINTER(_NnAct), _P,
                                    _P]),
    "ertm_nn_up2_wgrad": (C.c_int, [C.POINTER(_NnAct), C.POINTER(_NnAct), _P, C.c_int, _P, _P]),
    "ertm_nn_pool2": (C.c_int, [C.POINTER(_NnAct), _P, _P]),
    "ertm_nn_pool2_bwd": (C.c_int, [C.POINTER(_NnAct), _P, C.POINTER(_NnAct), C.c_int, _P]),
    "ertm_nn_bias_grad": (C.c_int, [C.POINTER(_NnAct), _P, _P]),
    "ertm_nn_mse": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_longlong, C.c_float, _P, _P, _P]),
    "ertm_nn_adam": (C.c_int, [_P, _P, _P, _P, _P, C.c_longlong, C.c_float, C.c_float, C.c_float,
                               C.c_float, C.c_int, _P]),
    "ertm_nn_flip3": (C.c_int, [_P, _P, C.c_int, C.c_int, _P]),
    "ertm_nn_transpose": (C.c_int, [_P, _P, C.c_int, C.c_int, _P]),
    "ertm_nn_to_bf16": (C.c_int, [_P, _P, C.c_longlong, _P]),
    "ertm_forward_together_using_real_model_noalloc": (
        C.c_int, [C.POINTER(_Config), _P, _P, _P, C.POINTER(_Shot), _P, _P, C.c_char_p, C.c_size_t]),
}

_lib_handle: C.CDLL | None = None


def lib() -> C.CDLL:
    """Load libertm.so (built by build.py); raise if it is missing."""
    global _lib_handle
    if _lib_handle is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libertm.so not built ({LIB_PATH}); run __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib_handle = L
    return _lib_handle


@dataclass
class Config:
    """Mirror of ertm_config (grid includes the absorbing layers; dt in ms)."""
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    dt_ms: float
    nt: int
    src_steps: int = 0
    order: int = 8
    coef_kind: int = COEF_TAYLOR
    coef: tuple = ()
    boundary: int = BOUNDARY_CPML
    pml: tuple = (0, 0, 0, 0, 0, 0)
    pml_r: float = 1e-3
    pml_f0: float = 10.0
    pml_vmax: float = 0.0
    sponge_coef: float = 0.0
    device: int = 0
    checkpoint_every: int = 0
    autotune: int = 0
    visco_nmech: int = 0
    visco_qp: float = 0.0
    visco_qs: float = 0.0
    visco_f0: float = 0.0

    def struct(self) -> _Config:
        c = _Config()
        for f in ("nx", "ny", "nz", "dx", "dy", "dz", "dt_ms", "nt", "src_steps", "order",
                  "coef_kind", "boundary", "pml_r", "pml_f0", "pml_vmax", "sponge_coef", "device",
                  "checkpoint_every", "autotune", "visco_nmech", "visco_qp", "visco_qs",
                  "visco_f0"):
            setattr(c, f, getattr(self, f))
        for i, v in enumerate(self.coef[:8]):
            c.coef[i] = v
        for i in range(6):
            c.pml[i] = int(self.pml[i])
        return c

    @property
    def shape(self):
        return (self.nz, self.ny, self.nx)


@dataclass
class Shot:
    """Mirror of ertm_shot: explosive source cell, wavelet, receiver grid."""
    sx: int
    sy: int
    sz: int
    wavelet: np.ndarray
    rx0: int = 0
    nrx: int = 0
    drx: int = 1
    ry0: int = 0
    nry: int = 1
    dry: int = 1
    rz: int = 0
    inject_mode: int = INJECT_ADD
    _keep: list = field(default_factory=list, repr=False)

    @property
    def nrec(self) -> int:
        return self.nrx * self.nry

    def struct(self) -> _Shot:
        s = _Shot()
        s.sx, s.sy, s.sz = self.sx, self.sy, self.sz
        w = self.wavelet
        if _is_torch(w):
            s.nw = int(w.numel())
            s.wavelet = w.data_ptr()
        else:
            w = np.ascontiguousarray(w, np.float32)
            self._keep[:] = [w]
            s.nw = len(w)
            s.wavelet = w.ctypes.data
        s.rx0, s.nrx, s.drx = self.rx0, self.nrx, self.drx
        s.ry0, s.nry, s.dry = self.ry0, self.nry, self.dry
        s.rz, s.inject_mode = self.rz, self.inject_mode
        return s


def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


def _ptr(a, n: int | None = None, writable: bool = False):
    """Raw pointer of a float32/int32 numpy array or torch tensor (contiguous)."""
    if a is None:
        return None
    if _is_torch(a):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        if n is not None and a.numel() != n:
            raise ValueError(f"tensor has {a.numel()} elements, expected {n}")
        return a.data_ptr()
    if not isinstance(a, np.ndarray) or not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be a C-contiguous numpy array")
    if a.dtype not in (np.float32, np.int32):
        raise ValueError(f"dtype {a.dtype}: float32/int32 expected")
    if n is not None and a.size != n:
        raise ValueError(f"array has {a.size} elements, expected {n}")
    if writable and not a.flags["WRITEABLE"]:
        raise ValueError("output array is read-only")
    return a.ctypes.data


def _pass_steps(cfg, name: str) -> int:
    """Time steps a pass call runs (for the run log's cell-update rates)."""
    src = cfg.src_steps or (2 * cfg.nt) // 3
    return {"forward_together_using_real_model": cfg.nt, "forward_together_using_smoothed_model": src,
            "backward_together_using_smoothed_model": cfg.nt, "rtm_shot": src + cfg.nt,
            "born_forward": 2 * cfg.nt, "born_adjoint": 3 * cfg.nt,
            "born_forward_shots": 2 * cfg.nt, "born_adjoint_shots": 3 * cfg.nt}.get(name, 0)


def _logged(fn):
    """Appends one JSON line per call to the context's run log (`Context.set_log`):
    the call, its wall time (the calls are synchronous), and cell-updates per
    second over the passes it runs (Born calls count background and scattered
    wavefields, and the adjoint its background rebuild)."""
    import functools
    import json
    import time

    @functools.wraps(fn)
    def wrap(self, *a, **k):
        if not getattr(self, "_log", None):
            return fn(self, *a, **k)
        t0 = time.perf_counter()
        out = fn(self, *a, **k)
        dt = time.perf_counter() - t0
        steps = _pass_steps(self.cfg, fn.__name__)
        if fn.__name__.endswith("_shots"):
            steps *= len(a[0])          # every shot of the call
        rec = {"event": "pass", "call": fn.__name__, "cells": self.ncell, "cell_steps": self.ncell * steps,
               "seconds": round(dt, 6), "gcell_s": round(self.ncell * steps / dt / 1e9, 4) if dt > 0 else None}
        with open(self._log, "a") as f:
            f.write(json.dumps(rec) + "\n")
        return out

    return wrap


class Context:
    """One GPU context: device state of one grid (the reference's GPUdevice)."""

    _log = None

    def set_log(self, path: str | None):
        """Append a JSON line per pass call to `path` (None stops logging)."""
        self._log = path

    def __init__(self, cfg: Config):
        self.cfg = cfg
        self._L = lib()
        h = C.c_void_p()
        self._cs = cfg.struct()
        rc = self._L.ertm_create(C.byref(self._cs), C.byref(h))
        if rc != 0:
            raise ErtmError(rc, self._msg(None))
        self._h = h

    def _msg(self, h) -> str:
        buf = C.create_string_buffer(1024)
        self._L.ertm_last_error(h, buf, len(buf))
        return buf.value.decode(errors="replace")

    def _ck(self, rc: int):
        if rc != 0:
            raise ErtmError(rc, self._msg(self._h))

    def close(self):
        if getattr(self, "_h", None):
            self._L.ertm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def ncell(self) -> int:
        return self.cfg.nx * self.cfg.ny * self.cfg.nz

    def _vol(self, out):
        return np.zeros(self.cfg.shape, np.float32) if out is None else out

    def set_stream(self, stream_ptr: int | None):
        self._ck(self._L.ertm_set_stream(self._h, stream_ptr))

    def set_grid(self, nx: int, ny: int, nt: int, src_steps: int = 0):
        """Shrink (or restore) the active grid; models must be set again afterwards."""
        self._ck(self._L.ertm_set_grid(self._h, nx, ny, nt, src_steps))
        self.cfg = Config(**{**self.cfg.__dict__, "nx": nx, "ny": ny, "nt": nt,
                             "src_steps": src_steps})

    def set_model(self, which: int, vp, vs, rho):
        n = self.ncell
        args = [vp, vs, rho]
        args = [a if _is_torch(a) else np.ascontiguousarray(a, np.float32) for a in args]
        self._ck(self._L.ertm_set_model(self._h, which, *[_ptr(a, n) for a in args]))

    @_logged
    def forward_together_using_real_model(self, shot: Shot, out=None):
        n = 3 * self.cfg.nt * shot.nrec
        if out is None:
            out = np.zeros((3, self.cfg.nt, shot.nrec), np.float32)
        s = shot.struct()
        self._ck(self._L.ertm_forward_together_using_real_model(self._h, C.byref(s),
                                                                _ptr(out, n, True)))
        return out

    @_logged
    def forward_together_using_smoothed_model(self, shot: Shot):
        s = shot.struct()
        self._ck(self._L.ertm_forward_together_using_smoothed_model(self._h, C.byref(s)))

    @_logged
    def backward_together_using_smoothed_model(self, shot: Shot, data, pp=None, ps=None, tp=None):
        n = self.ncell
        pp, ps, tp = self._vol(pp), self._vol(ps), self._vol(tp)
        d = data if _is_torch(data) else np.ascontiguousarray(data, np.float32)
        s = shot.struct()
        self._ck(self._L.ertm_backward_together_using_smoothed_model(
            self._h, C.byref(s), _ptr(d, 3 * self.cfg.nt * shot.nrec), _ptr(pp, n, True),
            _ptr(ps, n, True), _ptr(tp, n, True)))
        return pp, ps, tp

    @_logged
    def rtm_shot(self, shot: Shot, data, pp=None, ps=None, tp=None):
        n = self.ncell
        pp, ps, tp = self._vol(pp), self._vol(ps), self._vol(tp)
        d = data if _is_torch(data) else np.ascontiguousarray(data, np.float32)
        s = shot.struct()
        self._ck(self._L.ertm_rtm_shot(self._h, C.byref(s), _ptr(d, 3 * self.cfg.nt * shot.nrec),
                                       _ptr(pp, n, True), _ptr(ps, n, True), _ptr(tp, n, True)))
        return pp, ps, tp

    def rtm_batch(self, shots: list, data: list, pp=None, ps=None, tp=None):
        """RTM of several shots with the images stacked on the device."""
        n = self.ncell
        pp, ps, tp = self._vol(pp), self._vol(ps), self._vol(tp)
        arr = (_Shot * max(1, len(shots)))()
        keep = []
        for q, sh in enumerate(shots):
            arr[q] = sh.struct()
        ptrs = (C.c_void_p * max(1, len(data)))()
        for q, (sh, d) in enumerate(zip(shots, data)):
            d = d if _is_torch(d) else np.ascontiguousarray(d, np.float32)
            keep.append(d)
            ptrs[q] = _ptr(d, 3 * self.cfg.nt * sh.nrec)
        self._ck(self._L.ertm_rtm_batch(self._h, arr, len(shots), ptrs, _ptr(pp, n, True),
                                        _ptr(ps, n, True), _ptr(tp, n, True)))
        del keep
        return pp, ps, tp

    def get_wavefield(self, name_or_id, out=None):
        fid = FIELDS.index(name_or_id) if isinstance(name_or_id, str) else int(name_or_id)
        out = self._vol(out)
        self._ck(self._L.ertm_get_wavefield(self._h, fid, _ptr(out, self.ncell, True)))
        return out

    def get_excitation(self):
        n = self.ncell
        amp = np.zeros(self.cfg.shape, np.float32)
        t = np.zeros(self.cfg.shape, np.int32)
        ev = [np.zeros(self.cfg.shape, np.float32) for _ in range(4)]
        self._ck(self._L.ertm_get_excitation(self._h, _ptr(amp, n, True), _ptr(t, n, True),
                                             *[_ptr(e, n, True) for e in ev]))
        return {"amp": amp, "time": t, "evx": ev[0], "evy": ev[1], "evz": ev[2], "etp": ev[3]}

    def set_angles(self, on: bool = True):
        """Capture source / receiver P-wave propagation angles at the excitation
        time in the following passes (2D; see ertm_set_angles)."""
        self._ck(self._L.ertm_set_angles(self._h, 1 if on else 0))

    def get_angles(self, src: bool = True, rcv: bool = True):
        """(source angle, receiver angle) in degrees, (nz, 1, nx); None where not asked."""
        n = self.ncell
        a = np.zeros(self.cfg.shape, np.float32) if src else None
        b = np.zeros(self.cfg.shape, np.float32) if rcv else None
        self._ck(self._L.ertm_get_angles(self._h, _ptr(a, n, True), _ptr(b, n, True)))
        return a, b

    def divcurl(self, which: int = MIGRATION_MODEL):
        n = self.ncell
        outs = [np.zeros(self.cfg.shape, np.float32) for _ in range(4)]
        self._ck(self._L.ertm_divcurl(self._h, which, *[_ptr(o, n, True) for o in outs]))
        return tuple(outs)

    def propagate(self, which: int, shot: Shot, nsteps: int):
        s = shot.struct()
        self._ck(self._L.ertm_propagate(self._h, which, C.byref(s), nsteps))

    def time_kernels(self, shot: Shot, nsteps: int):
        ms = (C.c_float * 2)()
        s = shot.struct()
        self._ck(self._L.ertm_time_kernels(self._h, C.byref(s), nsteps, ms))
        return float(ms[0]), float(ms[1])

    @_logged
    def born_forward(self, shot: Shot, r_vp, r_vs, r_rho, out=None):
        """Linearised data (3, nt, nrec) for relative perturbations of the migration model."""
        n = self.ncell
        if out is None:
            out = np.zeros((3, self.cfg.nt, shot.nrec), np.float32)
        args = [a if _is_torch(a) else np.ascontiguousarray(a, np.float32) for a in (r_vp, r_vs, r_rho)]
        s = shot.struct()
        self._ck(self._L.ertm_born_forward(self._h, C.byref(s), *[_ptr(a, n) for a in args],
                                           _ptr(out, 3 * self.cfg.nt * shot.nrec, True)))
        return out

    @_logged
    def born_adjoint(self, shot: Shot, residual, g_vp=None, g_vs=None, g_rho=None):
        """Transpose of born_forward applied to residual (3, nt, nrec): (g_vp, g_vs, g_rho)."""
        n = self.ncell
        outs = [self._vol(o) for o in (g_vp, g_vs, g_rho)]
        r = residual if _is_torch(residual) else np.ascontiguousarray(residual, np.float32)
        s = shot.struct()
        self._ck(self._L.ertm_born_adjoint(self._h, C.byref(s), _ptr(r, 3 * self.cfg.nt * shot.nrec),
                                           *[_ptr(o, n, True) for o in outs]))
        return tuple(outs)

    def _shot_array(self, shots):
        arr = (_Shot * len(shots))()
        keep = []
        for i, sh in enumerate(shots):
            st = sh.struct()
            keep.append(st)
            arr[i] = st
        return arr, keep

    @_logged
    def born_forward_shots(self, shots, r_vp, r_vs, r_rho, out=None):
        """Linearised data of every shot, (nshots, 3, nt, nrec): the shots share each step's
        kernel launches (ertm_born_forward_shots)."""
        n, ns = self.ncell, len(shots)
        nrec = shots[0].nrec
        if out is None:
            out = np.zeros((ns, 3, self.cfg.nt, nrec), np.float32)
        args = [a if _is_torch(a) else np.ascontiguousarray(a, np.float32) for a in (r_vp, r_vs, r_rho)]
        arr, keep = self._shot_array(shots)
        self._ck(self._L.ertm_born_forward_shots(self._h, arr, ns, *[_ptr(a, n) for a in args],
                                                 _ptr(out, ns * 3 * self.cfg.nt * nrec, True)))
        del keep
        return out

    @_logged
    def born_adjoint_shots(self, shots, residual, g_vp=None, g_vs=None, g_rho=None):
        """Gradient summed over the shots for residuals (nshots, 3, nt, nrec)
        (ertm_born_adjoint_shots): (g_vp, g_vs, g_rho)."""
        n, ns = self.ncell, len(shots)
        outs = [self._vol(o) for o in (g_vp, g_vs, g_rho)]
        r = residual if _is_torch(residual) else np.ascontiguousarray(residual, np.float32)
        arr, keep = self._shot_array(shots)
        self._ck(self._L.ertm_born_adjoint_shots(self._h, arr, ns,
                                                 _ptr(r, ns * 3 * self.cfg.nt * shots[0].nrec),
                                                 *[_ptr(o, n, True) for o in outs]))
        del keep
        return tuple(outs)

    @property
    def kernel_launches(self) -> int:
        return int(self._L.ertm_kernel_launches(self._h))

    def set_step_variant(self, variant: int):
        """3D step kernels: STEP_SINGLE (one cell per thread, default) or STEP_PAIRS."""
        self._ck(self._L.ertm_set_step_variant(self._h, int(variant)))

    def set_wait_fault(self, plane: int = -1, polls: int = 0):
        """Test hook of the device-error path: the first CTA of each step kernel skips
        the staged copy of its z plane `plane`, so its bounded wait runs out after
        `polls` polls (0: default) and the pass raises ErtmError(ERTM_EDEVICE);
        plane = -1 turns it off."""
        self._ck(self._L.ertm_set_wait_fault(self._h, int(plane), int(polls)))


def forward_together_using_real_model_noalloc(cfg: Config, vp, vs, rho, shot: Shot, out,
                                              stream_ptr: int | None = None):
    """Modelling pass that allocates no GPU memory (see include/ertm.h).

    For callers that may not allocate device memory when they call in: every
    array (vp, vs, rho, shot.wavelet, out of shape (3, nt, nrec)) must already be
    a CUDA tensor; the library's wavefields live in a fixed 64 MiB device array.
    Calls share that array, so calls that overlap on the GPU race."""
    L = lib()
    n = cfg.nx * cfg.ny * cfg.nz
    cs, ss = cfg.struct(), shot.struct()
    buf = C.create_string_buffer(512)
    rc = L.ertm_forward_together_using_real_model_noalloc(
        C.byref(cs), _ptr(vp, n), _ptr(vs, n), _ptr(rho, n), C.byref(ss),
        _ptr(out, 3 * cfg.nt * shot.nrec), stream_ptr, buf, len(buf))
    if rc != 0:
        raise ErtmError(rc, buf.value.decode(errors="replace"))
    return out


@dataclass
class Window:
    """Mirror of ertm_window: aperture of one shot over a shared model (model cells)."""
    x0: int
    y0: int
    wx: int
    wy: int
    nt: int
    src_steps: int = 0

    def struct(self) -> _Window:
        w = _Window()
        w.x0, w.y0, w.wx, w.wy, w.nt, w.src_steps = (self.x0, self.y0, self.wx, self.wy, self.nt,
                                                      self.src_steps)
        return w


def rtm_multi(contexts: list, shots: list, data: list, outs: list | None = None):
    """Several 3D shots migrated together, shot q on contexts[q] (its own grid and
    migration model), one launch of each step kernel per time step for all of them
    (ertm_rtm_multi in include/ertm.h).  Returns [(pp, ps, tp)] per shot, into
    `outs` when given (host or device volumes of each context's grid)."""
    L = lib()
    n = len(contexts)
    if not (1 <= n <= MULTI_MAX) or len(shots) != n or len(data) != n:
        raise ValueError(f"rtm_multi: 1 .. {MULTI_MAX} contexts, one shot and one record each")
    outs = outs or [tuple(c._vol(None) for _ in range(3)) for c in contexts]
    hs = (C.c_void_p * n)(*[c._h for c in contexts])
    arr = (_Shot * n)(*[sh.struct() for sh in shots])
    keep, dp = [], (C.c_void_p * n)()
    for q, (c, sh, d) in enumerate(zip(contexts, shots, data)):
        d = d if _is_torch(d) else np.ascontiguousarray(d, np.float32)
        keep.append(d)
        dp[q] = _ptr(d, 3 * c.cfg.nt * sh.nrec)
    op = [(C.c_void_p * n)() for _ in range(3)]
    for q, (c, o) in enumerate(zip(contexts, outs)):
        for k in range(3):
            op[k][q] = _ptr(o[k], c.ncell, True)
    rc = L.ertm_rtm_multi(hs, n, arr, dp, op[0], op[1], op[2])
    del keep
    if rc != 0:
        raise ErtmError(rc, contexts[0]._msg(contexts[0]._h))
    return outs


def rtm_windows(base: Config, vp, vs, rho, windows: list, shots: list, data: list,
                lanes: int = MULTI_MAX, pp=None, ps=None, tp=None):
    """Batched RTM over aperture windows of one shared migration model (model cells,
    no absorbing layers, shape (nz, ny, nx) = base.shape); images stacked into
    pp, ps, tp of the model's shape; `lanes` 3D shots per launch (up to MULTI_MAX).
    See ertm_rtm_windows in include/ertm.h."""
    L = lib()
    n = base.nx * base.ny * base.nz
    outs = [np.zeros(base.shape, np.float32) if o is None else o for o in (pp, ps, tp)]
    model = [a if _is_torch(a) else np.ascontiguousarray(a, np.float32) for a in (vp, vs, rho)]
    k = max(1, len(shots))
    warr, sarr, parr = (_Window * k)(), (_Shot * k)(), (C.c_void_p * k)()
    keep = []
    for q, (w, sh, d) in enumerate(zip(windows, shots, data)):
        warr[q] = w.struct()
        sarr[q] = sh.struct()
        d = d if _is_torch(d) else np.ascontiguousarray(d, np.float32)
        keep.append(d)
        parr[q] = _ptr(d, 3 * w.nt * sh.nrec)
    cs = base.struct()
    buf = C.create_string_buffer(1024)
    rc = L.ertm_rtm_windows(C.byref(cs), *[_ptr(a, n) for a in model], len(shots), warr, sarr, parr,
                            lanes, *[_ptr(o, n, True) for o in outs], buf, len(buf))
    del keep
    if rc != 0:
        raise ErtmError(rc, buf.value.decode(errors="replace"))
    return tuple(outs)


def write_volume_xyz(path: str, vol, cut=None):
    """Write a (nz, ny, nx) float32 volume in the reference's x-outer, z-inner raw
    format; cut = (nx, ny, nz, bl, bf, bu) writes only that interior block
    (output_file_xyz_boundary)."""
    v = np.ascontiguousarray(vol, np.float32)
    nzb, nyb, nxb = v.shape
    nx, ny, nz, bl, bf, bu = cut if cut else (nxb, nyb, nzb, 0, 0, 0)
    rc = lib().ertm_write_volume_xyz(os.fsencode(path), v.ctypes.data, nxb, nyb, nzb, nx, ny, nz, bl, bf, bu)
    if rc != 0:
        raise ErtmError(rc, f"cannot write {path}")


def read_volume_xyz(path: str, nx: int, ny: int, nz: int, into=None, offsets=(0, 0, 0)):
    """Read an x-outer raw float32 volume of nx*ny*nz values into a (nz, ny, nx)
    array, or into the interior of `into` at offsets (bl, bf, bu)
    (input_file_xyz_boundary)."""
    out = np.zeros((nz, ny, nx), np.float32) if into is None else into
    if not (isinstance(out, np.ndarray) and out.dtype == np.float32 and out.flags["C_CONTIGUOUS"]):
        raise ValueError("into must be a C-contiguous float32 array")
    nzb, nyb, nxb = out.shape
    bl, bf, bu = offsets
    rc = lib().ertm_read_volume_xyz(os.fsencode(path), out.ctypes.data, nxb, nyb, nzb, nx, ny, nz, bl, bf, bu)
    if rc != 0:
        raise ErtmError(rc, f"cannot read {path}")
    return out


def _cut(cfg):
    bl, _, bf, _, bu, _ = cfg.pml
    nxi = cfg.nx - cfg.pml[0] - cfg.pml[1]
    nyi = cfg.ny - cfg.pml[2] - cfg.pml[3]
    nzi = cfg.nz - cfg.pml[4] - cfg.pml[5]
    return (nxi, nyi, nzi, bl, bf, bu)


def write_shot_results(directory: str, cfg: Config, shot: Shot, pp, ps, tp, vsp: bool = False,
                       prefix: str = "result"):
    """One shot's images as the reference writes them (output_3d_result,
    3D_output_file.cu:309-428): `<prefix>-tp-<sy>-<sx>`, `-pp-`, `-ps-` in
    `directory`, x-outer raw float32 with the absorbing layers cut off; sx, sy are
    the shot's interior cell (the padded cell minus boundary_left / the y offset).
    With vsp the names carry the interior source depth instead (`<prefix>-tp-<sz>`).
    prefix "compensate-result" gives output_3d_result_compensate's names."""
    os.makedirs(directory, exist_ok=True)
    cut = _cut(cfg)
    sx, sy, sz = shot.sx - cut[3], shot.sy - cut[4], shot.sz - cut[5]
    tag = f"{sz}" if vsp else f"{sy}-{sx}"
    paths = []
    for name, vol in (("tp", tp), ("pp", pp), ("ps", ps)):
        path = os.path.join(directory, f"{prefix}-{name}-{tag}")
        write_volume_xyz(path, vol, cut)
        paths.append(path)
    return paths


def write_excitation_files(directory: str, cfg: Config, shot: Shot, ex: dict):
    """The excitation arrays of one shot as the reference writes them
    (output_3d_wavefiled_excitation_amp_time, 3D_output_file.cu:155-250):
    `ex-time-<sy>-<sx>` (whole padded grid) and `cut-ex-time`, `cut-ex-amp`,
    `cut-ex-tp`, `cut-ex-vxp`, `cut-ex-vyp`, `cut-ex-vzp` (interior), x-outer raw
    float32 (the excitation time as a float, as the reference stores it).  `ex` is
    `Context.get_excitation()`."""
    os.makedirs(directory, exist_ok=True)
    cut = _cut(cfg)
    sx, sy = shot.sx - cut[3], shot.sy - cut[4]
    tag = f"{sy}-{sx}"
    t = np.asarray(ex["time"], np.float32)
    write_volume_xyz(os.path.join(directory, f"ex-time-{tag}"), t)
    out = [os.path.join(directory, f"ex-time-{tag}")]
    for name, key in (("time", "time"), ("amp", "amp"), ("tp", "etp"), ("vxp", "evx"), ("vyp", "evy"),
                      ("vzp", "evz")):
        path = os.path.join(directory, f"cut-ex-{name}-{tag}")
        write_volume_xyz(path, np.asarray(ex[key], np.float32), cut)
        out.append(path)
    return out


def write_shot_gathers(prefix: str, data):
    """Recorded data [3][nt][nrec] -> prefix_x.bin, prefix_y.bin, prefix_z.bin, each
    raw float32 [nrec][nt] (receiver-major, time fastest)."""
    d = np.asarray(data, np.float32)
    for c, name in enumerate("xyz"):
        np.ascontiguousarray(d[c].T).tofile(f"{prefix}_{name}.bin")


def read_shot_gathers(prefix: str, nt: int, nrec: int):
    out = np.zeros((3, nt, nrec), np.float32)
    for c, name in enumerate("xyz"):
        out[c] = np.fromfile(f"{prefix}_{name}.bin", np.float32).reshape(nrec, nt).T
    return out


def mute_direct(shot: Shot, data, dt_ms: float, h: tuple, v: float, extra: int = 0, stream_ptr=None):
    """Zero the direct arrival in recorded data [3][nt][nrec] (numpy or CUDA tensor),
    in place; h = (dx, dy, dz) in m, v in m/s (see ertm_mute_direct)."""
    nt = data.shape[1]
    s = shot.struct()
    if _is_torch(data):
        p = _ptr(data, 3 * nt * shot.nrec)
    else:
        if not (isinstance(data, np.ndarray) and data.dtype == np.float32 and data.flags["C_CONTIGUOUS"]):
            raise ValueError("data must be a C-contiguous float32 array")
        p = data.ctypes.data
    rc = lib().ertm_mute_direct(C.byref(s), p, nt, h[0], h[1], h[2], dt_ms, v, extra, stream_ptr)
    if rc != 0:
        raise ErtmError(rc, "mute_direct")
    return data


def laplace_filter(img, vp, h: tuple):
    """Laplacian image filter (see ertm_laplace_filter); returns a new (nz, ny, nx) array."""
    out = np.array(img, np.float32, order="C", copy=True)
    v = np.ascontiguousarray(vp, np.float32)
    if out.ndim != 3 or v.shape != out.shape:
        raise ValueError("img and vp must be (nz, ny, nx) arrays of one shape")
    nz, ny, nx = out.shape
    rc = lib().ertm_laplace_filter(out.ctypes.data, v.ctypes.data, nx, ny, nz, *h)
    if rc != 0:
        raise ErtmError(rc, "laplace_filter")
    return out


def hilbert_z(img):
    """Hilbert transform along depth of every column (see ertm_hilbert_z)."""
    x = np.ascontiguousarray(img, np.float32)
    out = np.zeros_like(x)
    nz, ny, nx = x.shape
    rc = lib().ertm_hilbert_z(x.ctypes.data, out.ctypes.data, nx, ny, nz)
    if rc != 0:
        raise ErtmError(rc, "hilbert_z")
    return out


AXIS_X, AXIS_Y, AXIS_Z = 1, 2, 4


def _arr_ptr(a, n):
    if _is_torch(a):
        return _ptr(a, n)
    if not (isinstance(a, np.ndarray) and a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]):
        raise ValueError("arrays must be C-contiguous float32")
    if a.size != n:
        raise ValueError("array size mismatch")
    return a.ctypes.data


def bell_smooth(img, rbell: int, axes: int = AXIS_X | AXIS_Z, stream_ptr=None):
    """Truncated Gaussian smoothing of an (nz, ny, nx) array (numpy or CUDA tensor)
    along the named axes (see ertm_bell_smooth); returns a new array."""
    nz, ny, nx = img.shape
    n = nx * ny * nz
    if _is_torch(img):
        import torch
        src = img.contiguous()
        out, work = torch.empty_like(src), torch.empty_like(src)
    else:
        src = np.ascontiguousarray(img, np.float32)
        out, work = np.empty_like(src), np.empty_like(src)
    rc = lib().ertm_bell_smooth(_arr_ptr(src, n), _arr_ptr(out, n), _arr_ptr(work, n), nx, ny, nz,
                                rbell, axes, stream_ptr)
    if rc != 0:
        raise ErtmError(rc, "bell_smooth")
    return out


def taper_x(img, left: int, right: int, power: int = 3, stream_ptr=None):
    """Cosine-power edge taper in x, in place (see ertm_taper_x)."""
    nz, ny, nx = img.shape
    rc = lib().ertm_taper_x(_arr_ptr(img, nx * ny * nz), nx, ny, nz, left, right, power, stream_ptr)
    if rc != 0:
        raise ErtmError(rc, "taper_x")
    return img


def aperture_taper(img, x0: int, x1: int, width: int, power: int = 2, stream_ptr=None):
    """Aperture mute in x, in place (see ertm_aperture_taper); -1 leaves a side open."""
    nz, ny, nx = img.shape
    rc = lib().ertm_aperture_taper(_arr_ptr(img, nx * ny * nz), nx, ny, nz, x0, x1, width, power, stream_ptr)
    if rc != 0:
        raise ErtmError(rc, "aperture_taper")
    return img


COMP_PP, COMP_PS, COMP_PP_SIGN, COMP_PS_SIGN = 0, 1, 2, 3


def angle_compensate(img, src_angle, rcv_angle, kind: int = COMP_PP, stream_ptr=None):
    """Angle-dependent compensation of a PP or PS image (see ertm_angle_compensate);
    numpy arrays or CUDA tensors of one shape; returns a new array."""
    n = int(np.prod(img.shape))
    if _is_torch(img):
        import torch
        out = torch.empty_like(img)
    else:
        img = np.ascontiguousarray(img, np.float32)
        src_angle = np.ascontiguousarray(src_angle, np.float32)
        rcv_angle = np.ascontiguousarray(rcv_angle, np.float32)
        out = np.empty_like(img)
    rc = lib().ertm_angle_compensate(_arr_ptr(img, n), _arr_ptr(src_angle, n), _arr_ptr(rcv_angle, n),
                                     _arr_ptr(out, n), n, kind, stream_ptr)
    if rc != 0:
        raise ErtmError(rc, "angle_compensate")
    return out


def adcig_bin(img, angle, nang: int, dangle: float, sx: int, zmin: int = 50, slope: float = 1.2,
              normal=None, cig=None, stream_ptr=None):
    """Add one shot's image to angle-domain common-image gathers
    cig[2*nang+1][nz][nx] (see ertm_adcig_bin); img and angle are (nz, 1, nx) or
    (nz, nx).  Returns cig (allocated when None)."""
    nz, nx = img.shape[0], img.shape[-1]
    n = nx * nz
    if cig is None:
        if _is_torch(img):
            import torch
            cig = torch.zeros((2 * nang + 1, nz, nx), dtype=torch.float32, device=img.device)
        else:
            cig = np.zeros((2 * nang + 1, nz, nx), np.float32)
    if not _is_torch(img):
        img = np.ascontiguousarray(img, np.float32)
        angle = np.ascontiguousarray(angle, np.float32)
        normal = None if normal is None else np.ascontiguousarray(normal, np.float32)
    rc = lib().ertm_adcig_bin(_arr_ptr(img, n), _arr_ptr(angle, n),
                              None if normal is None else _arr_ptr(normal, n),
                              _arr_ptr(cig, (2 * nang + 1) * n), nx, nz, nang, dangle, sx, zmin, slope,
                              stream_ptr)
    if rc != 0:
        raise ErtmError(rc, "adcig_bin")
    return cig
