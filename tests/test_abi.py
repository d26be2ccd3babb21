"""The C-ABI library loads and exports every entry point of include/ertm.h (no GPU needed)."""
import ctypes as C
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(REPO, "include", "ertm.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ertm_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_header_symbol(ertm):
    L = C.CDLL(ertm.LIB_PATH)
    names = header_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), f"libertm.so does not export {n}"
        assert n in ertm.SIGNATURES, f"no Python signature for {n}"


def test_abi_version(ertm):
    assert ertm.lib().ertm_abi_version() == 1


def test_bad_configs_are_rejected_before_touching_a_device(ertm):
    bad = [dict(nx=0), dict(order=10), dict(boundary=7), dict(dt_ms=0.0), dict(nt=0),
           dict(pml=(30, 30, 0, 0, 0, 0)), dict(coef_kind=1), dict(src_steps=-1)]
    for b in bad:
        kw = dict(nx=40, ny=1, nz=40, dx=5.0, dy=5.0, dz=5.0, dt_ms=0.5, nt=10)
        kw.update(b)
        with pytest.raises(ertm.ErtmError) as ei:
            ertm.Context(ertm.Config(**kw))
        assert ei.value.code in (-1, -5), (b, ei.value)
        assert str(ei.value)


def test_create_without_gpu_fails_cleanly(ertm):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(ertm.ErtmError) as ei:
        ertm.Context(ertm.Config(nx=40, ny=1, nz=40, dx=5, dy=5, dz=5, dt_ms=0.5, nt=10))
    assert ei.value.code == -3 and "CUDA" in str(ei.value)


def test_null_out_pointer(ertm):
    cfg = ertm.Config(nx=40, ny=1, nz=40, dx=5, dy=5, dz=5, dt_ms=0.5, nt=10).struct()
    assert ertm.lib().ertm_create(C.byref(cfg), None) == -1


def test_windows_are_validated_before_touching_a_device(ertm):
    import numpy as np
    base = ertm.Config(nx=40, ny=30, nz=20, dx=10, dy=10, dz=10, dt_ms=0.8, nt=1,
                       pml=(5, 5, 5, 5, 5, 5))
    m = np.ones((20, 30, 40), np.float32)
    w = np.zeros(8, np.float32)
    cases = [
        (ertm.Window(30, 0, 20, 10, 10), ertm.Shot(35, 5, 2, wavelet=w, nrx=1)),   # past x edge
        (ertm.Window(0, 0, 10, 10, 10), ertm.Shot(15, 5, 2, wavelet=w, nrx=1)),    # source outside
        (ertm.Window(0, 0, 10, 10, 0), ertm.Shot(5, 5, 2, wavelet=w, nrx=1)),      # nt = 0
    ]
    for win, sh in cases:
        d = np.zeros((3, win.nt, 1), np.float32)
        with pytest.raises(ertm.ErtmError) as ei:
            ertm.rtm_windows(base, m, m, m, [win], [sh], [d], lanes=1)
        assert ei.value.code == -1 and str(ei.value)
