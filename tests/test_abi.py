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
