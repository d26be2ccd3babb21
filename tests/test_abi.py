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


def test_header_is_c99_and_a_c_program_links_and_calls_the_library(tmp_path):
    """The header compiles as strict C99, and a C program linked against libertm.so
    calls host entry points through the C ABI (no Python, no GPU)."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    lib = os.path.join(REPO, "2d_and_3d_elastic_reverse_time_migration_b200", "_lib")
    src = tmp_path / "drv.c"
    src.write_text(r'''
#include <stdio.h>
#include "ertm.h"
int main(void)
{
    float img[5 * 4], vp[5 * 4], h[5 * 4];
    for (int i = 0; i < 20; i++) { img[i] = (float)((i * 7) % 5) - 2.0f; vp[i] = 2000.0f; }
    if (ertm_abi_version() != ERTM_ABI_VERSION) return 1;
    if (ertm_hilbert_z(img, h, 5, 1, 4) != ERTM_OK) return 2;
    if (ertm_laplace_filter(img, vp, 5, 1, 4, 5.0f, 5.0f, 5.0f) != ERTM_OK) return 3;
    if (ertm_laplace_filter(img, vp, 2, 1, 4, 5.0f, 5.0f, 5.0f) != ERTM_EINVAL) return 4;
    if (ertm_taper_x(img, 5, 1, 4, 2, 2, 3, NULL) != ERTM_OK) return 5;
    printf("ok %g %g\n", img[7], h[3]);
    return 0;
}
''')
    exe = tmp_path / "drv"
    subprocess.run([gcc, "-std=c99", "-Wall", "-Werror", "-pedantic", "-I", os.path.join(REPO, "include"),
                    str(src), "-o", str(exe), "-L", lib, "-lertm", "-Wl,-rpath," + lib], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.startswith("ok"), (out.returncode, out.stdout, out.stderr)


def test_integration_shim_compiles_against_the_header(tmp_path):
    """The reference-side C shim (what a maintainer adds to the reference's driver)
    compiles against include/ertm.h, given declarations of the reference globals it
    reads (3D_elastic_modeling_parameter)."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    shim = os.path.join(REPO, "2d_and_3d_elastic_reverse_time_migration_b200", "reference_shim",
                        "ertm_reference_shim.c")
    code = open(shim).read()
    globals_ = """
typedef struct GPUdevice GPUdevice;
extern int nnx, nny, nnz, lt, bl, br, bf, bb, bu, bd, wavelet_length;
extern int gpuid[8], sx_real, sy_real, sz_real, add_receiver_bool;
extern int receiver_start_x, receiver_num_x, receiver_interval_x;
extern int receiver_start_y, receiver_num_y, receiver_interval_y, receiver_start_z;
extern float dx, dy, dz, dt, coe_att;
extern float *velocity_pml, *velocity1_pml, *density_pml, *s_velocity_pml, *s_velocity1_pml, *s_density_pml;
extern float *wavelet, *obs_shot_all, *vresult_pp_h, *vresult_ps_h, *vresult_tp_h;
void err(const char *fmt, ...);
"""
    src = tmp_path / "shim.c"
    body = code.replace('#include "ertm.h"', '#include "ertm.h"\n' + globals_, 1)
    src.write_text(body)
    subprocess.run([gcc, "-std=c99", "-Wall", "-Werror", "-Wno-unused-function", "-I",
                    os.path.join(REPO, "include"), "-c", str(src), "-o", str(tmp_path / "shim.o")], check=True)


def test_nn_entry_points_validate_before_touching_a_device(ertm):
    """The tensor-core entry points refuse, before any launch, operands that their
    16-byte copies or their epilogues cannot take: a weight pointer off a 16-byte
    boundary, an input gradient of another grid than the output gradient, a ReLU
    mask that is not laid out like the gradient it masks (host memory, no GPU)."""
    import numpy as np
    L = ertm.lib()
    buf = np.zeros(1 << 14, np.uint16)
    p = buf.ctypes.data + (-buf.ctypes.data % 16)

    def act(n, h, w, c, cs=None, off=0):
        a = ertm._NnAct()
        a.data, a.n, a.h, a.w = p, n, h, w
        a.cstride, a.coff, a.c = cs or c, off, c
        return a

    x, y = act(1, 4, 8, 16), act(1, 4, 8, 16)
    assert L.ertm_nn_conv3x3(C.byref(x), p + 2, None, C.byref(y), 1, None, None, None) == -1
    assert L.ertm_nn_gemm(p + 8, p, p, 16, 16, 16, None, None) == -1
    assert L.ertm_nn_conv3x3_dgrad(C.byref(x), p, C.byref(act(1, 4, 4, 16)), None, None, None) == -1
    dx, mask = act(1, 4, 8, 16, cs=32), act(1, 4, 8, 16, cs=32, off=16)
    assert L.ertm_nn_conv3x3_dgrad(C.byref(x), p, C.byref(dx), C.byref(mask), None, None) == -1
