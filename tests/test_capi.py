"""CPU checks of the C ABI library: it loads, exports every symbol declared
in include/hodlr_b200.h, validates arguments, and refuses to run without a
GPU (there is no CPU fallback)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include")))
           if f.endswith(".h")]


def declared_symbols():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[a-z_]+\s*\*?\s*(hodlr_[a-z0-9_]+)\s*\(", text, re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("hodlr_create_kernel", "hodlr_create_dense", "hodlr_compress",
                 "hodlr_factorize", "hodlr_solve", "hodlr_destroy"):
        assert must in names


def test_library_exports_every_declared_symbol(gpu_lib):
    raw = ctypes.CDLL(os.path.join(ROOT, "dense_hodlr_b200", "libhodlr_b200.so"))
    missing = [n for n in sorted(declared_symbols()) if not hasattr(raw, n)]
    assert not missing, missing


def test_python_signatures_cover_header(gpu_lib):
    from dense_hodlr_b200._lib import SIGNATURES
    assert declared_symbols() <= set(SIGNATURES)


def test_argument_validation(gpu_lib):
    h = ctypes.c_void_p()
    pts = np.zeros(10)
    dp = pts.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    from dense_hodlr_b200._lib import KernelDesc
    d = KernelDesc(0, 0.1, 1.0, 0, 0.0)
    assert gpu_lib.hodlr_create_kernel(ctypes.byref(h), 0, 1, dp, ctypes.byref(d), 30) == 1
    assert gpu_lib.hodlr_create_kernel(ctypes.byref(h), 10, 4, dp, ctypes.byref(d), 30) == 1
    bad = KernelDesc(0, -1.0, 1.0, 0, 0.0)
    assert gpu_lib.hodlr_create_kernel(ctypes.byref(h), 10, 1, dp, ctypes.byref(bad), 30) == 1
    assert gpu_lib.hodlr_create_dense(ctypes.byref(h), 10, dp, 5, 30) == 1
    assert gpu_lib.hodlr_create_fnptr(ctypes.byref(h), 10, 10, None, None, 30) == 4
    assert gpu_lib.hodlr_set_lr_tolerance(None, 1e-6) == 1
    assert gpu_lib.hodlr_status_string(4) == b"unsupported on the GPU path"


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU behaviour")
def test_no_cpu_fallback_without_gpu(gpu_lib):
    from dense_hodlr_b200 import HODLR_Matrix, HODLRError, KernelSpec
    with pytest.raises(HODLRError) as e:
        HODLR_Matrix(64, 64, KernelSpec("gaussian", 0.1, 1.0), np.linspace(0, 1, 64)[None, :], 16)
    assert e.value.status == 2  # HODLR_ERR_CUDA


def test_device_functor_facade_compiles(gpu_lib, tmp_path):
    """The device-functor constructor of include/HODLR_Matrix.hpp and its test
    program build with nvcc for sm_100a (run by the GPU suite)."""
    import subprocess
    exe = tmp_path / "functor_test"
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O1", "-std=c++17",
                    os.path.join(ROOT, "tests", "cpp", "functor_test.cu"),
                    "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "dense_hodlr_b200", "csrc"),
                    "-L", os.path.join(ROOT, "dense_hodlr_b200"), "-lhodlr_b200",
                    "-o", str(exe)], check=True, timeout=600)
    assert exe.exists()
