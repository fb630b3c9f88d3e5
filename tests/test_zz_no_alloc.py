"""The allocation-free full-kernel product (hodlr_kernel_matvec_noalloc).

It serves callers that cannot allocate device memory at the point of use --
code running inside a CUDA-graph stream capture, or under a memory manager
that has already reserved the GPU -- by keeping its scratch in a static device
array.  This file is collected last so that a run stopping at the first
failure has already run every other test; it passes on its own in a fresh
process as well as after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-13  # relative difference, as for the handle's product against the oracle


def _run_noalloc(lib, n, dim, pts_d, desc, nrhs, x_d, y_d):
    return lib.hodlr_kernel_matvec_noalloc(n, dim, ctypes.c_void_p(pts_d.data_ptr()),
                                           ctypes.byref(desc), nrhs,
                                           ctypes.c_void_p(x_d.data_ptr()), n,
                                           ctypes.c_void_p(y_d.data_ptr()), n, None)


def test_noalloc_matvec_matches_handle_matvec_twice():
    import torch

    from dense_hodlr_b200 import HODLR_Matrix, KernelSpec
    from dense_hodlr_b200 import _lib
    from dense_hodlr_b200.points import uniform_cube

    lib = _lib.lib()
    n, dim, nrhs = 20000, 2, 3
    pts = uniform_cube(n, dim, 17)
    spec = KernelSpec("matern32", 0.2, 1e-2)
    g = HODLR_Matrix(n, n, spec, pts, 128)  # the existing entry point, through a handle
    pts_d = torch.from_numpy(pts).cuda()
    desc = spec.desc()
    rng = np.random.default_rng(5)
    for call in range(2):  # two calls in a row share the static scratch
        x_d = torch.from_numpy(rng.standard_normal((nrhs, n))).cuda()  # column-major n x nrhs
        y_ref = torch.empty_like(x_d)
        g.kernel_matvec_device(x_d.data_ptr(), y_ref.data_ptr(), nrhs)
        y_d = torch.full_like(x_d, float("nan"))
        assert _run_noalloc(lib, n, dim, pts_d, desc, nrhs, x_d, y_d) == 0, f"call {call}"
        torch.cuda.synchronize()
        ref = y_ref.cpu().numpy()
        got = y_d.cpu().numpy()
        assert np.isfinite(got).all()
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= TOL, f"call {call}"


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    from dense_hodlr_b200 import KernelSpec
    from dense_hodlr_b200 import _lib

    lib = _lib.lib()
    n, nrhs = 262144, 4  # n * nrhs = 1048576 > HODLR_NOALLOC_MAX_ELEMS
    pts_d = torch.zeros((1, n), dtype=torch.float64, device="cuda")
    x_d = torch.zeros((nrhs, n), dtype=torch.float64, device="cuda")
    y_d = torch.zeros_like(x_d)
    desc = KernelSpec("gaussian", 0.1, 1.0).desc()
    assert _run_noalloc(lib, n, 1, pts_d, desc, nrhs, x_d, y_d) == 1  # HODLR_ERR_ARG
