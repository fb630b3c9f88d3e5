"""The allocation-free full-kernel product (hodlr_kernel_matvec_noalloc).

It serves callers that cannot allocate device memory when they need K x --
an application whose memory manager has already reserved the GPU, a plugin
that must not allocate behind its host framework, latency-bound code that
avoids cudaMalloc's device synchronisation -- by keeping its scratch in a
static device array.  This file is collected last so that a run stopping at
the first failure has already run every other test; it passes on its own in a
fresh process as well as after the rest of the suite.
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


def test_noalloc_matvec_matches_oracle_and_allocates_nothing(oracle_mod):
    """Against the CPU oracle's K x directly, and with the device's free memory
    and torch's allocator unchanged across calls (after a first call, which
    loads the module and with it the static scratch)."""
    import torch

    from dense_hodlr_b200 import KernelSpec
    from dense_hodlr_b200 import _lib
    from dense_hodlr_b200.points import uniform_cube

    lib = _lib.lib()
    n, dim, nrhs = 6000, 3, 2
    pts = uniform_cube(n, dim, 23)
    spec = KernelSpec("gaussian", 0.3, 0.1)
    o = oracle_mod.OracleHODLR.from_kernel(pts, 0, 0.3, shift=0.1, leaf=64)
    pts_d = torch.from_numpy(pts).cuda()
    desc = spec.desc()
    rng = np.random.default_rng(9)
    x = rng.standard_normal((n, nrhs))
    x_d = torch.from_numpy(np.ascontiguousarray(x.T)).cuda()
    y_d = torch.empty_like(x_d)
    assert _run_noalloc(lib, n, dim, pts_d, desc, nrhs, x_d, y_d) == 0  # first call: set-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    ref = o.kernel_matvec(x)
    for call in range(2):
        y_d.fill_(float("nan"))
        assert _run_noalloc(lib, n, dim, pts_d, desc, nrhs, x_d, y_d) == 0, f"call {call}"
        torch.cuda.synchronize()
        got = y_d.cpu().numpy().T
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= TOL, f"call {call}"
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert torch.cuda.memory_allocated() == alloc0


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
