"""The tcgen05 tensor-core GEMMs of the mixed-precision form, against FP64.

Tolerances: products of BF16 operands (8-bit significand) with FP32
accumulation agree with FP64 to a relative Frobenius error of a few 1e-3;
TF32 operands (11-bit significand) to a few 1e-4.  The FP64 kernel of the
same entry point agrees to 1e-13.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# FP64, TF32, BF16, 3xTF32 (FP32 accumulation in tensor memory: ~1e-7 * sqrt(K))
TOL = {0: 1e-13, 1: 2e-3, 2: 1.5e-2, 3: 2e-5}


def _gemm(prec, mode, A, B, C):
    import torch
    from dense_hodlr_b200 import _lib
    lib = _lib.lib()
    dA = torch.from_numpy(np.asfortranarray(A).T.copy()).cuda()  # column-major storage
    dB = torch.from_numpy(np.asfortranarray(B).T.copy()).cuda()
    dC = torch.from_numpy(np.asfortranarray(C).T.copy()).cuda()
    if mode == 0:
        k, m = A.shape
    else:
        m, k = A.shape
    n = B.shape[1]
    rc = lib.hodlr_gemm_device(prec, mode, m, n, k, ctypes.c_void_p(dA.data_ptr()), A.shape[0],
                               ctypes.c_void_p(dB.data_ptr()), B.shape[0],
                               ctypes.c_void_p(dC.data_ptr()), C.shape[0], None)
    assert rc == 0
    torch.cuda.synchronize()
    return dC.cpu().numpy().T


@pytest.mark.parametrize("prec", [0, 1, 2, 3])
@pytest.mark.parametrize("m,n,k", [(100, 70, 300), (470, 8, 131072), (128, 64, 64), (3, 5, 7)])
def test_tn_products(prec, m, n, k):
    rng = np.random.default_rng(m + n + k)
    A = rng.standard_normal((k, m))
    B = rng.standard_normal((k, n))
    ref = A.T @ B
    got = _gemm(prec, 0, A, B, np.zeros((m, n)))
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < TOL[prec]


@pytest.mark.parametrize("prec", [0, 1, 2, 3])
@pytest.mark.parametrize("m,n,k", [(1000, 300, 80), (129, 65, 1), (64, 1500, 40)])
def test_nn_subtract(prec, m, n, k):
    rng = np.random.default_rng(m * 7 + k)
    A = rng.standard_normal((m, k))
    B = rng.standard_normal((k, n))
    C = rng.standard_normal((m, n))
    ref = C - A @ B
    got = _gemm(prec, 1, A, B, C.copy())
    assert np.linalg.norm(got - ref) / np.linalg.norm(A @ B) < TOL[prec]


@pytest.mark.parametrize("precision,shift", [("tf32x3", 1e-2), ("tf32", 1.0), ("bf16", 1.0)])
def test_mixed_precision_solve_reaches_target(precision, shift):
    """Mixed-precision factor (tensor-core Woodbury products) as the GMRES
    preconditioner: full accuracy is recovered with the FP64 residual.  TF32
    and BF16 need cond(K) * u < 1 (shift 1.0 here); 3xTF32 also handles the
    ill-conditioned shift-1e-2 system of the FP64-at-scale workload."""
    from dense_hodlr_b200 import HODLR_Matrix, KernelSpec
    from dense_hodlr_b200.points import uniform_cube
    n = 16384
    pts = uniform_cube(n, 2, 41)
    g = HODLR_Matrix(n, n, KernelSpec("matern32", 0.2, shift), pts, 128)
    g.set_LRTolerance(1e-8)
    g.set_precision(precision)
    b = np.random.default_rng(2).standard_normal((n, 4))
    x = g.iterative_Solve(b, 300, 1e-10)
    assert g.last_relres.max() <= 1e-10
    assert g.residual(x, b).max() <= 1.5e-10
    # the direct mixed solve is a usable approximation on its own
    g.set_precision("fp64")
    x64 = g.recLU_Solve(b)
    g.set_precision(precision)
    xm = g.recLU_Solve(b)
    tol = {"bf16": 0.05, "tf32": 0.01, "tf32x3": 1e-3}[precision]
    assert np.linalg.norm(xm - x64) / np.linalg.norm(x64) < tol
