"""recSM_Solve on the GPU (hodlr_set_solver_form(HODLR_FORM_RECSM)): the
recursive Sherman-Morrison factorization, whose nodes are perturbed
identities I + U V^T with the top block's rank first in every capacitance
system (src/HODLR_Matrix.cpp:520-610,805-841; src/perturbI.cpp:15-83),
against the oracle's restatement of that recursion.

Shapes: the reference's own recSM tests (test/test.cpp:76-89 exact rank-10
HODLR N=10000 leaf 50; test/test.cpp:132-147 dense 1D inverse multiquadric
N=10000 leaf 30 tol 1e-8), a 2D Matern-3/2 kernel at 32768 points whose
capacitance systems take the blocked solves, and the log-determinant
(test/test.cpp:578-590).
"""
import numpy as np
import pytest

from dense_hodlr_b200 import HODLR_Matrix, KernelSpec
from dense_hodlr_b200.points import uniform_cube

from .test_gpu_parity import SOLVE_TOL, _pair
from .test_oracle import exact_hodlr

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_recsm_exact_random_hodlr(oracle_mod):
    n = 10000
    A = exact_hodlr(n, 50, 10, seed=0)
    g = HODLR_Matrix(A, 50)
    o = oracle_mod.OracleHODLR.from_dense(A, leaf=50)
    xe = np.linspace(-2, 2, n)[:, None]
    b = A @ xe
    x = g.recSM_Solve(b)
    assert g.get_solver_form() == "recSM"
    xo = o.recsm_solve(b)
    # the random leaves' conditioning sets the agreement here, not the
    # compression (see test_reference_recsm_random_exact_hodlr): measured
    # 1.8e-8 between two FP64 recSM factorizations in different orders
    assert _rel(x, xo) <= 5e-8 and _rel(x, xe) < 5e-8
    assert np.linalg.norm(A @ x - b) / np.linalg.norm(b) <= 2.0 * np.linalg.norm(A @ xo - b) / np.linalg.norm(b) + 1e-14


def test_recsm_inverse_multiquadric(oracle_mod):
    n = 10000
    x = np.linspace(-1.0, 1.0, n)
    r = np.abs(x[:, None] - x[None, :])
    A = 1.0 / np.sqrt(1.0 + r * r)
    np.fill_diagonal(A, 0.0)
    g = HODLR_Matrix(A, 30)
    g.set_LRTolerance(1e-8)
    o = oracle_mod.OracleHODLR.from_dense(A, leaf=30)
    o.set_lr(1e-8)
    xe = np.linspace(-2, 2, n)[:, None]
    b = A @ xe
    xs = g.recSM_Solve(b)
    assert _rel(xs, xe) < 1e-6
    assert _rel(xs, o.recsm_solve(b)) <= 1e-8


def test_recsm_kernel_blocked_capacitance_and_switching(oracle_mod):
    """32768 points: capacitance systems of 128+ rows (blocked solves); recSM
    against the oracle's recSM, then back to recLU with the same bits as a
    handle that never left it, and the recSM log-determinant against the
    oracle's."""
    n = 32768
    pts = uniform_cube(n, 2, 29)
    g, o = _pair(oracle_mod, pts, "matern32", 0.2, 1e-2, 128, 1e-8)
    b = np.random.default_rng(4).standard_normal((n, 2))
    xs = g.recSM_Solve(b)
    xo = o.recsm_solve(b)
    assert _rel(xs, xo) <= SOLVE_TOL
    sg, ld = g.slogdet()
    so, lo = o.recsm_slogdet()
    assert sg == so and abs(ld - lo) <= 1e-10 * abs(lo)
    xl = g.recLU_Solve(b)
    assert g.get_solver_form() == "recLU"
    ref = HODLR_Matrix(n, n, KernelSpec("matern32", 0.2, 1e-2), pts, 128)
    ref.set_LRTolerance(1e-8)
    assert np.array_equal(xl, ref.recLU_Solve(b))
    assert _rel(xl, xs) <= SOLVE_TOL
