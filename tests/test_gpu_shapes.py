"""GPU parity at reduced size for the configurations measured at 2^20 points,
and for the minPivot skip-row path of ACA.

* The sphere / Matern-3/2 shape (unit sphere, l = 0.1, shift 1e-2, leaf 128,
  ACA tol 1e-10): its ranks make the top capacitance matrices large enough
  for the multi-CTA blocked LU (sd >= SCHUR_BIG_SD = 384).
* The cube / Gaussian shape (l = 0.3, shift 0.1, leaf 128, tol 1e-8) with 16
  right-hand sides, through HODLR-preconditioned GMRES with FP64, 3xTF32 and
  TF32 Woodbury products.
* minPivot >= 1 (src/lowRank.cpp:187-195 skip path, :197-203 and :217-227
  fallbacks): dense 10 * Gaussian + I with minPivot 2.5 (truncated to 2, as
  the reference passes it to an int).

Bit-exact: pivots, ranks, iteration counts and the W/V factors of the
largest blocks.  Solutions within 1e-10 of the oracle's.
"""
import numpy as np
import pytest

from dense_hodlr_b200 import HODLR_Matrix, KernelSpec
from dense_hodlr_b200.points import uniform_cube, unit_sphere

from .test_gpu_parity import SOLVE_TOL, _compare_compression, _pair

pytestmark = pytest.mark.gpu

BIG_SD = 384  # SCHUR_BIG_SD in csrc/lu.h


def _device_gmres(g, b, tol=1e-10, max_iter=60):
    import torch
    b_d = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
    x_d = torch.empty_like(b_d)
    it, rel = g.iterative_solve_device(b_d.data_ptr(), x_d.data_ptr(), b.shape[1], tol=tol,
                                       max_iter=max_iter, restart=32)
    return it, rel, x_d.cpu().numpy().T


def test_sphere_matern_tol_1e10_bit_exact_and_large_capacitance(oracle_mod):
    n = 16384
    pts = unit_sphere(n, 31)
    g, o = _pair(oracle_mod, pts, "matern32", 0.1, 1e-2, 128, 1e-10)
    _compare_compression(g, o, check_factors=False)
    assert np.array_equal([g.block_info(b)["iters"] for b in range(g.num_blocks())], o.iters())
    for b in (0, 1, 2, 3):
        info = g.block_info(b)
        W, V = g.lowrank(b)
        Wo, Vo = o.lowrank(b, info["m"], info["n"])
        assert np.array_equal(W, Wo) and np.array_equal(V, Vo), b
    r = g.ranks()
    assert r[0] + r[1] >= BIG_SD  # the root's capacitance LU takes the multi-CTA path
    b = np.random.default_rng(6).standard_normal((n, 2))
    x = g.recLU_Solve(b)
    xo = o.solve(b, nthreads=8)
    # This system is ill-conditioned (|x| ~ 1e4 |b|, capacitance matrices of
    # 2000+ rows): two FP64 factorizations of the same compressed matrix in
    # different summation orders agree to ~1e-8 here (measured 9.9e-9), not
    # to 1e-10.  So the direct solutions are held to that, and the GPU's to
    # the oracle's own accuracy: its FP64 residual no worse than the oracle's.
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-7
    assert g.residual(x, b).max() <= 1.5 * g.residual(xo, b).max() + 1e-14
    it, rel, xg = _device_gmres(g, b)
    assert rel.max() <= 1e-10
    assert np.all(g.residual(xg, b) <= 1e-10)


@pytest.mark.parametrize("n,leaf", [(256, 32), (4096, 64)])
def test_min_pivot_skip_rows_bit_exact(oracle_mod, n, leaf):
    rng = np.random.default_rng(22)
    x = np.sort(rng.uniform(-1.0, 1.0, n))
    A = 10.0 * np.exp(-((x[:, None] - x[None, :]) / 0.1) ** 2) + np.eye(n)
    g = HODLR_Matrix(A, leaf)
    g.set_LRTolerance(1e-10)
    g.set_minPivot(2.5)
    o = oracle_mod.OracleHODLR.from_dense(A, leaf=leaf)
    o.set_lr(1e-10, 2.5)
    _compare_compression(g, o)
    giters = np.array([g.block_info(b)["iters"] for b in range(g.num_blocks())])
    assert np.array_equal(giters, o.iters())
    assert (o.iters() > np.minimum(o.ranks(), o.iters())).any()  # rows were skipped
    bvec = np.random.default_rng(3).standard_normal((n, 2))
    xs, xo = g.recLU_Solve(bvec), o.solve(bvec)
    assert np.linalg.norm(xs - xo) / np.linalg.norm(xo) <= SOLVE_TOL


def test_cube_gaussian_16_rhs_gmres_fp64_and_tf32_forms(oracle_mod):
    n, nrhs = 16384, 16
    pts = uniform_cube(n, 3, 5)
    g, o = _pair(oracle_mod, pts, "gaussian", 0.3, 1e-1, 128, 1e-8)
    g.storeLRinTree()
    o.compress()
    assert np.array_equal(g.ranks(), o.ranks())
    b = np.random.default_rng(12).standard_normal((n, nrhs))
    xo = o.solve(b, nthreads=8)
    x64 = g.recLU_Solve(b)
    assert np.linalg.norm(x64 - xo) / np.linalg.norm(xo) <= SOLVE_TOL
    # BF16 is left out: a factor preconditions only while cond(K) * u < ~1, and
    # here cond(K) ~ 2.5e4 against u = 3.9e-3 (it stalls near 1, as measured)
    for prec in ("fp64", "tf32x3", "tf32"):
        g.set_precision(prec)
        g.recLU_Compute()
        it, rel, x = _device_gmres(g, b)
        assert rel.max() <= 1e-10, (prec, it, rel.max())
        assert np.all(g.residual(x, b) <= 1e-10), prec


def test_factor_in_place_matches_separate_panels(oracle_mod):
    """K^-1 U written over the U panels (hodlr_set_factor_in_place(1)) gives the
    solution of the separate-panel factorization; the overwritten W is
    refused afterwards, and another precision compresses again."""
    n = 8192
    pts = uniform_cube(n, 2, 19)
    g, o = _pair(oracle_mod, pts, "matern32", 0.2, 1e-2, 64, 1e-8)
    b = np.random.default_rng(2).standard_normal((n, 3))
    g.set_factor_in_place(0)
    x0 = g.recLU_Solve(b)
    assert g.factor_in_place_levels() == 0
    W0, V0 = g.lowrank(0)
    g.set_factor_in_place(1)
    x1 = g.recLU_Solve(b)
    assert g.factor_in_place_levels() == g.num_levels()
    assert np.linalg.norm(x1 - x0) / np.linalg.norm(x0) <= 1e-13
    xo = o.solve(b, nthreads=8)
    assert np.linalg.norm(x1 - xo) / np.linalg.norm(xo) <= SOLVE_TOL
    from dense_hodlr_b200 import HODLRError
    with pytest.raises(HODLRError):
        g.lowrank(0)
    g.set_precision("tf32x3")  # refactor: the U panels are compressed again
    it, rel, _ = _device_gmres(g, b)
    assert rel.max() <= 1e-10
    g.set_precision("fp64")
    g.set_factor_in_place(0)
    g.recLU_Compute()
    W2, V2 = g.lowrank(0)
    assert np.array_equal(W0, W2) and np.array_equal(V0, V2)


@pytest.mark.parametrize("n,dim", [(32768, 2), (20000, 3)])
def test_ring_streaming_bit_identical_to_per_thread_loads(n, dim):
    """The top-level ACA with its panel slices streamed through the bulk-copy
    ring, one copy per column (hodlr_set_aca_streaming(1)) or one 2D tensor
    copy per tile (2), against per-thread loads: the same pivots, ranks,
    iteration counts and W/V bits on every block."""
    pts = uniform_cube(n, dim, 13)
    out = []
    for on in (0, 1, 2):
        g = HODLR_Matrix(n, n, KernelSpec("matern32", 0.2, 1e-2), pts, 128)
        g.set_LRTolerance(1e-8)
        g.set_aca_streaming(on)
        g.storeLRinTree()
        nb = g.num_blocks()
        out.append((g.ranks(), [g.block_info(b)["iters"] for b in range(nb)],
                    [g.pivots(b) for b in range(nb)], [g.lowrank(b) for b in range(8)]))
    r0, i0, p0, f0 = out[0]
    for r1, i1, p1, f1 in out[1:]:
        assert np.array_equal(r0, r1) and i0 == i1
        for a, b in zip(p0, p1):
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        for (W0, V0), (W1, V1) in zip(f0, f1):
            assert np.array_equal(W0, W1) and np.array_equal(V0, V1)


def test_checked_mode_gives_the_same_solution():
    """hodlr_set_checked(1): every GEMM operand extent verified, the solve
    without its graph and a sync after every launch group -- the same bits as
    the unchecked path for the direct solve and the GMRES iterate."""
    n = 12000
    pts = uniform_cube(n, 2, 41)
    spec = KernelSpec("matern32", 0.2, 1e-2)
    b = np.random.default_rng(8).standard_normal((n, 3))
    out = []
    for checked in (False, True):
        g = HODLR_Matrix(n, n, spec, pts, 128)
        g.set_LRTolerance(1e-8)
        g.set_checked(checked)
        x = g.recLU_Solve(b)
        it, rel, xg = _device_gmres(g, b)
        out.append((x, it, xg))
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1] and np.array_equal(out[0][2], out[1][2])
