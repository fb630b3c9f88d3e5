"""Parity of the CUDA path (through the C ABI) against the CPU oracle.

Bit-exact: tree, ACA pivot sequences, ranks and the W/V factors (integer and
pivot-deciding FP64 work).  Tolerance: solutions within 1e-10 relative
difference of the oracle (the parity bar of the FP64 path), residuals
with the full kernel.  Blocks whose stopping test came within 1e-10 of the
tolerance (a "near tie", where reduction order may decide the rank) are
reported and excluded from the bit-exact rank comparison; the tests assert
there are none on these inputs.
"""
import numpy as np
import pytest

from dense_hodlr_b200 import HODLR_Matrix, HODLRError, KernelSpec, kernelMatrix
from dense_hodlr_b200.points import uniform_cube

from .conftest import c1_points

pytestmark = pytest.mark.gpu

SOLVE_TOL = 1e-10  # relative difference vs the oracle, FP64 path


def _pair(oracle_mod, pts, kind, l, shift, leaf, tol, diag_replace=False, diag_value=0.0):
    g = HODLR_Matrix(pts.shape[1], pts.shape[1],
                     KernelSpec(kind, l, shift, diag_replace, diag_value), pts, leaf)
    g.set_LRTolerance(tol)
    ktype = g_kind(kind)
    o = oracle_mod.OracleHODLR.from_kernel(pts, ktype, l, shift=shift, leaf=leaf,
                                           diag_replace=diag_replace, diag_value=diag_value)
    o.set_lr(tol)
    return g, o


def g_kind(kind):
    from dense_hodlr_b200.hodlr import _KERNEL_NAMES
    return _KERNEL_NAMES[kind] if isinstance(kind, str) else kind


def _compare_compression(g, o, check_factors=True):
    g.storeLRinTree()
    o.compress()
    nb = g.num_blocks()
    assert nb == o.num_blocks()
    gr, orr = g.ranks(), o.ranks()
    om = o.margins()
    near = [b for b in range(nb) if g.margin(b)[1] > 0 or om[b] < 1e-10]
    assert not near, f"near-tie blocks: {near}"
    assert np.array_equal(gr, orr), np.nonzero(gr != orr)
    inner = o.inner_nodes()
    for b in range(nb):
        info = g.block_info(b)
        lvl, mn, sp, mx = inner[b // 2]
        assert info["level"] == lvl
        if b % 2 == 0:
            assert (info["row0"], info["col0"], info["m"], info["n"]) == (mn, sp + 1, sp - mn + 1, mx - sp)
        else:
            assert (info["row0"], info["col0"], info["m"], info["n"]) == (sp + 1, mn, mx - sp, sp - mn + 1)
        gp = g.pivots(b)
        op = o.pivots(b)
        assert np.array_equal(gp[0], op[0]) and np.array_equal(gp[1], op[1]), f"block {b}"
        if check_factors:
            W, V = g.lowrank(b)
            Wo, Vo = o.lowrank(b, info["m"], info["n"])
            assert np.array_equal(W, Wo), f"W of block {b}"
            assert np.array_equal(V, Vo), f"V of block {b}"


def test_c1_gaussian_1d_bit_exact(oracle_mod):
    """N=4096 sorted uniform [-1,1], exp(-(dx)^2/0.1^2) + 1.0 delta, leaf 64, tol 1e-10."""
    pts, rng = c1_points()
    g, o = _pair(oracle_mod, pts, "gaussian", 0.1, 1.0, 64, 1e-10)
    _compare_compression(g, o)
    b = rng.standard_normal((4096, 1))
    x = g.recLU_Solve(b)
    xo = o.solve(b)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= SOLVE_TOL
    # dense FP64 LU oracle of the same K
    K = np.exp(-((pts[0][:, None] - pts[0][None, :]) ** 2) / 0.01) + np.eye(4096)
    xd = np.linalg.solve(K, b)
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-9
    rel = g.residual(x, b)
    assert rel.max() < 1e-9


def test_uneven_2d_matern(oracle_mod):
    """Uneven sizes exercise the left/right split asymmetry of createDefaultTree."""
    pts = uniform_cube(3001, 2, 11)
    g, o = _pair(oracle_mod, pts, "matern32", 0.2, 1e-2, 64, 1e-8)
    _compare_compression(g, o)
    b = np.random.default_rng(3).standard_normal((3001, 3))
    x = g.recLU_Solve(b)
    xo = o.solve(b)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= SOLVE_TOL


@pytest.mark.parametrize("kind,dim,n,l,shift,replace,value", [
    ("exponential", 2, 6000, 0.3, 0.5, False, 0.0),
    ("inv_multiquadric", 3, 5000, 0.5, 0.0, True, 2.0),
    ("quadratic", 1, 4000, 1.0, 0.0, True, 0.0),  # the reference's kernel test shape: K_ii = 0
])
def test_other_kernel_families_bit_exact(oracle_mod, kind, dim, n, l, shift, replace, value):
    """The remaining closed-form kernels through ACA and the solve: pivots,
    ranks and W/V bit for bit against the oracle, solutions within 1e-10."""
    pts = uniform_cube(n, dim, 40 + dim)
    g, o = _pair(oracle_mod, pts, kind, l, shift, 64, 1e-8, replace, value)
    _compare_compression(g, o)
    b = np.random.default_rng(n).standard_normal((n, 2))
    x = g.recLU_Solve(b)
    xo = o.solve(b)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= SOLVE_TOL


def test_3d_gaussian_group_levels(oracle_mod):
    """3D Gaussian, leaf 128: top levels run with many CTAs per block."""
    pts = uniform_cube(16384, 3, 5)
    g, o = _pair(oracle_mod, pts, "gaussian", 0.3, 1e-1, 128, 1e-8)
    _compare_compression(g, o, check_factors=False)
    for b in (0, 1, 2, 5):  # the largest blocks, W/V bit for bit
        info = g.block_info(b)
        W, V = g.lowrank(b)
        Wo, Vo = o.lowrank(b, info["m"], info["n"])
        assert np.array_equal(W, Wo) and np.array_equal(V, Vo)
    b = np.random.default_rng(4).standard_normal((16384, 4))
    x = g.recLU_Solve(b)
    xo = o.solve(b)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= SOLVE_TOL


def test_kernel_matvec_matches_oracle(oracle_mod):
    pts = uniform_cube(5000, 3, 9)
    g, o = _pair(oracle_mod, pts, "matern32", 0.1, 1e-2, 64, 1e-8)
    x = np.random.default_rng(2).standard_normal((5000, 3))
    import torch
    xd = torch.from_numpy(np.asfortranarray(x).T.copy()).cuda()  # column-major = rows of x.T
    yd = torch.empty_like(xd)
    g.kernel_matvec_device(xd.data_ptr(), yd.data_ptr(), 3)
    torch.cuda.synchronize()
    y = yd.cpu().numpy().T
    yo = o.kernel_matvec(x)
    assert np.linalg.norm(y - yo) / np.linalg.norm(yo) < 1e-13


@pytest.mark.parametrize("n,dim,kind,nrhs,diag_replace", [
    (777, 1, "gaussian", 1, False),      # one split, ragged last tile
    (24832, 2, "matern32", 8, False),    # 97 tiles: two per split, ragged last split
    (30001, 2, "exponential", 5, True),  # ragged tile and split, replaced diagonal
    (9000, 3, "inv_multiquadric", 4, False),
    (4097, 3, "gaussian", 8, False),     # tensor-core form, 3D, one row past a tile
    (1300, 1, "matern32", 6, False),     # tensor-core form, 1D, 6 of 8 columns live
    (100, 2, "matern32", 8, False),      # tensor-core form, one partial tile (diagonal pair only)
])
def test_symmetric_kernel_matvec(oracle_mod, n, dim, kind, nrhs, diag_replace):
    """The symmetric full-kernel product (each entry evaluated once for both
    K_ij x_j and K_ji x_i) against the oracle's row-by-row product, per column
    relative error 1e-13, and bit-identical on a repeated call."""
    import torch
    pts = uniform_cube(n, dim, 31 + n)
    g, o = _pair(oracle_mod, pts, kind, 0.15, 0.5, 64, 1e-8, diag_replace, 2.0)
    x = np.random.default_rng(n).standard_normal((n, nrhs))
    xd = torch.from_numpy(np.asfortranarray(x).T.copy()).cuda()
    yd = torch.empty_like(xd)
    g.kernel_matvec_device(xd.data_ptr(), yd.data_ptr(), nrhs)
    torch.cuda.synchronize()
    y = yd.cpu().numpy().T.copy()
    yo = o.kernel_matvec(x)
    err = np.linalg.norm(y - yo, axis=0) / np.linalg.norm(yo, axis=0)
    assert err.max() < 1e-13, err
    g.kernel_matvec_device(xd.data_ptr(), yd.data_ptr(), nrhs)
    torch.cuda.synchronize()
    assert np.array_equal(yd.cpu().numpy().T, y)


def test_dense_input_inverse_multiquadric(oracle_mod):
    """Reference test shape (test/test.cpp:112-129): dense 1D inverse multiquadric,
    diagonal replaced by 0, leaf 30, tol 1e-8, solution error < 1e-6."""
    n = 2000
    x = np.linspace(-1.0, 1.0, n)
    r = np.abs(x[:, None] - x[None, :])
    A = 1.0 / np.sqrt(1.0 + r * r)
    np.fill_diagonal(A, 0.0)
    g = HODLR_Matrix(A, 30)
    g.set_LRTolerance(1e-8)
    o = oracle_mod.OracleHODLR.from_dense(A, leaf=30)
    o.set_lr(1e-8)
    _compare_compression(g, o)
    xe = np.linspace(-2, 2, n)[:, None]
    b = A @ xe
    xs = g.recLU_Solve(b)
    assert np.linalg.norm(xs - xe) / np.linalg.norm(xe) < 1e-6
    xo = o.solve(b)
    assert np.linalg.norm(xs - xo) / np.linalg.norm(xo) <= SOLVE_TOL


def test_dense_input_from_matrix_file(oracle_mod, tmp_path):
    """Dense input through the reference's binary matrix file
    (saveMatrixXdToBinary / readBinaryIntoMatrixXd, src/matrixIO.cpp:159-202):
    a Gaussian 1D matrix written to a file, read back by the C ABI, compressed
    and solved on the GPU, against the oracle on the same entries, bit for bit
    in pivots and ranks, so no kernel-function rounding enters the parity."""
    import ctypes
    from dense_hodlr_b200 import _lib
    from dense_hodlr_b200.matrix_io import saveMatrixXdToBinary
    n = 3000
    x = np.sort(np.random.default_rng(8).uniform(-1.0, 1.0, n))
    A = np.exp(-((x[:, None] - x[None, :]) / 0.1) ** 2) + np.eye(n)
    path = tmp_path / "k.bin"
    saveMatrixXdToBinary(A, path)
    F = np.zeros((n, n), order="F")
    lib = _lib.lib()
    assert lib.hodlr_read_matrix_file(str(path).encode(), n, n,
                                      F.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n) == 0
    assert np.array_equal(F, A)
    g = HODLR_Matrix(F, 64)
    g.set_LRTolerance(1e-10)
    o = oracle_mod.OracleHODLR.from_dense(A, leaf=64)
    o.set_lr(1e-10)
    _compare_compression(g, o)
    b = np.random.default_rng(9).standard_normal((n, 2))
    xs, xo = g.recLU_Solve(b), o.solve(b)
    assert np.linalg.norm(xs - xo) / np.linalg.norm(xo) <= SOLVE_TOL


def test_reference_random_exact_hodlr():
    """Reference test shape (test/test.cpp:57-69): exact rank-10 HODLR, N=10000,
    leaf 50, relative error < 1e-8 on x = LinSpaced(-2, 2)."""
    from tests.test_oracle import exact_hodlr
    n = 10000
    A = exact_hodlr(n, 50, 10, seed=0)
    g = HODLR_Matrix(A, 50)
    xe = np.linspace(-2, 2, n)[:, None]
    b = A @ xe
    xs = g.recLU_Solve(b)
    assert np.linalg.norm(xs - xe) / np.linalg.norm(xe) < 1e-8


def test_tolerance_change_recompresses(oracle_mod):
    pts, rng = c1_points(2048, 7)
    g, o = _pair(oracle_mod, pts, "gaussian", 0.1, 1.0, 64, 1e-6)
    g.storeLRinTree()
    r1 = g.ranks().copy()
    g.set_LRTolerance(1e-10)
    o.set_lr(1e-10)
    _compare_compression(g, o, check_factors=False)
    assert g.ranks().sum() > r1.sum()


def test_errors_are_status_codes():
    with pytest.raises(HODLRError) as e:
        HODLR_Matrix(100, 100, lambda i, j, d: 0.0, np.zeros((1, 100)), 30)
    assert e.value.status == 4  # HODLR_ERR_UNSUPPORTED: host function pointer
    pts, _ = c1_points(256, 1)
    g = HODLR_Matrix(kernelMatrix(256, 256, KernelSpec("gaussian", 0.1, 1.0), pts), 32)
    with pytest.raises(HODLRError) as e:
        g.set_LRMethod("SVD")
    assert e.value.status == 4
    with pytest.raises(HODLRError):
        g.recLU_Solve(np.zeros((10, 1)))


def test_golden_c1_fixture():
    """The CUDA path against the committed C1 fixture directly (tests/golden/
    c1_aca.npz, made by tests/golden/make_golden.py): ranks, iteration counts,
    pivot sequences and the exact bytes of every block's W and V."""
    import os
    from tests.golden.make_golden import factor_hash
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "c1_aca.npz"))
    pts, _ = c1_points()
    assert np.array_equal(pts[0], d["points"])
    g = HODLR_Matrix(4096, 4096, KernelSpec("gaussian", 0.1, 1.0), pts, 64)
    g.set_LRTolerance(1e-10)
    g.storeLRinTree()
    nb = g.num_blocks()
    assert np.array_equal(g.ranks(), d["ranks"])
    assert np.array_equal([g.block_info(b)["iters"] for b in range(nb)], d["iters"])
    rows = np.concatenate([g.pivots(b)[0] for b in range(nb)])
    cols = np.concatenate([g.pivots(b)[1] for b in range(nb)])
    assert np.array_equal(rows, d["prow"]) and np.array_equal(cols, d["pcol"])
    wv = np.array([factor_hash(*g.lowrank(b)) for b in range(nb)], dtype=np.int64)
    assert np.array_equal(wv, d["wv_hash"])


def test_c2_full_size_ranks_and_pivots_match_fixture():
    """The FP64-at-scale workload at full size (N=262144, 4094 blocks): every
    block's rank, iteration count and pivot-sequence hash equals the oracle's
    (tests/golden/c2_blocks.npz, made by tests/golden/make_golden.py --c2)."""
    import os
    from tests.golden.make_golden import pivot_hash
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "c2_blocks.npz"))
    pts = uniform_cube(262144, 2, 2024)
    assert np.allclose([pts.sum(), (pts * pts).sum()], d["points_sum"], rtol=0, atol=1e-6)
    g = HODLR_Matrix(262144, 262144, KernelSpec("matern32", 0.2, 1e-2), pts, 128)
    g.set_LRTolerance(1e-8)
    g.storeLRinTree()
    ranks = g.ranks()
    near = [b for b in range(g.num_blocks()) if g.margin(b)[1] > 0 or d["margin"][b] < 1e-10]
    assert not near
    assert np.array_equal(ranks, d["rank"])
    iters = np.array([g.block_info(b)["iters"] for b in range(g.num_blocks())])
    assert np.array_equal(iters, d["iters"])
    hashes = np.array([pivot_hash(*g.pivots(b)) for b in range(g.num_blocks())], dtype=np.int64)
    assert np.array_equal(hashes, d["pivot_hash"])


def test_refinement_and_gmres_reach_residual_target():
    """2D Matern with a small diagonal shift: the direct solve at tol 1e-8 is far
    from 1e-10; refinement and HODLR-preconditioned GMRES both reach it with the
    full FP64 kernel residual, GMRES in fewer full-kernel products."""
    pts = uniform_cube(8192, 2, 31)
    g = HODLR_Matrix(8192, 8192, KernelSpec("matern32", 0.2, 1e-2), pts, 128)
    g.set_LRTolerance(1e-8)
    b = np.random.default_rng(8).standard_normal((8192, 4))
    x0 = g.recLU_Solve(b)
    assert g.residual(x0, b).max() > 1e-8
    x1, it1, rel1 = g.solve_refined(b, tol=1e-10, max_iter=60)
    assert rel1.max() <= 1e-10 and g.residual(x1, b).max() <= 1.5e-10
    x2 = g.iterative_Solve(b, 200, 1e-10)
    assert g.last_relres.max() <= 1e-10
    assert g.residual(x2, b).max() <= 1.5e-10
    assert g.last_iterations <= it1
    # same solution of the same system
    assert np.linalg.norm(x1 - x2) / np.linalg.norm(x2) < 1e-7


def test_cpp_facade_drop_in(tmp_path):
    """include/HODLR_Matrix.hpp compiled with g++ against libhodlr_b200.so and
    run: the reference's kernel-path test shape, a dense solve and
    iterative_Solve through the C++ drop-in class."""
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = tmp_path / "facade_test"
    subprocess.run(["g++", "-O2", "-std=c++17", os.path.join(root, "tests", "cpp", "facade_test.cpp"),
                    "-I", os.path.join(root, "include"), "-L", os.path.join(root, "dense_hodlr_b200"),
                    "-lhodlr_b200", "-Wl,-rpath," + os.path.join(root, "dense_hodlr_b200"),
                    "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr


def test_cpp_device_functor_constructor(tmp_path):
    """The device-functor form of HODLR_Matrix(int, int, kernel, data, leaf)
    (include/HODLR_Matrix.hpp, compiled with nvcc): a functor returning the
    library's closed-form entries gives the closed-form constructor's ranks and
    solution; a kernel without a closed form solves to a small residual."""
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = tmp_path / "functor_test"
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17",
                    os.path.join(root, "tests", "cpp", "functor_test.cu"),
                    "-I", os.path.join(root, "include"),
                    "-I", os.path.join(root, "dense_hodlr_b200", "csrc"),
                    "-L", os.path.join(root, "dense_hodlr_b200"), "-lhodlr_b200",
                    "-Xlinker", "-rpath", "-Xlinker", os.path.join(root, "dense_hodlr_b200"),
                    "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr


def test_solve_graph_replay_is_bit_identical():
    """The direct solve is captured as a CUDA graph on first use and replayed
    afterwards: replays give the same bits as the first (captured) run and as
    a fresh handle's solve."""
    import torch
    pts = uniform_cube(20000, 2, 21)
    spec = KernelSpec("matern32", 0.2, 1e-2)
    g = HODLR_Matrix(20000, 20000, spec, pts, 128)
    g.set_LRTolerance(1e-8)
    rng = np.random.default_rng(4)
    b1, b2 = (torch.from_numpy(rng.standard_normal((3, 20000))).cuda() for _ in range(2))
    x = [torch.empty_like(b1) for _ in range(3)]
    g.solve_device(b1.data_ptr(), x[0].data_ptr(), 3)   # captured
    g.solve_device(b2.data_ptr(), x[1].data_ptr(), 3)   # replayed
    g.solve_device(b1.data_ptr(), x[2].data_ptr(), 3)   # replayed
    torch.cuda.synchronize()
    assert torch.equal(x[0], x[2])
    f = HODLR_Matrix(20000, 20000, spec, pts, 128)
    f.set_LRTolerance(1e-8)
    y = torch.empty_like(b2)
    f.solve_device(b2.data_ptr(), y.data_ptr(), 3)
    torch.cuda.synchronize()
    assert torch.equal(x[1], y)


@pytest.mark.parametrize("kind,l,shift", [("gaussian", 0.1, 1.0), ("matern32", 0.3, 0.5)])
def test_log_determinant_matches_dense(kind, l, shift):
    """logAbsDeterminant / determinant from the factorization against the dense
    matrix's slogdet (N=3000, 1D, leaf 64, ACA tol 1e-12)."""
    n = 3000
    x = np.sort(np.random.default_rng(8).uniform(-1.0, 1.0, n))
    g = HODLR_Matrix(n, n, KernelSpec(kind, l, shift), x[None, :], 64)
    g.set_LRTolerance(1e-12)
    r = np.abs(x[:, None] - x[None, :])
    K = np.exp(-(r / l) ** 2) if kind == "gaussian" else (1 + np.sqrt(3) * r / l) * np.exp(-np.sqrt(3) * r / l)
    K += shift * np.eye(n)
    sgn, ld = np.linalg.slogdet(K)
    assert abs(g.logAbsDeterminant() - ld) <= 1e-9 * abs(ld)
    s2, ld2 = g.slogdet()  # determinant() itself under/overflows at this size
    assert s2 == sgn and ld2 == g.logAbsDeterminant()


def test_against_the_oracles_own_libm_entries(oracle_mod):
    """Against an oracle that evaluates the entries with its own code and libm
    (as the reference's kernel functors do), sharing no formula with the GPU.
    The reference's own kernel functor (quadraticKernel, test/test.cpp:12-17,
    r*r + 1 with a zero diagonal) is exact arithmetic: pivots, ranks and W/V
    bit for bit.  The C1 Gaussian goes through exp, where last-bit entry
    differences may move late pivots of a few blocks: there both solutions
    are held to the dense FP64 LU at the same bar."""
    rng = np.random.default_rng(11)
    x = rng.uniform(-1.0, 1.0, 4000)[None, :]
    g = HODLR_Matrix(4000, 4000, KernelSpec("quadratic", 1.0, 0.0, True, 0.0), x, 30)
    g.set_LRTolerance(1e-8)
    o = oracle_mod.OracleHODLR.from_kernel(x, 3, 1.0, leaf=30, diag_replace=True, libm=True)
    o.set_lr(1e-8)
    _compare_compression(g, o)
    pts, rng2 = c1_points()
    g = HODLR_Matrix(4096, 4096, KernelSpec("gaussian", 0.1, 1.0), pts, 64)
    g.set_LRTolerance(1e-10)
    o = oracle_mod.OracleHODLR.from_kernel(pts, 0, 0.1, shift=1.0, leaf=64, libm=True)
    o.set_lr(1e-10)
    b = rng2.standard_normal((4096, 1))
    K = np.exp(-((pts[0][:, None] - pts[0][None, :]) ** 2) / 0.01) + np.eye(4096)
    xd = np.linalg.solve(K, b)
    for xs in (g.recLU_Solve(b), o.solve(b)):
        assert np.linalg.norm(xs - xd) / np.linalg.norm(xd) < 1e-9
