"""Forests of independent systems (hodlr_create_forest): one handle whose
level launches span every system, checked system by system against one
handle per system."""
import ctypes

import numpy as np
import pytest

from dense_hodlr_b200 import HODLR_Matrix, KernelSpec, _lib
from dense_hodlr_b200.points import uniform_1d_sorted, uniform_cube


def test_forest_rejects_bad_arguments():
    lib = _lib.lib()
    h = ctypes.c_void_p()
    sizes = (ctypes.c_int * 2)(100, 0)
    pts = np.zeros(200)
    descs = (_lib.KernelDesc * 2)(KernelSpec("gaussian", 0.1).desc(), KernelSpec("gaussian", 0.1).desc())
    dp = pts.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    assert lib.hodlr_create_forest(ctypes.byref(h), 2, sizes, 1, dp, descs, 64) == _lib.ERR_ARG
    assert lib.hodlr_create_forest(ctypes.byref(h), 0, sizes, 1, dp, descs, 64) == _lib.ERR_ARG
    sizes[1] = 100
    bad = (_lib.KernelDesc * 2)(KernelSpec("gaussian", 0.1).desc(), KernelSpec("gaussian", -1.0).desc())
    assert lib.hodlr_create_forest(ctypes.byref(h), 2, sizes, 1, dp, bad, 64) == _lib.ERR_ARG


SYSTEMS = [  # (points, kernel)
    (lambda: uniform_1d_sorted(3000, -1.0, 1.0, 5), KernelSpec("gaussian", 0.1, 0.5)),
    (lambda: uniform_cube(9000, 2, 6), KernelSpec("matern32", 0.2, 1e-2)),
    (lambda: uniform_cube(700, 2, 7), KernelSpec("gaussian", 0.3, 1.0)),
    (lambda: uniform_1d_sorted(50, 0.0, 1.0, 8), KernelSpec("matern32", 0.5, 0.1)),
    (lambda: uniform_cube(17000, 2, 9), KernelSpec("gaussian", 0.3, 1.0)),
]


def _block_table(g, off=0, end=None):
    """(level, row0 - off, col0 - off) -> (rank, block) for blocks within [off, end)."""
    t = {}
    for b in range(g.num_blocks()):
        i = g.block_info(b)
        if end is not None and not (off <= i["row0"] < end):
            continue
        t[(i["level"], i["row0"] - off, i["col0"] - off)] = (i["rank"], b)
    return t


@pytest.mark.gpu
def test_forest_matches_one_handle_per_system():
    import torch
    systems = [(mk(), k) for mk, k in SYSTEMS]
    F = HODLR_Matrix.forest(systems, leaf=64)
    F.set_LRTolerance(1e-8)
    F.storeLRinTree()
    n = F.n
    rng = np.random.default_rng(3)
    b = rng.standard_normal((n, 2))
    xf = F.recLU_Solve(b)
    # block-diagonal product
    xd = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
    yd = torch.empty_like(xd)
    F.kernel_matvec_device(xd.data_ptr(), yd.data_ptr(), 2)
    torch.cuda.synchronize()
    yf = yd.cpu().numpy().T
    ft = _block_table(F)
    for q, (p, k) in enumerate(systems):
        o, e = int(F.offsets[q]), int(F.offsets[q + 1])
        g = HODLR_Matrix(e - o, e - o, k, p, 64)
        g.set_LRTolerance(1e-8)
        g.storeLRinTree()
        # the same tree and, off near ties of the stopping test, the same ranks
        gt = _block_table(g)
        sub = {key: v for key, v in _block_table(F, o, e).items()}
        assert set(sub) == set(gt)
        for key, (r, bi) in gt.items():
            if g.margin(bi)[0] > 1e-6:
                assert sub[key][0] == r, (q, key)
        # solutions
        xg = g.recLU_Solve(b[o:e])
        assert np.linalg.norm(xf[o:e] - xg) / np.linalg.norm(xg) <= 1e-10, q
        # full-kernel product of the system
        xs = torch.from_numpy(np.ascontiguousarray(b[o:e].T)).cuda()
        ys = torch.empty_like(xs)
        g.kernel_matvec_device(xs.data_ptr(), ys.data_ptr(), 2)
        torch.cuda.synchronize()
        yg = ys.cpu().numpy().T
        assert np.linalg.norm(yf[o:e] - yg) / np.linalg.norm(yg) <= 1e-13, q
    assert len(ft) == F.num_blocks()


@pytest.mark.gpu
def test_forest_refinement_reaches_target_per_system():
    """A batch in the shape of the uneven-systems workload, scaled down: 24
    systems, N log-uniform in [1024, 8192], 1D or 2D uniform points, Gaussian
    or Matern-3/2, l log-uniform in [0.05, 0.5], shift log-uniform in
    [1e-2, 1], leaf 64, tol 1e-8, one right-hand side each, refined until every
    system's own residual is <= 1e-10; checked by each system's own handle."""
    import torch
    rng = np.random.default_rng(11)
    systems = []
    for q in range(24):
        n = int(np.exp(rng.uniform(np.log(1024), np.log(8192))))
        p = uniform_1d_sorted(n, 0.0, 1.0, 100 + q) if q % 2 else uniform_cube(n, 2, 100 + q)
        kind = "gaussian" if rng.random() < 0.5 else "matern32"
        l = float(np.exp(rng.uniform(np.log(0.05), np.log(0.5))))
        sh = float(np.exp(rng.uniform(np.log(1e-2), np.log(1.0))))
        systems.append((p, KernelSpec(kind, l, sh)))
    F = HODLR_Matrix.forest(systems, leaf=64)
    F.set_LRTolerance(1e-8)
    b = rng.standard_normal(F.n)
    bd = torch.from_numpy(b).cuda()
    xd = torch.empty_like(bd)
    it, rel = F.forest_refine_device(bd.data_ptr(), xd.data_ptr(), 1, tol=1e-10, max_iter=60)
    assert rel.max() <= 1e-10, (it, rel.ravel())
    x = xd.cpu().numpy()
    for q in (0, 5, 11, 23):
        o, e = int(F.offsets[q]), int(F.offsets[q + 1])
        p, k = systems[q]
        g = HODLR_Matrix(e - o, e - o, k, p, 64)
        assert g.residual(x[o:e, None], b[o:e, None]).max() <= 1.5e-10


@pytest.mark.gpu
def test_forest_gmres_reaches_target_per_system():
    """HODLR-preconditioned GMRES on a forest (hodlr_iterative_solve_device):
    every system is its own GMRES problem -- inner products, Hessenberg matrix
    and stopping test on its own rows -- so each system's own residual reaches
    1e-10, checked by each system's own handle, with fewer iterations than
    the per-system refinement of the same batch needs passes."""
    import torch
    rng = np.random.default_rng(11)
    systems = []
    for q in range(24):
        n = int(np.exp(rng.uniform(np.log(1024), np.log(8192))))
        p = uniform_1d_sorted(n, 0.0, 1.0, 100 + q) if q % 2 else uniform_cube(n, 2, 100 + q)
        kind = "gaussian" if rng.random() < 0.5 else "matern32"
        l = float(np.exp(rng.uniform(np.log(0.05), np.log(0.5))))
        sh = float(np.exp(rng.uniform(np.log(1e-2), np.log(1.0))))
        systems.append((p, KernelSpec(kind, l, sh)))
    F = HODLR_Matrix.forest(systems, leaf=64)
    F.set_LRTolerance(1e-8)
    b = rng.standard_normal((F.n, 2))
    bd = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
    xd = torch.empty_like(bd)
    it, rel = F.iterative_solve_device(bd.data_ptr(), xd.data_ptr(), 2, tol=1e-10, max_iter=60)
    assert rel.max() <= 1e-10, (it, rel)
    xr = torch.empty_like(bd)
    it_ref, _ = F.forest_refine_device(bd.data_ptr(), xr.data_ptr(), 2, tol=1e-10, max_iter=60)
    assert it <= it_ref, (it, it_ref)
    x = xd.cpu().numpy().T
    for q in (0, 5, 11, 23):
        o, e = int(F.offsets[q]), int(F.offsets[q + 1])
        p, k = systems[q]
        g = HODLR_Matrix(e - o, e - o, k, p, 64)
        assert g.residual(x[o:e], b[o:e]).max() <= 1.5e-10
