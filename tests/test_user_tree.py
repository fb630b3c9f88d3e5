"""User index trees (hodlr_set_index_tree): the reference's userTree_To_HODLRTree
(src/HODLR_Tree.cpp:207-327) restated in the oracle (CPU) and on the GPU path,
checked against each other bit for bit."""
import numpy as np
import pytest

from dense_hodlr_b200.points import uniform_cube

# root split at 999; its left child a user node split at 499 with default
# subtrees; its right child a user node split at 1999 with default subtrees
TREE = ([999, 499, 1999], [1, -1, -1], [2, -1, -1])


def test_oracle_user_tree_shape(oracle_mod):
    pts = uniform_cube(3000, 2, 3)
    o = oracle_mod.OracleHODLR.from_kernel(pts, 1, 0.2, shift=1e-2, leaf=64)
    assert o.set_user_tree(*TREE) == 0
    inner = o.inner_nodes()
    assert inner[:3] == [(0, 0, 999, 2999), (1, 0, 499, 999), (1, 1000, 1999, 2999)]
    # below a user node without children: left child floor(s/2) on top (split
    # 249), right child split at split + floor(s/2) (749), as the reference
    assert (2, 0, 249, 499) in inner and (2, 500, 749, 999) in inner
    assert o.set_user_tree([3000], [-1], [-1]) == 1   # split outside the node
    assert o.set_user_tree([999, 499], [1, -1], [-1, -1]) == 1  # one child only


@pytest.mark.gpu
def test_user_tree_matches_oracle(oracle_mod):
    from dense_hodlr_b200 import HODLR_Matrix, HODLRError, KernelSpec
    from tests.test_gpu_parity import SOLVE_TOL, _compare_compression
    pts = uniform_cube(3000, 2, 3)
    g = HODLR_Matrix(3000, 3000, KernelSpec("matern32", 0.2, 1e-2), pts, 64)
    g.set_LRTolerance(1e-8)
    n_default = g.num_blocks()
    g.set_index_tree(*TREE)
    o = oracle_mod.OracleHODLR.from_kernel(pts, 1, 0.2, shift=1e-2, leaf=64)
    o.set_lr(1e-8)
    assert o.set_user_tree(*TREE) == 0
    _compare_compression(g, o)
    b = np.random.default_rng(5).standard_normal((3000, 2))
    x = g.recLU_Solve(b)
    xo = o.solve(b)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= SOLVE_TOL
    # an invalid tree is refused and the default tree comes back
    with pytest.raises(HODLRError):
        g.set_index_tree([5000], [-1], [-1])
    assert g.num_blocks() == n_default
