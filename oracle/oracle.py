"""ctypes binding of the CPU oracle (liboracle.so).  TEST INFRASTRUCTURE ONLY.

The oracle restates the reference's hot path on the CPU (see the header of
hodlr_oracle.cpp for the file:line map).  Only tests/, __graft_entry__.smoke()
and the cpu_baseline leg of bench.py use this module; the product package
never imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build():
    """Compile liboracle.so with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.orc_create_kernel.restype = ctypes.c_void_p
        L.orc_create_kernel.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int,
                                        ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                        ctypes.c_double, ctypes.c_int]
        L.orc_create_dense.restype = ctypes.c_void_p
        L.orc_create_dense.argtypes = [ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_set_entry_mode.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_set_user_tree.argtypes = [ctypes.c_void_p, ctypes.c_int, _ip, _ip, _ip]
        L.orc_set_user_tree.restype = ctypes.c_int
        L.orc_set_user_tree_bounds.argtypes = [ctypes.c_void_p, ctypes.c_int] + [_ip] * 7
        L.orc_set_user_tree_bounds.restype = ctypes.c_int
        L.orc_set_lr.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
        L.orc_compress.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_factorize.argtypes = [ctypes.c_void_p]
        L.orc_factorize_mt.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_solve.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.orc_solve_mt.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, ctypes.c_int]
        L.orc_recsm_solve.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.orc_recsm_logdet.argtypes = [ctypes.c_void_p, _ip]
        L.orc_recsm_logdet.restype = ctypes.c_double
        for f in ("orc_num_levels", "orc_num_inner", "orc_num_leaves"):
            getattr(L, f).argtypes = [ctypes.c_void_p]
        L.orc_inner_info.argtypes = [ctypes.c_void_p, ctypes.c_int, _ip, _ip, _ip, _ip]
        L.orc_leaf_info.argtypes = [ctypes.c_void_p, ctypes.c_int, _ip, _ip, _ip]
        for f in ("orc_block_rank", "orc_block_iters"):
            getattr(L, f).argtypes = [ctypes.c_void_p, ctypes.c_int]
        for f in ("orc_block_eps", "orc_block_margin"):
            getattr(L, f).argtypes = [ctypes.c_void_p, ctypes.c_int]
            getattr(L, f).restype = ctypes.c_double
        L.orc_block_pivots.argtypes = [ctypes.c_void_p, ctypes.c_int, _ip, _ip]
        L.orc_block_lowrank.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.orc_entry.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.orc_entry.restype = ctypes.c_double
        L.orc_exp.argtypes = [ctypes.c_double]
        L.orc_exp.restype = ctypes.c_double
        L.orc_exp_tang.argtypes = [ctypes.c_double]
        L.orc_exp_tang.restype = ctypes.c_double
        L.orc_exp_tang_neg.argtypes = [ctypes.c_double]
        L.orc_exp_tang_neg.restype = ctypes.c_double
        L.orc_tang_entry.argtypes = [ctypes.c_int]
        L.orc_tang_entry.restype = ctypes.c_double
        L.orc_kernel_matvec.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, ctypes.c_int]
        L.orc_kernel_matvec_rows.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp,
                                             ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_aca_block.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _dp, _ip]
        L.orc_aca_block_mt.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _dp, _ip,
                                       ctypes.c_int]
        L.orc_bench_node.restype = ctypes.c_double
        L.orc_bench_node.argtypes = [ctypes.c_int] * 6
        L.orc_bench_leaf.restype = ctypes.c_double
        L.orc_bench_leaf.argtypes = [ctypes.c_int] * 2
        _LIB = L
    return _LIB


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


class OracleHODLR:
    """CPU restatement of HODLR_Matrix for the recLU path (test oracle)."""

    def __init__(self, handle, n, keep=None):
        self.h = handle
        self.n = n
        self._keep = keep

    @classmethod
    def from_kernel(cls, pts, ktype, length_scale, shift=0.0, leaf=30,
                    diag_replace=False, diag_value=0.0, libm=False):
        """libm=True: entries from the oracle's own formulas with libm's exp and
        sqrt, as the reference's kernel functors compute them, instead of the
        closed forms the product shares (last-bit differences)."""
        pts = np.ascontiguousarray(np.atleast_2d(pts), dtype=np.float64)  # (dim, n)
        dim, n = pts.shape
        h = lib().orc_create_kernel(n, dim, _ptr(pts), int(ktype), float(length_scale),
                                    float(shift), int(bool(diag_replace)),
                                    float(diag_value), int(leaf))
        if libm:
            lib().orc_set_entry_mode(h, 1)
        return cls(h, n, pts)

    @classmethod
    def from_dense(cls, A, leaf=30):
        A = np.asfortranarray(A, dtype=np.float64)
        n = A.shape[0]
        h = lib().orc_create_dense(n, _ptr(A), n, int(leaf))
        return cls(h, n, A)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def set_user_tree(self, split, left, right, bounds=None):
        """User index tree in pre-order; returns 0, or 1 if invalid.  bounds:
        (top min, bottom min, top max, bottom max) rank bounds per user node
        (user_IndexTree::node, -1 for none), or None."""
        a = [np.ascontiguousarray(v, dtype=np.int32) for v in (split, left, right)]
        if bounds is None:
            return lib().orc_set_user_tree(self.h, len(a[0]), *[x.ctypes.data_as(_ip) for x in a])
        b = [np.ascontiguousarray(v, dtype=np.int32) for v in bounds]
        assert len(b) == 4 and all(len(v) == len(a[0]) for v in b)
        return lib().orc_set_user_tree_bounds(self.h, len(a[0]),
                                              *[x.ctypes.data_as(_ip) for x in a + b])

    def set_lr(self, tol, min_pivot=0.0):
        lib().orc_set_lr(self.h, float(tol), float(min_pivot))

    def compress(self, nthreads=None):
        lib().orc_compress(self.h, int(nthreads or os.cpu_count() or 1))

    def factorize(self, nthreads=1):
        """recLU_Factorize; nthreads > 1 runs sibling subtrees on threads
        (same results as the sequential recursion)."""
        return lib().orc_factorize_mt(self.h, int(nthreads))

    def solve(self, b, nthreads=1):
        b = np.asfortranarray(b, dtype=np.float64)
        if b.ndim == 1:
            b = b.reshape(-1, 1, order="F")
        x = np.zeros_like(b, order="F")
        lib().orc_solve_mt(self.h, b.shape[1], _ptr(b), _ptr(x), int(nthreads))
        return x

    def recsm_solve(self, b):
        """recSM_Solve (src/HODLR_Matrix.cpp:805-841): the recursive
        Sherman-Morrison factorization (kept) and its solve."""
        b = np.asfortranarray(b, dtype=np.float64)
        if b.ndim == 1:
            b = b.reshape(-1, 1, order="F")
        x = np.zeros_like(b, order="F")
        lib().orc_recsm_solve(self.h, b.shape[1], _ptr(b), _ptr(x))
        return x

    def recsm_slogdet(self):
        """(sign, log|det|) from the recSM factorization's leaf and perturbI
        LUs (calcDeterminant, src/HODLR_Matrix.cpp:1660-1697)."""
        sg = ctypes.c_int()
        ld = lib().orc_recsm_logdet(self.h, ctypes.byref(sg))
        return sg.value, ld

    # tree / block introspection
    def num_levels(self):
        return lib().orc_num_levels(self.h)

    def inner_nodes(self):
        L = lib()
        out = []
        a, b, c, d = (ctypes.c_int() for _ in range(4))
        for p in range(L.orc_num_inner(self.h)):
            L.orc_inner_info(self.h, p, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c),
                             ctypes.byref(d))
            out.append((a.value, b.value, c.value, d.value))
        return out

    def leaves(self):
        L = lib()
        out = []
        a, b, c = (ctypes.c_int() for _ in range(3))
        for p in range(L.orc_num_leaves(self.h)):
            L.orc_leaf_info(self.h, p, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
            out.append((a.value, b.value, c.value))
        return out

    def num_blocks(self):
        return 2 * lib().orc_num_inner(self.h)

    def ranks(self):
        L = lib()
        return np.array([L.orc_block_rank(self.h, b) for b in range(self.num_blocks())],
                        dtype=np.int32)

    def iters(self):
        L = lib()
        return np.array([L.orc_block_iters(self.h, b) for b in range(self.num_blocks())],
                        dtype=np.int32)

    def margins(self):
        L = lib()
        return np.array([L.orc_block_margin(self.h, b) for b in range(self.num_blocks())])

    def pivots(self, b):
        nb = self.n
        rows = np.zeros(nb, dtype=np.int32)
        cols = np.zeros(nb, dtype=np.int32)
        k = lib().orc_block_pivots(self.h, b, _ptr(rows, _ip), _ptr(cols, _ip))
        return rows[:k].copy(), cols[:k].copy()

    def lowrank(self, b, m, n):
        r = lib().orc_block_rank(self.h, b)
        W = np.zeros((m, r), order="F")
        V = np.zeros((n, r), order="F")
        lib().orc_block_lowrank(self.h, b, _ptr(W), _ptr(V))
        return W, V

    def aca_block_sample(self, b, budget_s, nthreads=1):
        """Run the ACA of block b for at most budget_s seconds (cost sampling)."""
        secs = ctypes.c_double()
        fin = ctypes.c_int()
        it = lib().orc_aca_block_mt(self.h, int(b), float(budget_s), ctypes.byref(secs),
                                    ctypes.byref(fin), int(nthreads))
        return it, secs.value, bool(fin.value)

    def entry(self, i, j):
        return lib().orc_entry(self.h, i, j)

    def kernel_matvec(self, x, nthreads=None):
        x = np.asfortranarray(x, dtype=np.float64)
        if x.ndim == 1:
            x = x.reshape(-1, 1, order="F")
        y = np.zeros_like(x, order="F")
        lib().orc_kernel_matvec(self.h, x.shape[1], _ptr(x), _ptr(y),
                                int(nthreads or os.cpu_count() or 1))
        return y

    def kernel_matvec_rows(self, x, row0, nrows, nthreads=None):
        """Rows [row0, row0 + nrows) of K x (the other rows of the result are 0)."""
        x = np.asfortranarray(x, dtype=np.float64)
        if x.ndim == 1:
            x = x.reshape(-1, 1, order="F")
        y = np.zeros_like(x, order="F")
        lib().orc_kernel_matvec_rows(self.h, x.shape[1], _ptr(x), _ptr(y), int(row0),
                                     int(nrows), int(nthreads or os.cpu_count() or 1))
        return y


def bench_node(st, sb, kt, kb, c, solve_only=False):
    return lib().orc_bench_node(int(st), int(sb), int(kt), int(kb), int(c), int(solve_only))


def bench_leaf(s, c):
    return lib().orc_bench_leaf(int(s), int(c))


def hx_exp(x):
    return lib().orc_exp(float(x))


def hx_exp_tang(x):
    return lib().orc_exp_tang(float(x))


def hx_exp_tang_neg(x):
    return lib().orc_exp_tang_neg(float(x))


def tang_entry(j):
    """Entry j of the 2^(j/256) table of the residual path's exp (kfast.cuh)."""
    return lib().orc_tang_entry(int(j))
