"""Python mirror of the reference's HODLR_Matrix interface for the recLU path.

Same names, argument meaning and error behaviour as include/HODLR_Matrix.hpp
(constructors :76 and :162, recLU_Solve :214, recLU_Compute :217,
set_LRTolerance / set_minPivot / set_LRMethod :222-225, timing getters
:234-241, printResultInfo :45).  Every call goes through the C ABI of
libhodlr_b200.so (include/hodlr_b200.h); there is no CPU fallback, and a
missing library or GPU raises HODLRError.
"""
import ctypes
import os

import numpy as np

from . import _lib as _L

GAUSSIAN = 0
MATERN32 = 1
INV_MULTIQUADRIC = 2
QUADRATIC = 3
EXPONENTIAL = 4

_KERNEL_NAMES = {"gaussian": GAUSSIAN, "matern32": MATERN32,
                 "inv_multiquadric": INV_MULTIQUADRIC, "quadratic": QUADRATIC,
                 "exponential": EXPONENTIAL}


class HODLRError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        super().__init__(f"{_L.status_string(status)} ({status}): {msg}")


class KernelSpec:
    """Closed-form kernel K_ij = f(r_ij), diagonal shifted or replaced."""

    def __init__(self, kind, length_scale=1.0, diag_shift=0.0, diag_replace=False,
                 diag_value=0.0):
        self.type = _KERNEL_NAMES[kind] if isinstance(kind, str) else int(kind)
        self.length_scale = float(length_scale)
        self.diag_shift = float(diag_shift)
        self.diag_replace = bool(diag_replace)
        self.diag_value = float(diag_value)

    def desc(self):
        return _L.KernelDesc(self.type, self.length_scale, self.diag_shift,
                             int(self.diag_replace), self.diag_value)


class kernelMatrix:
    """Stand-in for the reference kernelMatrix (include/kernel.hpp:6-33).

    The reference wraps `double (*)(int i, int j, void* data)`; on the GPU the
    entry must be a closed form of point coordinates, so `kernel` is a
    KernelSpec and `data` the points (dim x n).  A Python callable is
    rejected with HODLR_ERR_UNSUPPORTED, like hodlr_create_fnptr.
    """

    def __init__(self, numRows, numCols, kernel, data):
        if numRows != numCols:
            raise HODLRError(_L.ERR_ARG, "only square kernel matrices form a HODLR tree")
        self.numRows, self.numCols = int(numRows), int(numCols)
        self.kernel = kernel
        self.data = data

    def rows(self):
        return self.numRows

    def cols(self):
        return self.numCols


def _check(h, rc):
    if rc != 0:
        msg = _L.lib().hodlr_last_error(h).decode() if h else ""
        raise HODLRError(rc, msg)


def _as_f64_fortran(a):
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 1:
        a = a.reshape(-1, 1)
    return np.asfortranarray(a)


class HODLR_Matrix:
    """HODLR_Matrix for the recLU path on one B200.

    HODLR_Matrix(A, leaf=30, LR_Method="partialPiv_ACA")           dense input
    HODLR_Matrix(numRows, numCols, kernel, data, leaf=30)           kernel input
    HODLR_Matrix(kernelMatrix(...), leaf=30)
    """

    def __init__(self, *args, leaf=None, LR_Method="partialPiv_ACA", **kw):
        self.printResultInfo = False
        self._h = None
        lib = _L.lib()
        h = ctypes.c_void_p()
        if len(args) >= 1 and isinstance(args[0], np.ndarray) and args[0].ndim == 2:
            A = np.asfortranarray(args[0], dtype=np.float64)
            if A.shape[0] != A.shape[1]:
                raise HODLRError(_L.ERR_ARG, "matrix must be square")
            leaf = int(args[1]) if len(args) > 1 else (leaf or 30)
            if len(args) > 2:
                LR_Method = args[2]
            self.n = A.shape[0]
            rc = lib.hodlr_create_dense(ctypes.byref(h), self.n,
                                        A.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                        self.n, int(leaf))
            _check(None, rc)
        else:
            if len(args) >= 1 and isinstance(args[0], kernelMatrix):
                km = args[0]
                leaf = int(args[1]) if len(args) > 1 else (leaf or 30)
                n, kernel, data = km.numRows, km.kernel, km.data
            else:
                if len(args) < 4:
                    raise HODLRError(_L.ERR_ARG, "expected (numRows, numCols, kernel, data[, leaf])")
                n, ncols, kernel, data = args[:4]
                if n != ncols:
                    raise HODLRError(_L.ERR_ARG, "only square kernel matrices form a HODLR tree")
                leaf = int(args[4]) if len(args) > 4 else (leaf or 30)
            if callable(kernel) and not isinstance(kernel, KernelSpec):
                rc = lib.hodlr_create_fnptr(ctypes.byref(h), int(n), int(n), None, None, int(leaf))
                _check(None, rc)
            pts = np.ascontiguousarray(np.atleast_2d(np.asarray(data, dtype=np.float64)))
            dim = pts.shape[0]
            if pts.shape[1] != n:
                raise HODLRError(_L.ERR_ARG, "data must be dim x n point coordinates")
            d = kernel.desc()
            self.n = int(n)
            rc = lib.hodlr_create_kernel(ctypes.byref(h), self.n, dim,
                                         pts.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                         ctypes.byref(d), int(leaf))
            _check(None, rc)
        self._h = h
        self.leaf = leaf
        if LR_Method != "partialPiv_ACA":
            self.set_LRMethod(LR_Method)

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                _L.lib().hodlr_destroy(self._h)
            except TypeError:  # interpreter shutdown: the module globals are gone
                pass
            self._h = None

    # ------------------------------------------------------------ setters
    def set_LRTolerance(self, tolerance):
        _check(self._h, _L.lib().hodlr_set_lr_tolerance(self._h, float(tolerance)))

    def set_minPivot(self, minPivot):
        _check(self._h, _L.lib().hodlr_set_min_pivot(self._h, float(minPivot)))

    def set_LRMethod(self, method):
        _check(self._h, _L.lib().hodlr_set_lr_method(self._h, method.encode()))

    def set_precision(self, precision):
        """'fp64' (default), 'tf32', 'bf16' or 'tf32x3' for the Woodbury products."""
        code = ({"fp64": 0, "tf32": 1, "bf16": 2, "tf32x3": 3}[precision]
                if isinstance(precision, str) else int(precision))
        _check(self._h, _L.lib().hodlr_set_precision(self._h, code))

    def set_capacity_hint(self, caps):
        """Initial low-rank columns per inner level (results do not depend on it)."""
        a = np.ascontiguousarray(caps, dtype=np.int32)
        _check(self._h, _L.lib().hodlr_set_capacity_hint(
            self._h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(a)))

    def reset(self):
        """Drop the compression and factorization (reset_attributes,
        src/HODLR_Matrix.cpp:1232-1246): the next solve recomputes both."""
        _check(self._h, _L.lib().hodlr_reset(self._h))

    def set_checked(self, on=True):
        """Checked mode (hodlr_set_checked): operand extents verified before every
        launch group, the solve without its CUDA graph, and a synchronisation
        after every group, so that a device error names the group that raised
        it.  Same results, slower; HODLR_CHECKED=1 in the environment turns it
        on for every new handle."""
        _check(self._h, _L.lib().hodlr_set_checked(self._h, int(bool(on))))

    def set_aca_streaming(self, on):
        """Top-level ACA panels through the warps' rings, one 2D tensor copy per
        ring tile (2, default) or one bulk copy per panel column (1), or loaded
        per thread (0).  Same results in every mode."""
        _check(self._h, _L.lib().hodlr_set_aca_streaming(self._h, int(on)))

    def set_factor_in_place(self, mode):
        """K^-1 U over the U panels: 1 always, 0 never, -1 (default) only when
        separate memory cannot be allocated (hodlr_set_factor_in_place)."""
        _check(self._h, _L.lib().hodlr_set_factor_in_place(self._h, int(mode)))

    def factor_in_place_levels(self):
        v = ctypes.c_int()
        _check(self._h, _L.lib().hodlr_get_factor_in_place(self._h, ctypes.byref(v)))
        return v.value

    # ------------------------------------------------------------- solver
    def storeLRinTree(self):
        _check(self._h, _L.lib().hodlr_compress(self._h))

    def set_solver_form(self, form):
        """'recLU' (default) or 'recSM' (hodlr_set_solver_form): the
        factorization every solve, refinement and log-determinant uses.
        Changing it drops the factorization; the compression is kept."""
        f = {"recLU": _L.FORM_RECLU, "recSM": _L.FORM_RECSM}.get(form)
        if f is None:
            raise HODLRError(_L.ERR_ARG, "solver form is 'recLU' or 'recSM'")
        _check(self._h, _L.lib().hodlr_set_solver_form(self._h, f))

    def get_solver_form(self):
        f = ctypes.c_int()
        _check(self._h, _L.lib().hodlr_get_solver_form(self._h, ctypes.byref(f)))
        return "recSM" if f.value == _L.FORM_RECSM else "recLU"

    def recLU_Compute(self):
        """Compression and the recLU factorization (src/HODLR_Matrix.cpp:794-803)."""
        self.set_solver_form("recLU")
        _check(self._h, _L.lib().hodlr_factorize(self._h))

    def recLU_Solve(self, input_RHS):
        """recLU_Solve (src/HODLR_Matrix.cpp:757-792)."""
        self.set_solver_form("recLU")
        return self._direct_solve(input_RHS, "recLU")

    def recSM_Solve(self, input_RHS):
        """recSM_Solve (src/HODLR_Matrix.cpp:805-841): the recursive
        Sherman-Morrison factorization (perturbI nodes) and its solve."""
        self.set_solver_form("recSM")
        return self._direct_solve(input_RHS, "recSM")

    def _direct_solve(self, input_RHS, name):
        b = _as_f64_fortran(input_RHS)
        if b.shape[0] != self.n:
            raise HODLRError(_L.ERR_ARG, "right-hand side has the wrong number of rows")
        x = np.zeros_like(b, order="F")
        dp = ctypes.POINTER(ctypes.c_double)
        _check(self._h, _L.lib().hodlr_solve(self._h, b.shape[1], b.ctypes.data_as(dp), self.n,
                                             x.ctypes.data_as(dp), self.n))
        if self.printResultInfo:
            rel = self.residual(x, b)
            print("**************************************************")
            print(f"Solver Type                      = {name}")
            print(f"Low-Rank Computation Time        = {self.get_LR_ComputationTime()} seconds")
            print(f"Factorization Time               = {self.get_recLU_FactorizationTime()} seconds")
            print(f"Solve Time                       = {self.get_recLU_SolveTime()} seconds")
            print(f"Total Solve Time                 = {self.get_recLU_TotalTime()} seconds")
            print(f"Residual l2 Relative Error       = {rel.max()}")
        return x

    def solve_refined(self, input_RHS, tol=1e-10, max_iter=20):
        """recLU_Solve followed by iterative refinement with the full FP64
        kernel residual; returns (x, corrections, per-column rel. residual)."""
        b = _as_f64_fortran(input_RHS)
        if b.shape[0] != self.n:
            raise HODLRError(_L.ERR_ARG, "right-hand side has the wrong number of rows")
        x = np.zeros_like(b, order="F")
        rel = np.zeros(b.shape[1])
        it = ctypes.c_int()
        dp = ctypes.POINTER(ctypes.c_double)
        _check(self._h, _L.lib().hodlr_solve_refined(self._h, b.shape[1], b.ctypes.data_as(dp),
                                                     self.n, x.ctypes.data_as(dp), self.n,
                                                     float(tol), int(max_iter), ctypes.byref(it),
                                                     rel.ctypes.data_as(dp)))
        return x, it.value, rel

    def iterative_Solve(self, input_RHS, maxIterations=1000, stop_tolerance=1e-10,
                        init_LRTolerance=None, input_LR_Method="partialPiv_ACA",
                        directSolve_Method="recLU", restart=32):
        """iterative_Solve (include/HODLR_Matrix.hpp:219): HODLR-preconditioned
        GMRES from the recLU solution, to a relative residual ||b - K x|| / ||b||
        of stop_tolerance with the full FP64 kernel (formed once by a product,
        then updated from the products of the iterations).  Returns the
        solution like the reference; the iteration count and residuals are
        kept in self.last_iterations / last_relres."""
        if init_LRTolerance is not None:
            self.set_LRTolerance(init_LRTolerance)
        self.set_LRMethod(input_LR_Method)
        if directSolve_Method != "recLU":
            raise HODLRError(_L.ERR_UNSUPPORTED, "only the recLU direct solver is on the GPU path")
        b = _as_f64_fortran(input_RHS)
        if b.shape[0] != self.n:
            raise HODLRError(_L.ERR_ARG, "right-hand side has the wrong number of rows")
        x = np.zeros_like(b, order="F")
        rel = np.zeros(b.shape[1])
        it = ctypes.c_int()
        dp = ctypes.POINTER(ctypes.c_double)
        _check(self._h, _L.lib().hodlr_iterative_solve(
            self._h, b.shape[1], b.ctypes.data_as(dp), self.n, x.ctypes.data_as(dp), self.n,
            float(stop_tolerance), int(maxIterations), int(restart), ctypes.byref(it),
            rel.ctypes.data_as(dp)))
        self.last_iterations, self.last_relres = it.value, rel
        return x

    def iterative_solve_device(self, b_ptr, x_ptr, nrhs, tol=1e-10, max_iter=1000, restart=32):
        rel = np.zeros(nrhs)
        it = ctypes.c_int()
        _check(self._h, _L.lib().hodlr_iterative_solve_device(
            self._h, int(nrhs), ctypes.c_void_p(b_ptr), self.n, ctypes.c_void_p(x_ptr), self.n,
            float(tol), int(max_iter), int(restart), ctypes.byref(it),
            rel.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return it.value, rel

    def solve_refined_device(self, b_ptr, x_ptr, nrhs, tol=1e-10, max_iter=20):
        rel = np.zeros(nrhs)
        it = ctypes.c_int()
        _check(self._h, _L.lib().hodlr_solve_refined_device(
            self._h, int(nrhs), ctypes.c_void_p(b_ptr), self.n, ctypes.c_void_p(x_ptr), self.n,
            float(tol), int(max_iter), ctypes.byref(it),
            rel.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return it.value, rel

    def solve_device(self, b_ptr, x_ptr, nrhs, ldb=None, ldx=None):
        """recLU_Solve on device buffers (raw CUDA pointers)."""
        _check(self._h, _L.lib().hodlr_solve_device(self._h, int(nrhs), ctypes.c_void_p(b_ptr),
                                                    int(ldb or self.n), ctypes.c_void_p(x_ptr),
                                                    int(ldx or self.n)))

    def kernel_matvec_device(self, x_ptr, y_ptr, nrhs):
        _check(self._h, _L.lib().hodlr_kernel_matvec_device(self._h, int(nrhs),
                                                            ctypes.c_void_p(x_ptr), self.n,
                                                            ctypes.c_void_p(y_ptr), self.n))

    def residual(self, x, b):
        """Per-column ||K x - b|| / ||b|| with the full FP64 kernel."""
        x = _as_f64_fortran(x)
        b = _as_f64_fortran(b)
        out = np.zeros(b.shape[1])
        dp = ctypes.POINTER(ctypes.c_double)
        _check(self._h, _L.lib().hodlr_residual(self._h, b.shape[1], b.ctypes.data_as(dp), self.n,
                                                x.ctypes.data_as(dp), self.n,
                                                out.ctypes.data_as(dp)))
        return out

    # ------------------------------------------------------------ getters
    def _times(self):
        t = [ctypes.c_double() for _ in range(4)]
        _check(self._h, _L.lib().hodlr_get_times(self._h, *[ctypes.byref(x) for x in t]))
        return [x.value for x in t]

    def get_LR_ComputationTime(self):
        return self._times()[0]

    def get_recLU_FactorizationTime(self):
        return self._times()[1]

    def get_recLU_SolveTime(self):
        return self._times()[2]

    def get_recLU_TotalTime(self):
        return self._times()[3]

    # the recSM timings (members without getters in the reference,
    # include/HODLR_Matrix.hpp:297-299): the last factorization and solve,
    # whichever form ran
    def get_recSM_FactorizationTime(self):
        return self._times()[1]

    def get_recSM_SolveTime(self):
        return self._times()[2]

    def get_recSM_TotalTime(self):
        return self._times()[3]

    def get_MatrixSize(self):
        return self.n

    def rows(self):
        return self.n

    def cols(self):
        return self.n

    # -------------------------------------------------------- diagnostics
    def num_levels(self):
        v = ctypes.c_int()
        _check(self._h, _L.lib().hodlr_get_num_levels(self._h, ctypes.byref(v)))
        return v.value

    def num_blocks(self):
        v = ctypes.c_int()
        _check(self._h, _L.lib().hodlr_get_num_blocks(self._h, ctypes.byref(v)))
        return v.value

    def block_info(self, b):
        v = [ctypes.c_int() for _ in range(7)]
        _check(self._h, _L.lib().hodlr_get_block_info(self._h, int(b), *[ctypes.byref(x) for x in v]))
        return dict(zip(("level", "row0", "col0", "m", "n", "rank", "iters"), [x.value for x in v]))

    def ranks(self):
        out = np.zeros(self.num_blocks(), dtype=np.int32)
        _check(self._h, _L.lib().hodlr_get_ranks(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        return out

    def pivots(self, b):
        info = self.block_info(b)
        cap = max(1, min(info["m"], info["n"]))
        rows = np.zeros(cap, dtype=np.int32)
        cols = np.zeros(cap, dtype=np.int32)
        cnt = ctypes.c_int()
        ip = ctypes.POINTER(ctypes.c_int)
        _check(self._h, _L.lib().hodlr_get_pivots(self._h, int(b), rows.ctypes.data_as(ip),
                                                  cols.ctypes.data_as(ip), ctypes.byref(cnt)))
        return rows[:cnt.value].copy(), cols[:cnt.value].copy()

    def lowrank(self, b):
        info = self.block_info(b)
        W = np.zeros((info["m"], info["rank"]), order="F")
        V = np.zeros((info["n"], info["rank"]), order="F")
        dp = ctypes.POINTER(ctypes.c_double)
        _check(self._h, _L.lib().hodlr_get_lowrank(self._h, int(b), W.ctypes.data_as(dp),
                                                   V.ctypes.data_as(dp)))
        return W, V

    def margin(self, b):
        m = ctypes.c_double()
        n = ctypes.c_int()
        _check(self._h, _L.lib().hodlr_get_block_margin(self._h, int(b), ctypes.byref(m),
                                                        ctypes.byref(n)))
        return m.value, n.value

    # forests of independent systems
    @classmethod
    def forest(cls, systems, leaf=64):
        """One handle for many independent systems: `systems` is a list of
        (points dim_q x n_q, KernelSpec).  Points of lower dimension are
        padded with zero coordinates; rows and columns of system q are
        [offsets[q], offsets[q+1]) of the block-diagonal matrix."""
        lib = _L.lib()
        dim = max(np.atleast_2d(p).shape[0] for p, _ in systems)
        sizes = np.array([np.atleast_2d(p).shape[1] for p, _ in systems], dtype=np.int32)
        pts = np.zeros((dim, int(sizes.sum())), dtype=np.float64)
        o = 0
        for p, _ in systems:
            p = np.atleast_2d(np.asarray(p, dtype=np.float64))
            pts[:p.shape[0], o:o + p.shape[1]] = p
            o += p.shape[1]
        descs = (_L.KernelDesc * len(systems))(*[k.desc() for _, k in systems])
        h = ctypes.c_void_p()
        rc = lib.hodlr_create_forest(ctypes.byref(h), len(systems),
                                     sizes.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), dim,
                                     pts.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), descs,
                                     int(leaf))
        _check(None, rc)
        self = cls.__new__(cls)
        self.printResultInfo = False
        self._h = h
        self.n = int(sizes.sum())
        self.leaf = leaf
        self.offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        return self

    def logAbsDeterminant(self):
        """log|det K| from the factorization (src/HODLR_Matrix.cpp:1666)."""
        v, sg = ctypes.c_double(), ctypes.c_int()
        _check(self._h, _L.lib().hodlr_logdet(self._h, ctypes.byref(v), ctypes.byref(sg)))
        return v.value

    def slogdet(self):
        """(sign, log|det K|), like numpy.linalg.slogdet."""
        v, sg = ctypes.c_double(), ctypes.c_int()
        _check(self._h, _L.lib().hodlr_logdet(self._h, ctypes.byref(v), ctypes.byref(sg)))
        return sg.value, v.value

    def determinant(self):
        """det K (with the sign of the pivoting permutations); overflows to
        inf for large matrices -- prefer logAbsDeterminant."""
        v, sg = ctypes.c_double(), ctypes.c_int()
        _check(self._h, _L.lib().hodlr_logdet(self._h, ctypes.byref(v), ctypes.byref(sg)))
        return sg.value * float(np.exp(v.value))

    def set_index_tree(self, split, left, right, bounds=None):
        """User index tree in pre-order (node 0 = root): split row per node (-1:
        none), child node indices (-1: none; both -1 = default subtrees).
        bounds: (top min, bottom min, top max, bottom max) rank bounds per user
        node (user_IndexTree::node; -1 for none), or None."""
        sp, lf, rt = (np.ascontiguousarray(a, dtype=np.int32) for a in (split, left, right))
        pi = ctypes.POINTER(ctypes.c_int)
        if bounds is None:
            _check(self._h, _L.lib().hodlr_set_index_tree(
                self._h, len(sp), sp.ctypes.data_as(pi), lf.ctypes.data_as(pi),
                rt.ctypes.data_as(pi)))
            return
        bs = [np.ascontiguousarray(a, dtype=np.int32) for a in bounds]
        if len(bs) != 4 or any(len(a) != len(sp) for a in bs):
            raise HODLRError(_L.ERR_ARG, "bounds: four arrays, one value per user node")
        _check(self._h, _L.lib().hodlr_set_index_tree_bounds(
            self._h, len(sp), sp.ctypes.data_as(pi), lf.ctypes.data_as(pi),
            rt.ctypes.data_as(pi), *[a.ctypes.data_as(pi) for a in bs]))

    def num_systems(self):
        n = ctypes.c_int()
        _check(self._h, _L.lib().hodlr_get_num_systems(self._h, ctypes.byref(n)))
        return n.value

    def forest_refine_device(self, d_b, d_x, nrhs, tol=1e-10, max_iter=50):
        """Direct solve + refinement to a per-system residual target on device
        buffers (column-major n x nrhs); returns (corrections, relres nsys x nrhs)."""
        ns = self.num_systems()
        it = ctypes.c_int()
        rel = np.zeros(ns * nrhs, dtype=np.float64)
        _check(self._h, _L.lib().hodlr_forest_refine_device(
            self._h, int(nrhs), ctypes.c_void_p(d_b), self.n, ctypes.c_void_p(d_x), self.n,
            float(tol), int(max_iter), ctypes.byref(it),
            rel.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return it.value, rel.reshape(ns, nrhs)

    # rank predictor (csrc/rank_mlp.cu)
    def set_rank_model(self, params, length_scale):
        """FP32 parameter blob of the rank MLP (None removes it) and the
        kernel length scale of the log-l feature."""
        if params is None:
            _check(self._h, _L.lib().hodlr_set_rank_model(self._h, None, 0.0))
            return
        p = np.ascontiguousarray(params, dtype=np.float32)
        _check(self._h, _L.lib().hodlr_set_rank_model(
            self._h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), float(length_scale)))

    def predicted_ranks(self):
        out = np.zeros(self.num_blocks(), dtype=np.int32)
        _check(self._h, _L.lib().hodlr_get_predicted_ranks(
            self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        return out

    def block_features(self, length_scale):
        out = np.zeros((self.num_blocks(), 14), dtype=np.float32)
        _check(self._h, _L.lib().hodlr_block_features(
            self._h, float(length_scale), out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def aca_stats(self):
        a, s, b = ctypes.c_int(), ctypes.c_double(), ctypes.c_double()
        _check(self._h, _L.lib().hodlr_get_aca_stats(self._h, ctypes.byref(a), ctypes.byref(s),
                                                     ctypes.byref(b)))
        return {"launches": a.value, "seconds": s.value, "bytes": b.value}
