"""Loader of libhodlr_b200.so and ctypes signatures of include/hodlr_b200.h."""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhodlr_b200.so")

OK = 0
ERR_ARG = 1
ERR_CUDA = 2
ERR_ALLOC = 3
ERR_UNSUPPORTED = 4
ERR_SINGULAR = 5
ERR_STATE = 6
ERR_NONFINITE = 7
ERR_TIMEOUT = 8
ERR_IO = 9
ERR_CHECK = 10
FORM_RECLU = 0
FORM_RECSM = 1

_STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "device memory exhausted",
           4: "unsupported on the GPU path", 5: "exact-zero pivot", 6: "call out of order",
           7: "non-finite value", 8: "device wait timed out",
           9: "file could not be read or written",
           10: "check failed: an extent or index outside its buffer"}


def status_string(s):
    return _STATUS.get(s, "unknown status")


class KernelDesc(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("length_scale", ctypes.c_double),
                ("diag_shift", ctypes.c_double), ("diag_replace", ctypes.c_int),
                ("diag_value", ctypes.c_double)]


_H = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_PD = ctypes.POINTER(ctypes.c_double)
_PI = ctypes.POINTER(ctypes.c_int)
_V = ctypes.c_void_p
_VP = ctypes.c_void_p
_PF = ctypes.POINTER(ctypes.c_float)

SIGNATURES = {
    "hodlr_create_kernel": (_I, [ctypes.POINTER(_H), _I, _I, _PD, ctypes.POINTER(KernelDesc), _I]),
    "hodlr_create_dense": (_I, [ctypes.POINTER(_H), _I, _PD, _I, _I]),
    "hodlr_create_dense_device": (_I, [ctypes.POINTER(_H), _I, _I, ctypes.POINTER(_VP),
                                       ctypes.POINTER(ctypes.c_int64)]),
    "hodlr_matrix_file_dims": (_I, [ctypes.c_char_p, _PI, _PI]),
    "hodlr_read_matrix_file": (_I, [ctypes.c_char_p, _I, _I, _PD, _I]),
    "hodlr_write_matrix_file": (_I, [ctypes.c_char_p, _I, _I, _PD, _I]),
    "hodlr_create_fnptr": (_I, [ctypes.POINTER(_H), _I, _I, _V, _V, _I]),
    "hodlr_destroy": (None, [_H]),
    "hodlr_reset": (_I, [_H]),
    "hodlr_set_stream": (_I, [_H, _V]),
    "hodlr_get_launch_count": (_I, [_H, ctypes.POINTER(ctypes.c_longlong)]),
    "hodlr_set_capacity_hint": (_I, [_H, _PI, _I]),
    "hodlr_set_factor_in_place": (_I, [_H, _I]),
    "hodlr_set_aca_streaming": (_I, [_H, _I]),
    "hodlr_set_wait_limit": (_I, [_H, ctypes.c_uint, _I]),
    "hodlr_set_checked": (_I, [_H, _I]),
    "hodlr_set_solver_form": (_I, [_H, _I]),
    "hodlr_get_solver_form": (_I, [_H, ctypes.POINTER(ctypes.c_int)]),
    "hodlr_get_factor_in_place": (_I, [_H, _PI]),
    "hodlr_trim_device_memory": (_I, []),
    "hodlr_create_forest": (_I, [ctypes.POINTER(_H), _I, _PI, _I, _PD, ctypes.POINTER(KernelDesc),
                                 _I]),
    "hodlr_get_num_systems": (_I, [_H, _PI]),
    "hodlr_set_index_tree": (_I, [_H, _I, _PI, _PI, _PI]),
    "hodlr_set_index_tree_bounds": (_I, [_H, _I, _PI, _PI, _PI, _PI, _PI, _PI, _PI]),
    "hodlr_logdet": (_I, [_H, _PD, _PI]),
    "hodlr_forest_refine_device": (_I, [_H, _I, _VP, _I, _VP, _I, _D, _I, _PI, _PD]),
    "hodlr_set_rank_model": (_I, [_H, _PF, _D]),
    "hodlr_get_predicted_ranks": (_I, [_H, _PI]),
    "hodlr_block_features": (_I, [_H, _D, _PF]),
    "hodlr_mlp_scratch_floats": (_I, [_I, ctypes.POINTER(ctypes.c_longlong)]),
    "hodlr_mlp_forward": (_I, [_VP, _VP, _I, _VP, _VP]),
    "hodlr_mlp_train_step": (_I, [_VP, _VP, _VP, _VP, _VP, _I, _VP, ctypes.c_float, _I, _VP, _VP,
                                  _VP]),
    "hodlr_set_precision": (_I, [_H, _I]),
    "hodlr_gemm_device": (_I, [_I, _I, _I, _I, _I, _V, _I, _V, _I, _V, _I, _V]),
    "hodlr_set_lr_tolerance": (_I, [_H, _D]),
    "hodlr_set_min_pivot": (_I, [_H, _D]),
    "hodlr_set_lr_method": (_I, [_H, ctypes.c_char_p]),
    "hodlr_compress": (_I, [_H]),
    "hodlr_factorize": (_I, [_H]),
    "hodlr_solve": (_I, [_H, _I, _PD, _I, _PD, _I]),
    "hodlr_solve_device": (_I, [_H, _I, _V, _I, _V, _I]),
    "hodlr_kernel_matvec_device": (_I, [_H, _I, _V, _I, _V, _I]),
    "hodlr_solve_refined_device": (_I, [_H, _I, _V, _I, _V, _I, _D, _I, _PI, _PD]),
    "hodlr_solve_refined": (_I, [_H, _I, _PD, _I, _PD, _I, _D, _I, _PI, _PD]),
    "hodlr_iterative_solve_device": (_I, [_H, _I, _V, _I, _V, _I, _D, _I, _I, _PI, _PD]),
    "hodlr_iterative_solve": (_I, [_H, _I, _PD, _I, _PD, _I, _D, _I, _I, _PI, _PD]),
    "hodlr_residual": (_I, [_H, _I, _PD, _I, _PD, _I, _PD]),
    "hodlr_get_times": (_I, [_H, _PD, _PD, _PD, _PD]),
    "hodlr_get_num_levels": (_I, [_H, _PI]),
    "hodlr_get_num_blocks": (_I, [_H, _PI]),
    "hodlr_get_block_info": (_I, [_H, _I, _PI, _PI, _PI, _PI, _PI, _PI, _PI]),
    "hodlr_get_ranks": (_I, [_H, _PI]),
    "hodlr_get_pivots": (_I, [_H, _I, _PI, _PI, _PI]),
    "hodlr_get_lowrank": (_I, [_H, _I, _PD, _PD]),
    "hodlr_get_block_margin": (_I, [_H, _I, _PD, _PI]),
    "hodlr_get_aca_stats": (_I, [_H, _PI, _PD, _PD]),
    "hodlr_kernel_matvec_noalloc": (_I, [_I, _I, _V, ctypes.POINTER(KernelDesc), _I, _V, _I, _V,
                                         _I, _V]),
    "hodlr_status_string": (ctypes.c_char_p, [_I]),
    "hodlr_last_error": (ctypes.c_char_p, [_H]),
}

_LIB = None


def lib():
    """Load the CUDA library; raise if it has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                "libhodlr_b200.so is missing: build it with `python -m dense_hodlr_b200.build` "
                "(the solver has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB
