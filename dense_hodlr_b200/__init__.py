"""B200-native HODLR direct solver: kernel-matrix assembly, partial-pivot ACA,
recursive LU / Sherman-Morrison-Woodbury factorization and solve, as
hand-written sm_100a CUDA behind the C ABI in include/hodlr_b200.h."""
from .hodlr import (EXPONENTIAL, GAUSSIAN, INV_MULTIQUADRIC, MATERN32, QUADRATIC,  # noqa: F401
                    HODLR_Matrix, HODLRError, KernelSpec, kernelMatrix)
from .matrix_io import readBinaryIntoMatrixXd, saveMatrixXdToBinary  # noqa: F401,E402
