"""Dense-matrix files in the reference's binary format (include/matrixIO.hpp:
38-53, src/matrixIO.cpp:159-202): two native int32 (rows, cols), then the
rows x cols FP64 values row by row.  Same names as the reference
(saveMatrixXdToBinary, readBinaryIntoMatrixXd), plus snake_case aliases.
Pure numpy, no GPU; a missing or short file raises OSError."""
import numpy as np


def readBinaryIntoMatrixXd(inputFileName):
    """The matrix stored in inputFileName, as a float64 (rows, cols) array."""
    with open(inputFileName, "rb") as f:
        hdr = np.fromfile(f, dtype=np.int32, count=2)
        if hdr.size != 2 or hdr[0] < 0 or hdr[1] < 0:
            raise OSError(f"{inputFileName}: not a dense-matrix file (bad header)")
        rows, cols = int(hdr[0]), int(hdr[1])
        vals = np.fromfile(f, dtype=np.float64, count=rows * cols)
    if vals.size != rows * cols:
        raise OSError(f"{inputFileName}: short file ({vals.size} of {rows * cols} values)")
    return vals.reshape(rows, cols)


def saveMatrixXdToBinary(inputMatrix, outputFileName):
    """Write a 2-D array (any layout) to outputFileName."""
    a = np.asarray(inputMatrix, dtype=np.float64)
    if a.ndim != 2:
        raise ValueError("a 2-D matrix is required")
    with open(outputFileName, "wb") as f:
        np.array(a.shape, dtype=np.int32).tofile(f)
        np.ascontiguousarray(a).tofile(f)


read_binary = readBinaryIntoMatrixXd
save_binary = saveMatrixXdToBinary
