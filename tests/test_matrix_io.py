"""Dense-matrix files in the reference's binary format (include/matrixIO.hpp:
38-53, src/matrixIO.cpp:159-202): int32 rows, int32 cols, then the values row
by row.  CPU tests of the C ABI's host-only file calls, of the numpy module,
and of include/matrixIO.hpp compiled with g++; the dense GPU path through a
file is in tests/test_gpu_parity.py."""
import ctypes
import os
import struct
import subprocess

import numpy as np
import pytest

from dense_hodlr_b200 import _lib
from dense_hodlr_b200.matrix_io import readBinaryIntoMatrixXd, saveMatrixXdToBinary

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_dp = ctypes.POINTER(ctypes.c_double)


def _c_read(lib, path):
    r, c = ctypes.c_int(), ctypes.c_int()
    st = lib.hodlr_matrix_file_dims(str(path).encode(), ctypes.byref(r), ctypes.byref(c))
    if st:
        return st, None
    a = np.zeros((r.value, c.value), order="F")
    st = lib.hodlr_read_matrix_file(str(path).encode(), r.value, c.value,
                                    a.ctypes.data_as(_dp), max(r.value, 1))
    return st, a


def test_byte_layout_matches_the_reference_format(gpu_lib, tmp_path):
    """The bytes are exactly: two native int32, then row-major doubles."""
    a = np.arange(12, dtype=np.float64).reshape(3, 4) * 0.5 - 1.0
    want = struct.pack("=ii", 3, 4) + struct.pack("=12d", *a.ravel(order="C"))
    pc, pn = tmp_path / "c.bin", tmp_path / "n.bin"
    af = np.asfortranarray(a)
    assert gpu_lib.hodlr_write_matrix_file(str(pc).encode(), 3, 4, af.ctypes.data_as(_dp), 3) == 0
    saveMatrixXdToBinary(a, pn)
    assert pc.read_bytes() == want
    assert pn.read_bytes() == want


def test_read_hand_made_file_and_leading_dimension(gpu_lib, tmp_path):
    rng = np.random.default_rng(3)
    a = rng.standard_normal((5, 7))
    p = tmp_path / "m.bin"
    p.write_bytes(struct.pack("=ii", 5, 7) + a.tobytes(order="C"))
    st, got = _c_read(gpu_lib, p)
    assert st == 0 and np.array_equal(got, a)
    assert np.array_equal(readBinaryIntoMatrixXd(p), a)
    # column-major with lda > rows: the padding rows stay untouched
    buf = np.full((8, 7), 99.0, order="F")
    assert gpu_lib.hodlr_read_matrix_file(str(p).encode(), 5, 7, buf.ctypes.data_as(_dp), 8) == 0
    assert np.array_equal(buf[:5], a) and np.all(buf[5:] == 99.0)


def test_round_trip_between_implementations(gpu_lib, tmp_path):
    a = np.random.default_rng(4).standard_normal((33, 17))
    p = tmp_path / "r.bin"
    saveMatrixXdToBinary(a, p)
    st, got = _c_read(gpu_lib, p)
    assert st == 0 and np.array_equal(got, a)
    q = tmp_path / "s.bin"
    assert gpu_lib.hodlr_write_matrix_file(str(q).encode(), 33, 17,
                                           got.ctypes.data_as(_dp), 33) == 0
    assert np.array_equal(readBinaryIntoMatrixXd(q), a)
    e = np.zeros((0, 3))  # empty matrices round-trip too
    saveMatrixXdToBinary(e, tmp_path / "e.bin")
    assert readBinaryIntoMatrixXd(tmp_path / "e.bin").shape == (0, 3)


def test_errors(gpu_lib, tmp_path):
    missing = str(tmp_path / "none.bin").encode()
    r, c = ctypes.c_int(), ctypes.c_int()
    assert gpu_lib.hodlr_matrix_file_dims(missing, ctypes.byref(r), ctypes.byref(c)) == _lib.ERR_IO
    short = tmp_path / "short.bin"
    short.write_bytes(struct.pack("=ii", 4, 4) + struct.pack("=5d", *range(5)))
    buf = np.zeros((4, 4), order="F")
    assert gpu_lib.hodlr_read_matrix_file(str(short).encode(), 4, 4,
                                          buf.ctypes.data_as(_dp), 4) == _lib.ERR_IO
    assert gpu_lib.hodlr_read_matrix_file(str(short).encode(), 3, 4,
                                          buf.ctypes.data_as(_dp), 4) == _lib.ERR_ARG
    assert gpu_lib.hodlr_read_matrix_file(str(short).encode(), 4, 4,
                                          buf.ctypes.data_as(_dp), 3) == _lib.ERR_ARG
    neg = tmp_path / "neg.bin"
    neg.write_bytes(struct.pack("=ii", -1, 4))
    assert gpu_lib.hodlr_matrix_file_dims(str(neg).encode(), ctypes.byref(r),
                                          ctypes.byref(c)) == _lib.ERR_IO
    assert gpu_lib.hodlr_write_matrix_file(str(tmp_path / "no" / "dir.bin").encode(), 1, 1,
                                           buf.ctypes.data_as(_dp), 1) == _lib.ERR_IO
    assert _lib.status_string(_lib.ERR_IO) == "file could not be read or written"
    with pytest.raises(OSError):
        readBinaryIntoMatrixXd(short)
    with pytest.raises(OSError):
        readBinaryIntoMatrixXd(tmp_path / "none.bin")


def test_cpp_header_round_trip(gpu_lib, tmp_path):
    """include/matrixIO.hpp with the reference's function names, built with g++;
    a file it cannot open throws hodlr_b200::Error with HODLR_ERR_IO."""
    src = tmp_path / "io.cpp"
    src.write_text(r'''
#include <cstdio>
#include "matrixIO.hpp"
int main(int argc, char** argv) {
  hodlr_b200::Matrix a(3, 2);
  for (int j = 0; j < 2; ++j)
    for (int i = 0; i < 3; ++i) a(i, j) = 10 * i + j + 0.25;
  std::string p = std::string(argv[1]) + "/cpp.bin";
  saveMatrixXdToBinary(a, p);
  hodlr_b200::Matrix b = readBinaryIntoMatrixXd(p);
  int bad = b.rows() != 3 || b.cols() != 2;
  for (int j = 0; j < 2 && !bad; ++j)
    for (int i = 0; i < 3; ++i) bad |= b(i, j) != a(i, j);
  try {
    readBinaryIntoMatrixXd(std::string(argv[1]) + "/missing.bin");
    bad = 1;
  } catch (const hodlr_b200::Error& e) {
    bad |= e.status() != HODLR_ERR_IO;
  }
  std::printf(bad ? "FAIL\n" : "ok\n");
  return bad;
}
''')
    exe = tmp_path / "io"
    subprocess.run(["g++", "-O1", "-std=c++17", str(src), "-I", os.path.join(ROOT, "include"),
                    "-L", os.path.join(ROOT, "dense_hodlr_b200"), "-lhodlr_b200",
                    "-Wl,-rpath," + os.path.join(ROOT, "dense_hodlr_b200"), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stdout + out.stderr
    want = struct.pack("=ii", 3, 2) + struct.pack("=6d", 0.25, 1.25, 10.25, 11.25, 20.25, 21.25)
    assert (tmp_path / "cpp.bin").read_bytes() == want
