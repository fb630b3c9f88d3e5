// matrixIO.hpp -- the dense-matrix binary files of amiraa127/Dense_HODLR
// (include/matrixIO.hpp:38-53: saveMatrixXdToBinary, readBinaryIntoMatrixXd),
// header-only over the host-only file functions of libhodlr_b200.so.
//
// Format (src/matrixIO.cpp:159-202): two native int32 (rows, cols), then the
// rows x cols FP64 values row by row.  Same names and arguments as the
// reference; with Eigen on the include path readBinaryIntoMatrixXd returns
// Eigen::MatrixXd, otherwise hodlr_b200::Matrix.  Where the reference prints
// and calls exit(EXIT_FAILURE) (a file it cannot open), these throw
// hodlr_b200::Error; a short file, which the reference reads into
// uninitialised values, throws as well.
#ifndef HODLR_B200_MATRIX_IO_HPP
#define HODLR_B200_MATRIX_IO_HPP

#include <string>

#include "HODLR_Matrix.hpp"

namespace hodlr_b200 {

inline Matrix read_matrix_file(const std::string& path) {
  int rows = 0, cols = 0;
  check(nullptr, hodlr_matrix_file_dims(path.c_str(), &rows, &cols), ("readBinaryIntoMatrixXd " + path).c_str());
  Matrix m(rows, cols);
  check(nullptr, hodlr_read_matrix_file(path.c_str(), rows, cols, m.data(), rows > 0 ? rows : 1),
        ("readBinaryIntoMatrixXd " + path).c_str());
  return m;
}

}  // namespace hodlr_b200

inline void saveMatrixXdToBinary(const hodlr_b200::Matrix& inputMatrix,
                                 const std::string outputFileName) {
  hodlr_b200::check(nullptr,
                    hodlr_write_matrix_file(outputFileName.c_str(), inputMatrix.rows(),
                                            inputMatrix.cols(), inputMatrix.data(),
                                            inputMatrix.rows() > 0 ? inputMatrix.rows() : 1),
                    ("saveMatrixXdToBinary " + outputFileName).c_str());
}

#ifdef HODLR_B200_HAVE_EIGEN
inline void saveMatrixXdToBinary(const Eigen::MatrixXd& inputMatrix,
                                 const std::string outputFileName) {
  const int rows = (int)inputMatrix.rows();
  hodlr_b200::check(nullptr,
                    hodlr_write_matrix_file(outputFileName.c_str(), rows, (int)inputMatrix.cols(),
                                            inputMatrix.data(), rows > 0 ? rows : 1),
                    ("saveMatrixXdToBinary " + outputFileName).c_str());
}

inline Eigen::MatrixXd readBinaryIntoMatrixXd(const std::string inputFileName) {
  int rows = 0, cols = 0;
  hodlr_b200::check(nullptr, hodlr_matrix_file_dims(inputFileName.c_str(), &rows, &cols),
                    ("readBinaryIntoMatrixXd " + inputFileName).c_str());
  Eigen::MatrixXd m(rows, cols);
  hodlr_b200::check(nullptr,
                    hodlr_read_matrix_file(inputFileName.c_str(), rows, cols, m.data(),
                                           rows > 0 ? rows : 1),
                    ("readBinaryIntoMatrixXd " + inputFileName).c_str());
  return m;
}
#else
inline hodlr_b200::Matrix readBinaryIntoMatrixXd(const std::string inputFileName) {
  return hodlr_b200::read_matrix_file(inputFileName);
}
#endif

#endif  // HODLR_B200_MATRIX_IO_HPP
