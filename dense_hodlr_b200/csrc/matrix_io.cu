// Dense-matrix files in the reference's binary format (saveMatrixXdToBinary /
// readBinaryIntoMatrixXd, src/matrixIO.cpp:159-202): two native 32-bit ints
// (rows, cols), then the rows x cols FP64 values row by row.  Host code only:
// these entries need no GPU.  Where the reference reads a short file into
// uninitialised values, these calls report HODLR_ERR_IO.
#include <stdint.h>
#include <stdio.h>

#include <vector>

#include "../../include/hodlr_b200.h"

namespace {

struct File {
  FILE* f;
  explicit File(FILE* p) : f(p) {}
  ~File() {
    if (f) fclose(f);
  }
};

int read_header(FILE* f, int* rows, int* cols) {
  int32_t hdr[2];
  if (fread(hdr, sizeof(int32_t), 2, f) != 2 || hdr[0] < 0 || hdr[1] < 0) return HODLR_ERR_IO;
  *rows = hdr[0];
  *cols = hdr[1];
  return HODLR_OK;
}

}  // namespace

extern "C" {

int hodlr_matrix_file_dims(const char* path, int* rows, int* cols) {
  if (!path || !rows || !cols) return HODLR_ERR_ARG;
  File in(fopen(path, "rb"));
  if (!in.f) return HODLR_ERR_IO;
  return read_header(in.f, rows, cols);
}

int hodlr_read_matrix_file(const char* path, int rows, int cols, double* A, int lda) {
  if (!path || rows < 0 || cols < 0 || (rows > 0 && cols > 0 && !A) || lda < (rows > 0 ? rows : 1))
    return HODLR_ERR_ARG;
  File in(fopen(path, "rb"));
  if (!in.f) return HODLR_ERR_IO;
  int fr = 0, fc = 0;
  int rc = read_header(in.f, &fr, &fc);
  if (rc) return rc;
  if (fr != rows || fc != cols) return HODLR_ERR_ARG;
  std::vector<double> row((size_t)cols);
  for (int i = 0; i < rows; ++i) {
    if (fread(row.data(), sizeof(double), (size_t)cols, in.f) != (size_t)cols) return HODLR_ERR_IO;
    for (int j = 0; j < cols; ++j) A[(int64_t)j * lda + i] = row[j];
  }
  return HODLR_OK;
}

int hodlr_write_matrix_file(const char* path, int rows, int cols, const double* A, int lda) {
  if (!path || rows < 0 || cols < 0 || (rows > 0 && cols > 0 && !A) || lda < (rows > 0 ? rows : 1))
    return HODLR_ERR_ARG;
  File out(fopen(path, "wb"));
  if (!out.f) return HODLR_ERR_IO;
  const int32_t hdr[2] = {rows, cols};
  if (fwrite(hdr, sizeof(int32_t), 2, out.f) != 2) return HODLR_ERR_IO;
  std::vector<double> row((size_t)cols);
  for (int i = 0; i < rows; ++i) {
    for (int j = 0; j < cols; ++j) row[j] = A[(int64_t)j * lda + i];
    if (fwrite(row.data(), sizeof(double), (size_t)cols, out.f) != (size_t)cols) return HODLR_ERR_IO;
  }
  if (fflush(out.f) != 0) return HODLR_ERR_IO;
  return HODLR_OK;
}

}  // extern "C"
