// Dense FP64 helpers for the coarsest multigrid level.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace tfb {
// A (n x n, row-major) <- (A + A^T) / 2
void dense_symmetrize(double* A, int n, cudaStream_t s);
// X = L^-1 for the lower Cholesky factor L of the SPD matrix A (X lower triangular, upper part
// zero); A is overwritten, *info_dev gets 1 + the first non-positive pivot (set while it is 0).
// work: dense_factor_work(n) bytes (the inverted 32 x 32 diagonal blocks).
void dense_cholesky_inverse(double* A, double* X, int n, int* info_dev, double* work, cudaStream_t s);
size_t dense_factor_work(int n);
// C = op(X) B with X lower triangular, B and C stored as [ncol][n]; op = X or X^T.
// work: dense_trimul_work(n, ncol) bytes of split-K partials.
void dense_trimul(const double* X, const double* B, double* C, int n, int ncol, int transpose, const int* active, double* work,
                  cudaStream_t s);
size_t dense_trimul_work(int n, int ncol);
// dense_trimul of several independent systems, one launch per stage for all of them
struct TrimulJob {
  const double* X;
  const double* B;
  double* C;
  double* work;
  int n, ncol;
  const int* active;
};
void dense_trimul_batch(const TrimulJob* jobs, int count, int transpose, cudaStream_t s);

// Banded FP64 Cholesky (tf_band.cu).  Band storage AB[j * (bw + 1) + d] = A[j + d][j], 0 <= d <= bw.
// bandwidth of a CSR matrix (max |i - j| over its entries); scratch_dev holds one int
int band_width(int n, const int32_t* indptr, const int32_t* indices, int* scratch_dev, cudaStream_t s);
// AB <- the band of (A + A^T) / 2
void band_assemble(int n, const int32_t* indptr, const int32_t* indices, const double* data, int bw, double* AB, cudaStream_t s);
// AB <- L (A = L L^T) in place; *info_dev = 1 + the first non-positive pivot's column (0 on success)
void band_cholesky(double* AB, int n, int bw, int* info_dev, cudaStream_t s);
// x = A^-1 b for nrhs columns stored [nrhs][n]
void band_solve(const double* AB, int n, int bw, const double* b, double* x, int nrhs, cudaStream_t s);
}  // namespace tfb
