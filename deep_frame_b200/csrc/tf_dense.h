// Dense FP64 helpers for the coarsest multigrid level.
#pragma once
#include <cstddef>
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
}  // namespace tfb
