// Dense FP64 helpers for the coarsest multigrid level.
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

namespace tfb {
// A (n x n, row-major) <- (A + A^T) / 2
void dense_symmetrize(double* A, int n, cudaStream_t s);
// In-place lower Cholesky factor of the SPD matrix A; *info_dev gets 1 + the first non-positive pivot.
void dense_cholesky(double* A, int n, int* info_dev, cudaStream_t s);
// X = L^-1 for the lower-triangular factor L (X is lower triangular, upper part zero).
void dense_trinv(const double* L, double* X, int n, cudaStream_t s);
// C = op(X) B with X lower triangular, B and C stored as [ncol][n]; op = X or X^T.
// work: dense_trimul_work(n, ncol) bytes of split-K partials.
void dense_trimul(const double* X, const double* B, double* C, int n, int ncol, int transpose, const int* active, double* work,
                  cudaStream_t s);
size_t dense_trimul_work(int n, int ncol);
}  // namespace tfb
