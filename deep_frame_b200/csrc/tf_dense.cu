// Dense FP64 kernels for the coarsest multigrid level (sm_100a).
//
// The reference factors its coarsest Galerkin matrix with cuDSS (sparse FP64
// Cholesky, deep_frame/topology_multigrid.py:230-283).  Here the coarsest grid
// is kept small (a few thousand dofs), factored once per hierarchy by a blocked
// right-looking Cholesky, and the factor is inverted (X = L^-1).  Every
// coarsest solve in a V-cycle is then two triangular matrix products,
// x = X^T (X b), one launch each, instead of 2 * n / NB dependent substitution
// steps.
#include "tf_common.h"
#include "tf_dense.h"

namespace tfb {

namespace {
constexpr int NB = 32;     // panel width
constexpr int TILE = 64;   // syrk / product tile

// Factor the NB x NB diagonal block at (k0, k0) in place (lower).
__global__ void potrf_diag_kernel(double* A, int n, int k0, int* info) {
  __shared__ double s[NB][NB + 1];
  const int nb = min(NB, n - k0);
  for (int t = threadIdx.x; t < nb * nb; t += blockDim.x) {
    const int r = t / nb, c = t % nb;
    s[r][c] = A[(long long)(k0 + r) * n + k0 + c];
  }
  __syncthreads();
  for (int k = 0; k < nb; ++k) {
    if (threadIdx.x == 0) {
      const double d = s[k][k];
      if (!(d > 0.0)) {
        if (*info == 0) *info = k0 + k + 1;
        s[k][k] = 1.0;
      } else {
        s[k][k] = sqrt(d);
      }
    }
    __syncthreads();
    for (int r = k + 1 + threadIdx.x; r < nb; r += blockDim.x) s[r][k] /= s[k][k];
    __syncthreads();
    for (int t = threadIdx.x; t < nb * nb; t += blockDim.x) {
      const int r = t / nb, c = t % nb;
      if (r > k && c > k && c <= r) s[r][c] -= s[r][k] * s[c][k];
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < nb * nb; t += blockDim.x) {
    const int r = t / nb, c = t % nb;
    A[(long long)(k0 + r) * n + k0 + c] = (c <= r) ? s[r][c] : 0.0;
  }
}

// Rows below the diagonal block: A[i, k0:k0+nb] <- A[i, k0:k0+nb] L_kk^-T.
__global__ void trsm_panel_kernel(double* A, int n, int k0) {
  __shared__ double L[NB][NB + 1];
  const int nb = min(NB, n - k0);
  for (int t = threadIdx.x; t < nb * nb; t += blockDim.x) {
    const int r = t / nb, c = t % nb;
    L[r][c] = A[(long long)(k0 + r) * n + k0 + c];
  }
  __syncthreads();
  for (int i = k0 + nb + blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double x[NB];
    double* row = A + (long long)i * n + k0;
#pragma unroll
    for (int c = 0; c < NB; ++c) x[c] = (c < nb) ? row[c] : 0.0;
#pragma unroll
    for (int c = 0; c < NB; ++c) {
      if (c < nb) {
        double v = x[c];
#pragma unroll
        for (int t = 0; t < NB; ++t)
          if (t < c) v -= x[t] * L[c][t];
        x[c] = v / L[c][c];
      }
    }
#pragma unroll
    for (int c = 0; c < NB; ++c)
      if (c < nb) row[c] = x[c];
  }
}

// Trailing update of the lower triangle: A[i][j] -= sum_t P[i][t] P[j][t], i >= j >= k0 + nb.
__global__ void __launch_bounds__(256) syrk_update_kernel(double* A, int n, int k0) {
  const int nb = min(NB, n - k0);
  const int start = k0 + nb;
  const int m = n - start;
  const int tiles = (m + TILE - 1) / TILE;
  // map blockIdx.x to a lower-triangular tile pair (ti >= tj)
  int b = blockIdx.x, ti = 0;
  while (b >= ti + 1) { b -= ti + 1; ++ti; }
  const int tj = b;
  if (ti >= tiles) return;
  __shared__ double Pi[TILE][NB + 1];
  __shared__ double Pj[TILE][NB + 1];
  const int i0 = start + ti * TILE, j0 = start + tj * TILE;
  for (int t = threadIdx.x; t < TILE * NB; t += blockDim.x) {
    const int r = t / NB, c = t % NB;
    Pi[r][c] = (i0 + r < n && c < nb) ? A[(long long)(i0 + r) * n + k0 + c] : 0.0;
    Pj[r][c] = (j0 + r < n && c < nb) ? A[(long long)(j0 + r) * n + k0 + c] : 0.0;
  }
  __syncthreads();
  const int tr = (threadIdx.x / 16) * 4, tc = (threadIdx.x % 16) * 4;
  double acc[4][4] = {};
  for (int t = 0; t < NB; ++t) {
    double a[4], bb[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) { a[q] = Pi[tr + q][t]; bb[q] = Pj[tc + q][t]; }
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[p][q] += a[p] * bb[q];
  }
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int i = i0 + tr + p;
    if (i >= n) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int j = j0 + tc + q;
      if (j >= n || j > i) continue;
      A[(long long)i * n + j] -= acc[p][q];
    }
  }
}

// Invert every NB x NB lower-triangular diagonal block of L into X.
__global__ void trinv_diag_kernel(const double* L, double* X, int n) {
  __shared__ double s[NB][NB + 1];
  __shared__ double x[NB][NB + 1];
  const int k0 = blockIdx.x * NB;
  const int nb = min(NB, n - k0);
  for (int t = threadIdx.x; t < NB * NB; t += blockDim.x) {
    const int r = t / NB, c = t % NB;
    s[r][c] = (r < nb && c < nb) ? L[(long long)(k0 + r) * n + k0 + c] : 0.0;
  }
  __syncthreads();
  // column c of the inverse by forward substitution (one thread per column)
  for (int c = threadIdx.x; c < nb; c += blockDim.x) {
    for (int r = 0; r < nb; ++r) {
      double v = (r == c) ? 1.0 : 0.0;
      for (int t = c; t < r; ++t) v -= s[r][t] * x[t][c];
      x[r][c] = (r < c) ? 0.0 : v / s[r][r];
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nb * nb; t += blockDim.x) {
    const int r = t / nb, c = t % nb;
    X[(long long)(k0 + r) * n + k0 + c] = x[r][c];
  }
}

// Block row bi of X = L^-1:  X[bi][bj] = -X[bi][bi] * sum_{bk=bj}^{bi-1} L[bi][bk] X[bk][bj]  (one CTA per bj < bi).
__global__ void __launch_bounds__(256) trinv_row_kernel(const double* L, double* X, int n, int bi) {
  const int bj = blockIdx.x;
  __shared__ double La[NB][NB + 1];
  __shared__ double Xb[NB][NB + 1];
  __shared__ double S[NB][NB + 1];
  const int i0 = bi * NB, j0 = bj * NB;
  const int ni = min(NB, n - i0);
  // each thread owns 4 entries of the NB x NB tile
  double acc[4] = {0, 0, 0, 0};
  for (int bk = bj; bk < bi; ++bk) {
    const int k0 = bk * NB;
    for (int t = threadIdx.x; t < NB * NB; t += blockDim.x) {
      const int r = t / NB, c = t % NB;
      La[r][c] = (r < ni) ? L[(long long)(i0 + r) * n + k0 + c] : 0.0;
      Xb[r][c] = X[(long long)(k0 + r) * n + j0 + c];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int t = threadIdx.x + q * 256;
      const int r = t / NB, c = t % NB;
      double v = 0.0;
#pragma unroll 8
      for (int kk = 0; kk < NB; ++kk) v += La[r][kk] * Xb[kk][c];
      acc[q] += v;
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int t = threadIdx.x + q * 256;
    S[t / NB][t % NB] = acc[q];
  }
  // diagonal inverse of block bi
  for (int t = threadIdx.x; t < NB * NB; t += blockDim.x) {
    const int r = t / NB, c = t % NB;
    La[r][c] = (r < ni && c < ni) ? X[(long long)(i0 + r) * n + i0 + c] : 0.0;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int t = threadIdx.x + q * 256;
    const int r = t / NB, c = t % NB;
    if (r >= ni) continue;
    double v = 0.0;
    for (int kk = 0; kk <= r; ++kk) v += La[r][kk] * S[kk][c];
    X[(long long)(i0 + r) * n + j0 + c] = -v;
  }
}

__global__ void symmetrize_kernel(double* A, int n) {
  const long long total = (long long)n * n;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int i = static_cast<int>(t / n), j = static_cast<int>(t % n);
    if (j < i) {
      const double v = 0.5 * (A[(long long)i * n + j] + A[(long long)j * n + i]);
      A[(long long)i * n + j] = v;
      A[(long long)j * n + i] = v;
    }
  }
}
}  // namespace

void dense_symmetrize(double* A, int n, cudaStream_t s) {
  symmetrize_kernel<<<grid_for((long long)n * n, 256), 256, 0, s>>>(A, n);
  TF_LAUNCH_CHECK("symmetrize_kernel");
}

void dense_cholesky(double* A, int n, int* info_dev, cudaStream_t s) {
  for (int k0 = 0; k0 < n; k0 += NB) {
    potrf_diag_kernel<<<1, 256, 0, s>>>(A, n, k0, info_dev);
    TF_LAUNCH_CHECK("potrf_diag_kernel");
    const int below = n - k0 - NB;
    if (below <= 0) break;
    trsm_panel_kernel<<<grid_for(below, 128, 4096), 128, 0, s>>>(A, n, k0);
    TF_LAUNCH_CHECK("trsm_panel_kernel");
    const int tiles = (below + TILE - 1) / TILE;
    syrk_update_kernel<<<tiles * (tiles + 1) / 2, 256, 0, s>>>(A, n, k0);
    TF_LAUNCH_CHECK("syrk_update_kernel");
  }
}

void dense_trinv(const double* L, double* X, int n, cudaStream_t s) {
  TF_CUDA_CHECK(cudaMemsetAsync(X, 0, sizeof(double) * (size_t)n * n, s));
  const int blocks = (n + NB - 1) / NB;
  trinv_diag_kernel<<<blocks, 64, 0, s>>>(L, X, n);
  TF_LAUNCH_CHECK("trinv_diag_kernel");
  for (int bi = 1; bi < blocks; ++bi) {
    trinv_row_kernel<<<bi, 256, 0, s>>>(L, X, n, bi);
    TF_LAUNCH_CHECK("trinv_row_kernel");
  }
}

// Split-K form of C = op(X) B: CTA (row block rb, K chunk kc, column group) multiplies 32 rows of op(X)
// restricted to K chunk kc (256 wide) with up to 48 columns of B and stores the partial tile; chunks
// that lie entirely in the zero triangle of op(X) are skipped.  trimul_sum_kernel adds the partials of
// every row in chunk order (deterministic) into C.  Balanced over 148 SMs for the coarsest sizes
// (a few thousand unknowns), where a whole-K row tile would leave most SMs idle.
constexpr int TM_RB = 32, TM_KCH = 256, TM_KS = 32, TM_CW = 48;

__device__ __forceinline__ bool trimul_chunk_live(int i0, int kc, int transpose) {
  return transpose ? (kc + 1) * TM_KCH - 1 >= i0 : kc * TM_KCH <= i0 + TM_RB - 1;
}

__global__ void __launch_bounds__(256) trimul_split_kernel(const double* __restrict__ X, const double* __restrict__ B,
                                                           double* __restrict__ P, int n, int ncol, int transpose) {
  __shared__ double Xs[TM_RB][TM_KS + 1];
  __shared__ double Bs[TM_CW][TM_KS + 1];
  const int i0 = blockIdx.x * TM_RB, kc = blockIdx.y, c0 = blockIdx.z * TM_CW;
  if (!trimul_chunk_live(i0, kc, transpose)) return;
  const int t = threadIdx.x, r = t % TM_RB, cg = t / TM_RB;   // 8 column groups of 6
  const int k_lo = kc * TM_KCH, k_hi = min(n, k_lo + TM_KCH);
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int k0 = k_lo; k0 < k_hi; k0 += TM_KS) {
    for (int e = t; e < TM_RB * TM_KS; e += 256) {
      // contiguous global reads: k fastest for X rows, row fastest for X^T
      const int rr = transpose ? e % TM_RB : e / TM_KS, kk = transpose ? e / TM_RB : e % TM_KS;
      const int i = i0 + rr, k = k0 + kk;
      double v = 0.0;
      if (i < n && k < k_hi) v = transpose ? X[(long long)k * n + i] : X[(long long)i * n + k];
      Xs[rr][kk] = v;
    }
    for (int e = t; e < TM_CW * TM_KS; e += 256) {
      const int cc = e / TM_KS, kk = e % TM_KS, col = c0 + cc, k = k0 + kk;
      Bs[cc][kk] = (col < ncol && k < k_hi) ? B[(long long)col * n + k] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < TM_KS; ++kk) {
      const double a = Xs[r][kk];
#pragma unroll
      for (int q = 0; q < 6; ++q) acc[q] = fma(a, Bs[cg * 6 + q][kk], acc[q]);
    }
    __syncthreads();
  }
  const int i = i0 + r;
  if (i >= n) return;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const int col = c0 + cg * 6 + q;
    if (col < ncol) P[((long long)kc * ncol + col) * n + i] = acc[q];
  }
}

__global__ void trimul_sum_kernel(const double* __restrict__ P, double* __restrict__ C, int n, int ncol, int nchunks, int transpose,
                                  const int* __restrict__ active) {
  const long long total = (long long)n * ncol;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
    const int col = static_cast<int>(idx / n), i = static_cast<int>(idx % n);
    if (active && !active[col]) continue;
    const int i0 = (i / TM_RB) * TM_RB;
    double s = 0.0;
    for (int kc = 0; kc < nchunks; ++kc)
      if (trimul_chunk_live(i0, kc, transpose)) s += P[((long long)kc * ncol + col) * n + i];
    C[(long long)col * n + i] = s;
  }
}

size_t dense_trimul_work(int n, int ncol) {
  return sizeof(double) * (size_t)((n + TM_KCH - 1) / TM_KCH) * ncol * (size_t)n;
}

void dense_trimul(const double* X, const double* B, double* C, int n, int ncol, int transpose, const int* active, double* work,
                  cudaStream_t s) {
  const int nchunks = (n + TM_KCH - 1) / TM_KCH;
  dim3 grid((n + TM_RB - 1) / TM_RB, nchunks, (ncol + TM_CW - 1) / TM_CW);
  trimul_split_kernel<<<grid, 256, 0, s>>>(X, B, work, n, ncol, transpose);
  TF_LAUNCH_CHECK("trimul_split_kernel");
  trimul_sum_kernel<<<grid_for((long long)n * ncol, 256), 256, 0, s>>>(work, C, n, ncol, nchunks, transpose, active);
  TF_LAUNCH_CHECK("trimul_sum_kernel");
}

}  // namespace tfb

// ---------------------------------------------------------------------------
// Dense FP64 direct solver of a small sparse SPD system (the drop-in for the
// reference's CudaDirectSolver, deep_frame/topology_optimization.py:80-244):
// the CSR matrix is scattered into a dense n x n array, symmetrised, factored
// (A = L L^T), and L is inverted once; each solve is x = L^-T (L^-1 b).
// ---------------------------------------------------------------------------
#include <algorithm>
#include <string>
#include "tf_b200.h"

namespace {
__global__ void csr_to_dense_kernel(int n, const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                                    const double* __restrict__ data, double* __restrict__ A) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double* row = A + (long long)i * n;
    for (int k = indptr[i]; k < indptr[i + 1]; ++k) {
      const int j = indices[k];
      if ((unsigned)j < (unsigned)n) row[j] = data[k];
    }
  }
}
}  // namespace

struct tf_chol {
  int n = 0;
  tfb::DevBuf A, X, tmp, info, work;
  bool factored = false;
  std::string err;
};

namespace {
template <typename F>
int chol_guard(tf_chol* h, F&& f) {
  try {
    f();
    return tfb::TF_OK;
  } catch (const tfb::Error& e) {
    if (h) h->err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    if (h) h->err = e.what();
    return tfb::TF_INTERNAL;
  }
}
constexpr int64_t CHOL_MAX_N = 32768;
}  // namespace

extern "C" int tf_chol_create(int64_t n, tf_chol** out) {
  if (!out) return tfb::TF_INVALID;
  *out = nullptr;
  tf_chol* h = new tf_chol();
  const int rc = chol_guard(h, [&] {
    tfb::require(n >= 1 && n <= CHOL_MAX_N, "the dense direct solver handles 1 to 32768 unknowns");
    h->n = static_cast<int>(n);
    h->A.alloc(sizeof(double) * n * n);
    h->X.alloc(sizeof(double) * n * n);
    h->info.alloc(sizeof(int));
  });
  if (rc != tfb::TF_OK) {
    tfb::record_unhandled_error(h->err);
    delete h;
    return rc;
  }
  *out = h;
  return tfb::TF_OK;
}

extern "C" int tf_chol_factor_csr(tf_chol* h, const int32_t* indptr_dev, const int32_t* indices_dev, const double* data_dev,
                                  void* stream) {
  if (!h) return tfb::TF_INVALID;
  return chol_guard(h, [&] {
    tfb::require(indptr_dev && indices_dev && data_dev, "tf_chol_factor_csr: NULL argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int n = h->n;
    h->factored = false;
    TF_CUDA_CHECK(cudaMemsetAsync(h->A.p, 0, h->A.bytes, s));
    csr_to_dense_kernel<<<tfb::grid_for(n, 128), 128, 0, s>>>(n, indptr_dev, indices_dev, data_dev, h->A.as<double>());
    TF_LAUNCH_CHECK("csr_to_dense_kernel");
    tfb::dense_symmetrize(h->A.as<double>(), n, s);
    TF_CUDA_CHECK(cudaMemsetAsync(h->info.p, 0, sizeof(int), s));
    tfb::dense_cholesky(h->A.as<double>(), n, h->info.as<int>(), s);
    int info = 0;
    TF_CUDA_CHECK(cudaMemcpyAsync(&info, h->info.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    TF_CUDA_CHECK(cudaStreamSynchronize(s));
    if (info != 0) throw tfb::Error(tfb::TF_NUMERIC, "matrix is not positive definite (pivot " + std::to_string(info) + ")");
    tfb::dense_trinv(h->A.as<double>(), h->X.as<double>(), n, s);
    h->factored = true;
  });
}

extern "C" int tf_chol_solve(tf_chol* h, const double* b_dev, int32_t nrhs, double* x_dev, void* stream) {
  if (!h) return tfb::TF_INVALID;
  return chol_guard(h, [&] {
    tfb::require(h->factored, "tf_chol_solve: no factorisation (call tf_chol_factor_csr first)");
    tfb::require(nrhs >= 1 && b_dev && x_dev, "tf_chol_solve: invalid right-hand sides");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t need = sizeof(double) * (size_t)h->n * nrhs;
    if (h->tmp.bytes < need) h->tmp.alloc(need);
    h->work.ensure(std::max(h->work.bytes, tfb::dense_trimul_work(h->n, nrhs)));
    tfb::dense_trimul(h->X.as<double>(), b_dev, h->tmp.as<double>(), h->n, nrhs, 0, nullptr, h->work.as<double>(), s);
    tfb::dense_trimul(h->X.as<double>(), h->tmp.as<double>(), x_dev, h->n, nrhs, 1, nullptr, h->work.as<double>(), s);
  });
}

extern "C" int tf_chol_destroy(tf_chol* h) {
  if (h) {
    cudaDeviceSynchronize();
    delete h;
  }
  return tfb::TF_OK;
}

extern "C" const char* tf_chol_last_error(const tf_chol* h) { return h ? h->err.c_str() : ""; }
