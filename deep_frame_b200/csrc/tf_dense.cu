// Dense FP64 kernels for the coarsest multigrid level (sm_100a).
//
// The reference factors its coarsest Galerkin matrix with cuDSS (sparse FP64
// Cholesky, deep_frame/topology_multigrid.py:230-283).  Here the coarsest grid
// is kept small (a few thousand dofs) and, once per hierarchy, a blocked
// right-looking Cholesky and the inversion of its factor (X = L^-1) run
// together, two launches per 32-wide panel.  Every coarsest solve in a V-cycle
// is then two triangular matrix products, x = X^T (X b), instead of 2 * n / 32
// dependent substitution steps.
#include "tf_common.h"
#include "tf_dense.h"
#include "tf_batch.cuh"
#include "tf_reduce.cuh"

namespace tfb {

namespace {
// Blocked Cholesky factorisation fused with the inversion of its factor, one launch per 32-wide
// panel.  Launch k (panel rows / columns k0 = 32 k .. k0 + 31) reads Linv_kk, the inverse of the
// factor of the diagonal block W_kk = L_kk L_kk^T, from `work` and runs three kinds of CTA:
//  * trailing tiles (ti >= tj, 64 x 64): L_i = W_ik Linv_kk^T for the tile's two row ranges, then
//    W_ij -= L_i L_j^T (the Schur complement; W is the input matrix and is overwritten).  Tile
//    (0, 0) holds the next diagonal block, final after this update, so that CTA then factors and
//    inverts it for launch k + 1 while the other tiles run (look-ahead);
//  * inverse tiles (a row tile below the panel x 64 columns j < k0 + 32): X_k = Linv_kk R_k for
//    those columns, then R_ij -= L_i X_k.  R lives in the output buffer X; it starts as the identity
//    and, when panel k runs, block row k of R is the right-hand side of L_kk X_k = R_k;
//  * finishing tiles: block row k - 1 of R is complete after panel k - 1 and is replaced in place by
//    X_{k-1} = Linv_{k-1} R_{k-1}.
// The three kinds read and write disjoint parts of W, X and `work`, so a launch needs no other
// synchronisation.  A one-CTA launch factors block 0 first; a last launch finishes the last block
// row.  L itself is never stored: the coarsest solve only uses X = L^-1 (x = X^T X b).
constexpr int FB = 32;       // panel width
constexpr int FT = 64;       // update tile
constexpr int FP = FT + 1;   // shared-memory pitch of the K-major operand tiles
constexpr int F_THREADS = 256;

struct DiagShared {
  double L[FB][FB + 1];    // factor of the diagonal block
  double Li[FB][FB + 1];   // its inverse
  double col[FB];          // the current column of L
  double dinv[FB];         // 1 / L_rr
};

struct FactorShared {
  double Li[FB][FB + 1];   // inverse of the diagonal factor
  double A[FB][FP];        // K-major left operand (L_i^T)
  double B[FB][FP];        // K-major right operand (L_j^T or X_k)
  double T[FB][FP];        // staging
};

// CTA counts of the update launch of panel k (the same arithmetic on host and device)
struct FactorStep {
  int trailing, syrk, ctiles, upd, lead, finish;
  __host__ __device__ FactorStep(int n, int k) {
    const int nblk = (n + FB - 1) / FB;
    const int k0 = k * FB, start = k0 + FB;
    trailing = k < nblk ? (max(0, n - start) + FT - 1) / FT : 0;
    syrk = trailing * (trailing + 1) / 2;
    ctiles = (min(start, n) + FT - 1) / FT;
    upd = trailing * ctiles;
    lead = syrk + upd;
    finish = k >= 1 ? (min(k0, n) + FT - 1) / FT : 0;
  }
};

// Factor and invert the diagonal block at (k0, k0) (rows beyond n padded with the identity) and
// store Linv in Dk; a non-positive pivot is replaced by 1 and reported as 1 + its global index in
// *info (when *info is still 0).  Called by every thread of one CTA; the elimination is one warp.
__device__ void factor_diag(const double* W, int n, int k0, DiagShared& s, double* __restrict__ Dk, int* __restrict__ info) {
  const int nb = min(FB, n - k0);
  {
    double v[FB * FB / F_THREADS];
#pragma unroll
    for (int q = 0; q < FB * FB / F_THREADS; ++q) {
      const int e = threadIdx.x + q * F_THREADS, r = e / FB, c = e % FB;
      v[q] = (r == c) ? 1.0 : 0.0;
      if (r < nb && c < nb) v[q] = (c <= r) ? W[(long long)(k0 + r) * n + k0 + c] : 0.0;
    }
#pragma unroll
    for (int q = 0; q < FB * FB / F_THREADS; ++q) {
      const int e = threadIdx.x + q * F_THREADS;
      s.L[e / FB][e % FB] = v[q];
    }
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    // Lane r holds the not yet eliminated part of row r in registers, a[j] = W_r,k+j at pivot k;
    // the row shifts left by one per pivot so that the pivot loop runs rolled: unrolled, the code
    // executes once per launch and is bound by instruction fetch.
    const int lane = threadIdx.x;
    double a[FB];
#pragma unroll
    for (int c = 0; c < FB; ++c) a[c] = s.L[lane][c];
    int bad = 0;
#pragma unroll 1
    for (int k = 0; k < FB; ++k) {
      double piv = __shfl_sync(0xffffffffu, a[0], k);
      if (!(piv > 0.0)) {
        if (bad == 0) bad = k + 1;
        piv = 1.0;
      }
      const double rs = rsqrt(piv);
      const double l = (lane == k) ? piv * rs : a[0] * rs;   // L_rk (rows above k: unused)
      if (lane == k) s.dinv[k] = rs;
      if (lane >= k) s.L[lane][k] = l;
      s.col[lane] = l;
      __syncwarp();
#pragma unroll
      for (int j = 1; j < FB; ++j) {
        const int c = k + j;
        if (c < FB && lane >= c) a[j] = fma(-l, s.col[c], a[j]);
      }
      __syncwarp();
#pragma unroll
      for (int j = 0; j + 1 < FB; ++j) a[j] = a[j + 1];
      a[FB - 1] = 0.0;
    }
    __syncwarp();
    // lane c: column c of L^-1 by right-looking forward substitution (short dependency chain),
    // v[j] = pending entry t + j, shifted the same way
    double v[FB];
#pragma unroll
    for (int r = 0; r < FB; ++r) v[r] = (r == lane) ? 1.0 : 0.0;
#pragma unroll 1
    for (int t = 0; t < FB; ++t) {
      const double x = v[0] * s.dinv[t];
      s.Li[t][lane] = x;
#pragma unroll
      for (int j = 1; j < FB; ++j) {
        const int r = t + j;
        if (r < FB) v[j] = fma(-s.L[r][t], x, v[j]);
      }
#pragma unroll
      for (int j = 0; j + 1 < FB; ++j) v[j] = v[j + 1];
      v[FB - 1] = 0.0;
    }
    if (lane == 0 && bad && *info == 0) *info = k0 + bad;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < FB * FB / F_THREADS; ++q) {
    const int e = threadIdx.x + q * F_THREADS;
    Dk[e] = s.Li[e / FB][e % FB];
  }
}

// the factor of diagonal block 0, before the first panel launch
__global__ void __launch_bounds__(F_THREADS) factor_first_kernel(const double* __restrict__ W, int n, double* __restrict__ D,
                                                                 int* __restrict__ info) {
  __shared__ DiagShared s;
  factor_diag(W, n, 0, s, D, info);
}

// s.Li <- the 32 x 32 block Dk
__device__ void load_inverse(const double* __restrict__ Dk, FactorShared& s) {
  double v[FB * FB / F_THREADS];
#pragma unroll
  for (int q = 0; q < FB * FB / F_THREADS; ++q) v[q] = Dk[threadIdx.x + q * F_THREADS];
#pragma unroll
  for (int q = 0; q < FB * FB / F_THREADS; ++q) {
    const int e = threadIdx.x + q * F_THREADS;
    s.Li[e / FB][e % FB] = v[q];
  }
}

// out = Li T (32 x 64); Li lower triangular.  The finishing and the inverse tiles both form X_k with
// this routine, so the stored X_k has the bits the updates used.
__device__ void tri_times(const double (*Li)[FB + 1], const double (*T)[FP], double (*out)[FP]) {
  const int r0 = 2 * (threadIdx.x / 16), c0 = threadIdx.x % 16;
  double acc[2][4] = {};
#pragma unroll 8
  for (int t = 0; t < FB; ++t) {
    const double l0 = Li[r0][t], l1 = Li[r0 + 1][t];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double b = T[t][c0 + 16 * q];
      acc[0][q] = fma(l0, b, acc[0][q]);
      acc[1][q] = fma(l1, b, acc[1][q]);
    }
  }
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) out[r0 + p][c0 + 16 * q] = acc[p][q];
}

// T[t][r] <- W[i0 + r][k0 + t]: 64 panel rows below the diagonal block, transposed; 0 beyond n.
__device__ void load_panel(const double* __restrict__ W, int n, int k0, int i0, double (*T)[FP]) {
  double v[FT * FB / F_THREADS];
#pragma unroll
  for (int q = 0; q < FT * FB / F_THREADS; ++q) {
    const int e = threadIdx.x + q * F_THREADS, r = e / FB, t = e % FB, i = i0 + r;
    v[q] = (i < n) ? W[(long long)i * n + k0 + t] : 0.0;
  }
#pragma unroll
  for (int q = 0; q < FT * FB / F_THREADS; ++q) {
    const int e = threadIdx.x + q * F_THREADS;
    T[e % FB][e / FB] = v[q];
  }
}

// T[t][c] <- R[k0 + t][j0 + c] for columns below col_end (0 elsewhere).  The diagonal block of R is
// the identity and is not stored: no update reaches it before its block row is finished.
__device__ void load_rows(const double* __restrict__ R, int n, int k0, int j0, int col_end, double (*T)[FP]) {
  double v[FB * FT / F_THREADS];
#pragma unroll
  for (int q = 0; q < FB * FT / F_THREADS; ++q) {
    const int e = threadIdx.x + q * F_THREADS, t = e / FT, c = e % FT, i = k0 + t, j = j0 + c;
    v[q] = 0.0;
    if (i < n && j < col_end) v[q] = (j >= k0) ? (j == i ? 1.0 : 0.0) : R[(long long)i * n + j];
  }
#pragma unroll
  for (int q = 0; q < FB * FT / F_THREADS; ++q) {
    const int e = threadIdx.x + q * F_THREADS;
    T[e / FT][e % FT] = v[q];
  }
}

// C[i0 + r][j0 + c] -= sum_t A[t][r] B[t][c] for rows below n, columns below col_end (and j <= i
// when `lower`).  The old values of C are fetched before the products so their latency overlaps.
__device__ void update_tile(double* __restrict__ C, int n, int i0, int j0, int col_end, bool lower, const double (*A)[FP],
                            const double (*B)[FP]) {
  const int rr = threadIdx.x / 16, cc = threadIdx.x % 16;
  double old[4][4];
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int i = i0 + rr + 16 * p;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int j = j0 + cc + 16 * q;
      old[p][q] = (i < n && j < col_end && (!lower || j <= i)) ? C[(long long)i * n + j] : 0.0;
    }
  }
  double acc[4][4] = {};
#pragma unroll 4
  for (int t = 0; t < FB; ++t) {
    double a[4], b[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) a[p] = A[t][rr + 16 * p];
#pragma unroll
    for (int q = 0; q < 4; ++q) b[q] = B[t][cc + 16 * q];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[p][q] = fma(a[p], b[q], acc[p][q]);
  }
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int i = i0 + rr + 16 * p;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int j = j0 + cc + 16 * q;
      if (i < n && j < col_end && (!lower || j <= i)) C[(long long)i * n + j] = old[p][q] - acc[p][q];
    }
  }
}

__global__ void __launch_bounds__(F_THREADS, 2) factor_step_kernel(double* __restrict__ W, double* __restrict__ X,
                                                                   double* __restrict__ D, int n, int k, int* __restrict__ info) {
  extern __shared__ __align__(16) unsigned char f_smem[];
  FactorShared& s = *reinterpret_cast<FactorShared*>(f_smem);
  const FactorStep st(n, k);
  const int k0 = k * FB, start = k0 + FB;
  const int b = blockIdx.x;
  if (b >= st.lead) {
    // finishing tile: X_{k-1} = Linv_{k-1} R_{k-1} for 64 columns
    const int p0 = k0 - FB, col_end = min(k0, n), j0 = (b - st.lead) * FT;
    load_inverse(D + (long long)(k - 1) * FB * FB, s);
    load_rows(X, n, p0, j0, col_end, s.T);
    __syncthreads();
    tri_times(s.Li, s.T, s.A);
    __syncthreads();
    for (int e = threadIdx.x; e < FB * FT; e += blockDim.x) {
      const int r = e / FT, c = e % FT, i = p0 + r, j = j0 + c;
      if (i < n && j < col_end) X[(long long)i * n + j] = s.A[r][c];
    }
    return;
  }
  load_inverse(D + (long long)k * FB * FB, s);
  if (b < st.syrk) {
    int ti = 0, r = b;
    while (r > ti) {
      r -= ti + 1;
      ++ti;
    }
    const int tj = r;
    const int i0 = start + ti * FT, j0 = start + tj * FT;
    load_panel(W, n, k0, i0, s.T);
    if (ti != tj) load_panel(W, n, k0, j0, s.B);
    __syncthreads();
    tri_times(s.Li, s.T, s.A);
    if (ti != tj) {
      __syncthreads();
      tri_times(s.Li, s.B, s.T);
    }
    __syncthreads();
    update_tile(W, n, i0, j0, n, ti == tj, s.A, ti == tj ? s.A : s.T);
    if (b == 0) {
      // tile (0, 0) holds diagonal block k + 1, final now: factor it for the next launch
      __syncthreads();
      factor_diag(W, n, start, *reinterpret_cast<DiagShared*>(f_smem), D + (long long)(k + 1) * FB * FB, info);
    }
  } else {
    const int u = b - st.syrk, ti = u / st.ctiles, tj = u % st.ctiles;
    const int i0 = start + ti * FT, j0 = tj * FT;
    load_panel(W, n, k0, i0, s.T);
    load_rows(X, n, k0, j0, start, s.B);
    __syncthreads();
    tri_times(s.Li, s.T, s.A);
    __syncthreads();
    tri_times(s.Li, s.B, s.T);
    __syncthreads();
    update_tile(X, n, i0, j0, start, false, s.A, s.T);
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

size_t dense_factor_work(int n) { return sizeof(double) * FB * FB * (size_t)((n + FB - 1) / FB); }

void dense_cholesky_inverse(double* A, double* X, int n, int* info_dev, double* work, cudaStream_t s) {
  static_assert(sizeof(DiagShared) <= sizeof(FactorShared), "the look-ahead factor reuses the update tiles' shared memory");
  const int smem = static_cast<int>(sizeof(FactorShared));
  TF_CUDA_CHECK(cudaFuncSetAttribute(factor_step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  TF_CUDA_CHECK(cudaMemsetAsync(X, 0, sizeof(double) * (size_t)n * n, s));
  factor_first_kernel<<<1, F_THREADS, 0, s>>>(A, n, work, info_dev);
  TF_LAUNCH_CHECK("factor_first_kernel");
  const int nblk = (n + FB - 1) / FB;
  for (int k = 0; k <= nblk; ++k) {
    const FactorStep st(n, k);
    if (st.lead + st.finish == 0) continue;
    factor_step_kernel<<<st.lead + st.finish, F_THREADS, smem, s>>>(A, X, work, n, k, info_dev);
    TF_LAUNCH_CHECK("factor_step_kernel");
  }
}

// Split-K form of C = op(X) B: CTA (row block rb, K chunk kc, column group) multiplies 64 rows of op(X)
// restricted to K chunk kc (128 wide) with up to 48 columns of B and stores the partial tile; chunks
// that lie entirely in the zero triangle of op(X) are skipped.  trimul_sum_kernel adds the partials of
// every row in chunk order (deterministic) into C.  Each of the 128 threads holds a 4 x 6 register
// tile (10 shared-memory loads per 24 FMA); the split keeps ~150 CTAs busy at the coarsest sizes
// (a few thousand unknowns), where a whole-K row tile would leave most SMs idle.
constexpr int TM_RB = 64, TM_KCH = 128, TM_KS = 32, TM_CW = 48, TM_THREADS = 128;

__device__ __forceinline__ bool trimul_chunk_live(int i0, int kc, int transpose) {
  return transpose ? (kc + 1) * TM_KCH - 1 >= i0 : kc * TM_KCH <= i0 + TM_RB - 1;
}

__device__ __forceinline__ void trimul_split_body(const VGrid vg_,const double* __restrict__ X, const double* __restrict__ B,
                                                                  double* __restrict__ P, int n, int ncol, int transpose) {
  TF_VGRID(vg_);
  __shared__ double Xs[TM_RB][TM_KS + 1];
  __shared__ double Bs[TM_CW][TM_KS + 1];
  const int i0 = blockIdx.x * TM_RB, kc = blockIdx.y, c0 = blockIdx.z * TM_CW;
  if (!trimul_chunk_live(i0, kc, transpose)) return;
  const int t = threadIdx.x, cg = t % 8, rg = t / 8;   // 16 row groups of 4 x 8 column groups of 6
  const int k_lo = kc * TM_KCH, k_hi = min(n, k_lo + TM_KCH);
  double acc[4][6] = {};
  for (int k0 = k_lo; k0 < k_hi; k0 += TM_KS) {
    for (int e = t; e < TM_RB * TM_KS; e += TM_THREADS) {
      // contiguous global reads: k fastest for X rows, row fastest for X^T
      const int rr = transpose ? e % TM_RB : e / TM_KS, kk = transpose ? e / TM_RB : e % TM_KS;
      const int i = i0 + rr, k = k0 + kk;
      double v = 0.0;
      if (i < n && k < k_hi) v = transpose ? X[(long long)k * n + i] : X[(long long)i * n + k];
      Xs[rr][kk] = v;
    }
    for (int e = t; e < TM_CW * TM_KS; e += TM_THREADS) {
      const int cc = e / TM_KS, kk = e % TM_KS, col = c0 + cc, k = k0 + kk;
      Bs[cc][kk] = (col < ncol && k < k_hi) ? B[(long long)col * n + k] : 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < TM_KS; ++kk) {
      double a[4], b[6];
#pragma unroll
      for (int p = 0; p < 4; ++p) a[p] = Xs[rg * 4 + p][kk];
#pragma unroll
      for (int q = 0; q < 6; ++q) b[q] = Bs[cg * 6 + q][kk];
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 6; ++q) acc[p][q] = fma(a[p], b[q], acc[p][q]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int i = i0 + rg * 4 + p;
    if (i >= n) continue;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const int col = c0 + cg * 6 + q;
      if (col < ncol) P[((long long)kc * ncol + col) * n + i] = acc[p][q];
    }
  }
}
__global__ void __launch_bounds__(TM_THREADS) trimul_split_kernel(const double* __restrict__ X, const double* __restrict__ B,
                                                                  double* __restrict__ P, int n, int ncol, int transpose) {
  trimul_split_body(vgrid(), X, B, P, n, ncol, transpose);
}

__device__ __forceinline__ void trimul_sum_body(const VGrid vg_,const double* __restrict__ P, double* __restrict__ C, int n, int ncol, int nchunks, int transpose,
                                  const int* __restrict__ active) {
  TF_VGRID(vg_);
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
__global__ void trimul_sum_kernel(const double* __restrict__ P, double* __restrict__ C, int n, int ncol, int nchunks, int transpose,
                                  const int* __restrict__ active) {
  trimul_sum_body(vgrid(), P, C, n, ncol, nchunks, transpose, active);
}

struct TrimulSplitRec {
  const double* X;
  const double* B;
  double* P;
  int n, ncol, transpose;
};
__global__ void __launch_bounds__(TM_THREADS) trimul_split_batch(const __grid_constant__ Batch<TrimulSplitRec> b) {
  VGrid vg;
  const TrimulSplitRec& r = b.rec[batch_locate(b, vg)];
  trimul_split_body(vg, r.X, r.B, r.P, r.n, r.ncol, r.transpose);
}
struct TrimulSumRec {
  const double* P;
  double* C;
  int n, ncol, nchunks, transpose;
  const int* active;
};
__global__ void trimul_sum_batch(const __grid_constant__ Batch<TrimulSumRec> b) {
  VGrid vg;
  const TrimulSumRec& r = b.rec[batch_locate(b, vg)];
  trimul_sum_body(vg, r.P, r.C, r.n, r.ncol, r.nchunks, r.transpose, r.active);
}

size_t dense_trimul_work(int n, int ncol) {
  return sizeof(double) * (size_t)((n + TM_KCH - 1) / TM_KCH) * ncol * (size_t)n;
}

void dense_trimul(const double* X, const double* B, double* C, int n, int ncol, int transpose, const int* active, double* work,
                  cudaStream_t s) {
  const int nchunks = (n + TM_KCH - 1) / TM_KCH;
  dim3 grid((n + TM_RB - 1) / TM_RB, nchunks, (ncol + TM_CW - 1) / TM_CW);
  trimul_split_kernel<<<grid, TM_THREADS, 0, s>>>(X, B, work, n, ncol, transpose);
  TF_LAUNCH_CHECK("trimul_split_kernel");
  trimul_sum_kernel<<<grid_for((long long)n * ncol, 256), 256, 0, s>>>(work, C, n, ncol, nchunks, transpose, active);
  TF_LAUNCH_CHECK("trimul_sum_kernel");
}

void dense_trimul_batch(const TrimulJob* jobs, int count, int transpose, cudaStream_t s) {
  std::vector<std::pair<dim3, TrimulSplitRec>> split;
  std::vector<std::pair<dim3, TrimulSumRec>> sum;
  for (int i = 0; i < count; ++i) {
    const TrimulJob& j = jobs[i];
    if (j.n <= 0 || j.ncol <= 0) continue;
    const int nchunks = (j.n + TM_KCH - 1) / TM_KCH;
    split.push_back({dim3((j.n + TM_RB - 1) / TM_RB, nchunks, (j.ncol + TM_CW - 1) / TM_CW),
                     TrimulSplitRec{j.X, j.B, j.work, j.n, j.ncol, transpose}});
    sum.push_back({dim3(grid_for((long long)j.n * j.ncol, 256)), TrimulSumRec{j.work, j.C, j.n, j.ncol, nchunks, transpose, j.active}});
  }
  launch_batched<TrimulSplitRec>(trimul_split_batch, split, dim3(TM_THREADS), 0, s, "trimul_split_batch");
  launch_batched<TrimulSumRec>(trimul_sum_batch, sum, dim3(256), 0, s, "trimul_sum_batch");
}

}  // namespace tfb

// ---------------------------------------------------------------------------
// FP64 direct solver of a sparse SPD system (the drop-in for the reference's
// CudaDirectSolver, deep_frame/topology_optimization.py:80-244).  A matrix whose
// band is much smaller than the dense matrix (a voxel grid's reduced stiffness)
// is factored banded (tf_band.cu); otherwise the CSR matrix is scattered into a
// dense n x n array, symmetrised, factored (A = L L^T), and L is inverted once;
// each solve is x = L^-T (L^-1 b).
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
  int bw = -1;          // bandwidth of the last factored matrix
  bool band = false;    // the last factorisation is banded (else dense with the explicit inverse factor)
  tfb::DevBuf A, X, tmp, info, work, fwork, AB, scratch;
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
constexpr int64_t CHOL_DENSE_MAX_N = 32768;          // dense factor and inverse: 2 n^2 doubles
constexpr double CHOL_BAND_MAX_BYTES = 96.0 * (1 << 30);  // band storage (bw + 1) n doubles
}  // namespace

extern "C" int tf_chol_create(int64_t n, tf_chol** out) {
  if (!out) return tfb::TF_INVALID;
  *out = nullptr;
  tf_chol* h = new tf_chol();
  const int rc = chol_guard(h, [&] {
    tfb::require(n >= 1 && n < (1LL << 31), "the direct solver handles 1 to 2^31 - 1 unknowns");
    h->n = static_cast<int>(n);
    h->info.alloc(sizeof(int));
    h->scratch.alloc(sizeof(int));
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
    // a banded factor when the band is much smaller than the dense matrix (a grid's stiffness in
    // its natural order), the dense factor with its explicit inverse otherwise
    h->bw = tfb::band_width(n, indptr_dev, indices_dev, h->scratch.as<int>(), s);
    h->band = n > CHOL_DENSE_MAX_N || (double)(h->bw + 1) * 8.0 <= (double)n;
    if (h->band) {
      const double bytes = 8.0 * (h->bw + 1) * (double)n;
      tfb::require(bytes <= CHOL_BAND_MAX_BYTES, "the band of this matrix needs " + std::to_string(bytes / 1e9) +
                                                     " GB; reorder it to a smaller bandwidth or use the multigrid solver");
      h->AB.ensure(static_cast<size_t>(bytes));
      tfb::band_assemble(n, indptr_dev, indices_dev, data_dev, h->bw, h->AB.as<double>(), s);
      tfb::band_cholesky(h->AB.as<double>(), n, h->bw, h->info.as<int>(), s);
      int info = 0;
      TF_CUDA_CHECK(cudaMemcpyAsync(&info, h->info.p, sizeof(int), cudaMemcpyDeviceToHost, s));
      TF_CUDA_CHECK(cudaStreamSynchronize(s));
      if (info != 0) throw tfb::Error(tfb::TF_NUMERIC, "matrix is not positive definite (pivot " + std::to_string(info) + ")");
      h->factored = true;
      return;
    }
    h->A.ensure(sizeof(double) * n * n);
    h->X.ensure(sizeof(double) * n * n);
    TF_CUDA_CHECK(cudaMemsetAsync(h->A.p, 0, h->A.bytes, s));
    csr_to_dense_kernel<<<tfb::grid_for(n, 128), 128, 0, s>>>(n, indptr_dev, indices_dev, data_dev, h->A.as<double>());
    TF_LAUNCH_CHECK("csr_to_dense_kernel");
    tfb::dense_symmetrize(h->A.as<double>(), n, s);
    TF_CUDA_CHECK(cudaMemsetAsync(h->info.p, 0, sizeof(int), s));
    if (h->fwork.bytes < tfb::dense_factor_work(n)) h->fwork.alloc(tfb::dense_factor_work(n));
    tfb::dense_cholesky_inverse(h->A.as<double>(), h->X.as<double>(), n, h->info.as<int>(), h->fwork.as<double>(), s);
    int info = 0;
    TF_CUDA_CHECK(cudaMemcpyAsync(&info, h->info.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    TF_CUDA_CHECK(cudaStreamSynchronize(s));
    if (info != 0) throw tfb::Error(tfb::TF_NUMERIC, "matrix is not positive definite (pivot " + std::to_string(info) + ")");
    h->factored = true;
  });
}

extern "C" int tf_chol_solve(tf_chol* h, const double* b_dev, int32_t nrhs, double* x_dev, void* stream) {
  if (!h) return tfb::TF_INVALID;
  return chol_guard(h, [&] {
    tfb::require(h->factored, "tf_chol_solve: no factorisation (call tf_chol_factor_csr first)");
    tfb::require(nrhs >= 1 && b_dev && x_dev, "tf_chol_solve: invalid right-hand sides");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (h->band) {
      tfb::band_solve(h->AB.as<double>(), h->n, h->bw, b_dev, x_dev, nrhs, s);
      return;
    }
    const size_t need = sizeof(double) * (size_t)h->n * nrhs;
    if (h->tmp.bytes < need) h->tmp.alloc(need);
    h->work.ensure(std::max(h->work.bytes, tfb::dense_trimul_work(h->n, nrhs)));
    tfb::dense_trimul(h->X.as<double>(), b_dev, h->tmp.as<double>(), h->n, nrhs, 0, nullptr, h->work.as<double>(), s);
    tfb::dense_trimul(h->X.as<double>(), h->tmp.as<double>(), x_dev, h->n, nrhs, 1, nullptr, h->work.as<double>(), s);
  });
}

extern "C" int tf_chol_destroy(tf_chol* h) {
  if (!h) return tfb::TF_OK;
  // an error the device reports here (from earlier work) is returned, and the handle is freed regardless
  const cudaError_t e = cudaDeviceSynchronize();
  delete h;
  if (e != cudaSuccess) {
    tfb::record_unhandled_error(std::string("tf_chol_destroy: ") + cudaGetErrorString(e));
    return tfb::TF_CUDA;
  }
  return tfb::TF_OK;
}

extern "C" const char* tf_chol_last_error(const tf_chol* h) { return h ? h->err.c_str() : tfb::unhandled_error(); }
