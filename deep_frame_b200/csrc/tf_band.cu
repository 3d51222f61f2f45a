// Banded FP64 Cholesky of a sparse SPD system: the direct solver for systems too large for a dense
// factor (the drop-in for the reference's sparse CudaDirectSolver, deep_frame/topology_optimization.py:
// 80-244, on the reduced stiffness of a voxel grid).
//
// A voxel grid's reduced stiffness in its natural dof order (x slowest) is banded: a dof couples
// only to dofs of nodes within one cell, so |i - j| <= bw ~ 3 (ny + 1)(nz + 1).  Band Cholesky
// creates no fill outside the band.  Storage is column-major band: AB[j * ld + d] = A[j + d][j] for
// 0 <= d <= bw, ld = bw + 1, so a column's entries (and a tile's rows) are contiguous.
//
// Factorisation, right-looking in block columns of NB: factor the NB x NB diagonal block in one CTA
// (band_potrf_kernel), solve the block's sub-diagonal rows against it (band_trsm_kernel, one row per
// thread), and update the trailing m x m window, m <= bw, with the block's rank-NB product
// (band_syrk_kernel, 64 x 64 tiles of the window's lower triangle).  Entries with i - j > bw have no
// storage and are structurally zero throughout.  Solves run one CTA per right-hand side, block by
// block (forward L y = b, then backward L^T x = y).
#include <algorithm>
#include <string>

#include "tf_common.h"
#include "tf_dense.h"

namespace tfb {
namespace {

constexpr int NB = 64;          // block column width
constexpr int ST = 64;          // SYRK tile edge
constexpr int SYRK_THREADS = 256;

// bandwidth: max (i - j) over the stored entries with i >= j (both triangles are scanned; the matrix is
// symmetrised on assembly)
__global__ void band_width_kernel(int n, const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices, int* __restrict__ out) {
  int local = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (int k = indptr[i]; k < indptr[i + 1]; ++k) {
      const int j = indices[k];
      if ((unsigned)j < (unsigned)n) local = max(local, abs(i - j));
    }
  for (int o = 16; o > 0; o >>= 1) local = max(local, __shfl_xor_sync(0xffffffffu, local, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, local);
}

// AB <- (A + A^T) / 2 on the band: every stored entry adds half of itself at its lower-triangle slot.
// Each slot receives at most two additions to zero (a_ij / 2 and a_ji / 2): the sum does not depend on
// their order.
__global__ void band_scatter_kernel(int n, const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                                    const double* __restrict__ data, int ld, double* __restrict__ AB) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (int k = indptr[i]; k < indptr[i + 1]; ++k) {
      const int j = indices[k];
      if ((unsigned)j >= (unsigned)n) continue;
      const int lo = min(i, j), hi = max(i, j);
      atomicAdd(&AB[(long long)lo * ld + (hi - lo)], i == j ? data[k] : 0.5 * data[k]);
    }
}

// Cholesky of the kb x kb diagonal block at column k0, in place (one CTA).  info (1 + global column
// of the first non-positive pivot) is set when a pivot fails; the block is then left unfinished.
__global__ void __launch_bounds__(256) band_potrf_kernel(double* __restrict__ AB, int ld, int bw, int k0, int kb, int* __restrict__ info) {
  __shared__ double L[NB][NB + 1];
  __shared__ int bad;
  if (*info) return;
  for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
    const int r = t / kb, c = t % kb;
    L[r][c] = (r >= c && r - c <= bw) ? AB[(long long)(k0 + c) * ld + (r - c)] : 0.0;
  }
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  for (int c = 0; c < kb; ++c) {
    if (threadIdx.x == 0) {
      const double d = L[c][c];
      if (!(d > 0.0) || !isfinite(d)) bad = 1;
      else L[c][c] = sqrt(d);
    }
    __syncthreads();
    if (bad) {
      if (threadIdx.x == 0) atomicCAS(info, 0, k0 + c + 1);
      return;
    }
    const double piv = L[c][c];
    for (int r = c + 1 + threadIdx.x; r < kb; r += blockDim.x) L[r][c] /= piv;
    __syncthreads();
    // trailing update of the block: L[r][q] -= L[r][c] L[q][c] for c < q <= r
    for (int t = threadIdx.x; t < (kb - c - 1) * (kb - c - 1); t += blockDim.x) {
      const int r = c + 1 + t / (kb - c - 1), q = c + 1 + t % (kb - c - 1);
      if (q <= r) L[r][q] -= L[r][c] * L[q][c];
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
    const int r = t / kb, c = t % kb;
    if (r >= c && r - c <= bw) AB[(long long)(k0 + c) * ld + (r - c)] = L[r][c];
  }
}

// Rows i in [k0 + kb, k0 + kb + m) of the block column: L21 = A21 L11^-T, one row per thread.
// Entries with i - j > bw stay absent (they are zero before and after).
__global__ void __launch_bounds__(128) band_trsm_kernel(double* __restrict__ AB, int ld, int bw, int k0, int kb, int m,
                                                        const int* __restrict__ info) {
  __shared__ double L[NB][NB + 1];
  if (*info) return;
  for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
    const int r = t / kb, c = t % kb;
    L[r][c] = (r >= c && r - c <= bw) ? AB[(long long)(k0 + c) * ld + (r - c)] : 0.0;
  }
  __syncthreads();
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= m) return;
  const int i = k0 + kb + row;
  double x[NB];
#pragma unroll
  for (int c = 0; c < NB; ++c) {
    if (c >= kb) break;
    const int d = i - (k0 + c);
    double v = d <= bw ? AB[(long long)(k0 + c) * ld + d] : 0.0;
#pragma unroll
    for (int l = 0; l < NB; ++l) {
      if (l >= c) break;
      v -= x[l] * L[c][l];
    }
    x[c] = v / L[c][c];
    if (d <= bw) AB[(long long)(k0 + c) * ld + d] = x[c];
  }
}

// Trailing window update A[i][j] -= sum_c L21[i][c] L21[j][c] for rows and columns in
// [w0, w0 + m), i >= j; one CTA per 64 x 64 tile of the window's lower triangle (blockIdx.x enumerates
// them row by row), 4 x 4 outputs per thread.
constexpr size_t SYRK_SMEM = sizeof(double) * 2 * NB * (ST + 1);
__global__ void __launch_bounds__(SYRK_THREADS) band_syrk_kernel(double* __restrict__ AB, int ld, int bw, int k0, int kb, int m,
                                                                 const int* __restrict__ info) {
  extern __shared__ double syrk_smem[];
  double (*Li)[ST + 1] = reinterpret_cast<double (*)[ST + 1]>(syrk_smem);
  double (*Lj)[ST + 1] = reinterpret_cast<double (*)[ST + 1]>(syrk_smem + NB * (ST + 1));
  if (*info) return;
  // tile (ti, tj), tj <= ti, from the linear index
  int ti = static_cast<int>((sqrt(8.0 * blockIdx.x + 1.0) - 1.0) / 2.0);
  while ((ti + 1) * (ti + 2) / 2 <= (int)blockIdx.x) ++ti;
  while (ti * (ti + 1) / 2 > (int)blockIdx.x) --ti;
  const int tj = blockIdx.x - ti * (ti + 1) / 2;
  const int w0 = k0 + kb;
  const int i0 = w0 + ti * ST, j0 = w0 + tj * ST;
  for (int t = threadIdx.x; t < kb * ST; t += blockDim.x) {
    const int c = t / ST, r = t % ST;
    const int col = k0 + c;
    const int ii = i0 + r, jj = j0 + r;
    Li[c][r] = (ii < w0 + m && ii - col <= bw) ? AB[(long long)col * ld + (ii - col)] : 0.0;
    Lj[c][r] = (jj < w0 + m && jj - col <= bw) ? AB[(long long)col * ld + (jj - col)] : 0.0;
  }
  __syncthreads();
  const int tr = threadIdx.x % 16, tc = threadIdx.x / 16;   // rows tr + 16 p, columns tc + 16 q
  double acc[4][4] = {};
  for (int c = 0; c < kb; ++c) {
    double a[4], b[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) a[p] = Li[c][tr + 16 * p];
#pragma unroll
    for (int q = 0; q < 4; ++q) b[q] = Lj[c][tc + 16 * q];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[p][q] = fma(a[p], b[q], acc[p][q]);
  }
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int i = i0 + tr + 16 * p;
    if (i >= w0 + m) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int j = j0 + tc + 16 * q;
      if (j > i || j >= w0 + m) continue;
      AB[(long long)j * ld + (i - j)] -= acc[p][q];
    }
  }
}

// Forward and backward substitution for one right-hand side per CTA: x = L^-T L^-1 b.
constexpr int SOLVE_THREADS = 512;
__global__ void __launch_bounds__(SOLVE_THREADS) band_solve_kernel(const double* __restrict__ AB, int ld, int bw, int n,
                                                                   const double* __restrict__ b, double* __restrict__ x) {
  __shared__ double yb[NB];
  __shared__ double red[SOLVE_THREADS / 32][NB];
  const double* bc = b + (long long)blockIdx.x * n;
  double* xc = x + (long long)blockIdx.x * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) xc[i] = bc[i];
  __syncthreads();
  // forward: y = L^-1 b, in place in xc
  for (int k0 = 0; k0 < n; k0 += NB) {
    const int kb = min(NB, n - k0);
    if (threadIdx.x < 32) {
      // one warp solves the diagonal block: lane l owns rows l and l + 32
      for (int c = 0; c < kb; ++c) {
        double yc = 0.0;
        if (threadIdx.x == (c & 31)) {
          double v = xc[k0 + c];
          for (int l = max(0, c - bw); l < c; ++l) v -= AB[(long long)(k0 + l) * ld + (c - l)] * yb[l];
          yc = v / AB[(long long)(k0 + c) * ld];
          yb[c] = yc;
        }
        __syncwarp();
      }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < kb; c += blockDim.x) xc[k0 + c] = yb[c];
    const int m = min(n - k0 - kb, bw);
    for (int r = threadIdx.x; r < m; r += blockDim.x) {
      const int i = k0 + kb + r;
      double v = 0.0;
      for (int c = 0; c < kb; ++c) {
        const int d = i - (k0 + c);
        if (d <= bw) v += AB[(long long)(k0 + c) * ld + d] * yb[c];
      }
      xc[i] -= v;
    }
    __syncthreads();
  }
  // backward: x = L^-T y
  const int last = ((n - 1) / NB) * NB;
  for (int k0 = last; k0 >= 0; k0 -= NB) {
    const int kb = min(NB, n - k0);
    const int m = min(n - k0 - kb, bw);
    // t_c = sum_r L21[r][c] x[k0 + kb + r]: per-thread partial sums over rows, then a fixed-order tree
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int c = 0; c < kb; ++c) {
      double v = 0.0;
      for (int r = threadIdx.x; r < m; r += blockDim.x) {
        const int i = k0 + kb + r, d = i - (k0 + c);
        if (d <= bw) v += AB[(long long)(k0 + c) * ld + d] * xc[i];
      }
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) red[warp][c] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int c = kb - 1; c >= 0; --c) {
        double t = 0.0;
        for (int w = 0; w < SOLVE_THREADS / 32; ++w) t += red[w][c];
        double v = xc[k0 + c] - t;
        for (int l = c + 1; l < kb && l - c <= bw; ++l) v -= AB[(long long)(k0 + c) * ld + (l - c)] * yb[l];
        yb[c] = v / AB[(long long)(k0 + c) * ld];
      }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < kb; c += blockDim.x) xc[k0 + c] = yb[c];
    __syncthreads();
  }
}

}  // namespace

int band_width(int n, const int32_t* indptr, const int32_t* indices, int* scratch_dev, cudaStream_t s) {
  TF_CUDA_CHECK(cudaMemsetAsync(scratch_dev, 0, sizeof(int), s));
  band_width_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, s>>>(n, indptr, indices, scratch_dev);
  TF_LAUNCH_CHECK("band_width_kernel");
  int bw = 0;
  TF_CUDA_CHECK(cudaMemcpyAsync(&bw, scratch_dev, sizeof(int), cudaMemcpyDeviceToHost, s));
  TF_CUDA_CHECK(cudaStreamSynchronize(s));
  return bw;
}

void band_assemble(int n, const int32_t* indptr, const int32_t* indices, const double* data, int bw, double* AB, cudaStream_t s) {
  TF_CUDA_CHECK(cudaMemsetAsync(AB, 0, sizeof(double) * (size_t)(bw + 1) * n, s));
  band_scatter_kernel<<<grid_for(n, 128), 128, 0, s>>>(n, indptr, indices, data, bw + 1, AB);
  TF_LAUNCH_CHECK("band_scatter_kernel");
}

void band_cholesky(double* AB, int n, int bw, int* info_dev, cudaStream_t s) {
  const int ld = bw + 1;
  static bool configured = false;   // per process; the attribute is per function
  if (!configured) {
    TF_CUDA_CHECK(cudaFuncSetAttribute(band_syrk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SYRK_SMEM));
    configured = true;
  }
  TF_CUDA_CHECK(cudaMemsetAsync(info_dev, 0, sizeof(int), s));
  for (int k0 = 0; k0 < n; k0 += NB) {
    const int kb = std::min(NB, n - k0);
    band_potrf_kernel<<<1, 256, 0, s>>>(AB, ld, bw, k0, kb, info_dev);
    TF_LAUNCH_CHECK("band_potrf_kernel");
    const int m = std::min(n - k0 - kb, bw);
    if (m <= 0) continue;
    band_trsm_kernel<<<(m + 127) / 128, 128, 0, s>>>(AB, ld, bw, k0, kb, m, info_dev);
    TF_LAUNCH_CHECK("band_trsm_kernel");
    const int tiles = (m + ST - 1) / ST;
    band_syrk_kernel<<<tiles * (tiles + 1) / 2, SYRK_THREADS, SYRK_SMEM, s>>>(AB, ld, bw, k0, kb, m, info_dev);
    TF_LAUNCH_CHECK("band_syrk_kernel");
  }
}

void band_solve(const double* AB, int n, int bw, const double* b, double* x, int nrhs, cudaStream_t s) {
  band_solve_kernel<<<nrhs, SOLVE_THREADS, 0, s>>>(AB, bw + 1, bw, n, b, x);
  TF_LAUNCH_CHECK("band_solve_kernel");
}

}  // namespace tfb
