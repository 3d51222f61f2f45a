// Small dense FP64 helpers of the covariance measure.
//
// tf_gram computes F = A B^T for two column blocks [ra][n] and [rb][n] (the
// flexibility P^T U of topology_problem.py:639-646): every CTA reduces one
// slab of the n dofs for all ra x rb pairs through shared-memory tiles, and a
// second launch sums the per-CTA partials in a fixed order, so the result is
// bitwise reproducible.
#include "tf_b200.h"
#include "tf_common.h"
#include <algorithm>

using namespace tfb;

namespace {
constexpr int GRAM_MAX = 64;   // rows per operand
constexpr int KC = 32;         // dofs per shared-memory tile
constexpr int GRAM_BLOCKS = 296;

__global__ void __launch_bounds__(256) gram_partial_kernel(const double* __restrict__ a, int ra, const double* __restrict__ b, int rb,
                                                           long long n, double* __restrict__ partial) {
  __shared__ double As[GRAM_MAX][KC + 1];
  __shared__ double Bs[GRAM_MAX][KC + 1];
  const long long chunk = (n + gridDim.x - 1) / gridDim.x;
  const long long k_begin = (long long)blockIdx.x * chunk;
  const long long k_end = min(n, k_begin + chunk);
  const int pairs = ra * rb;
  double acc[(GRAM_MAX * GRAM_MAX + 255) / 256];
#pragma unroll
  for (int q = 0; q < (GRAM_MAX * GRAM_MAX + 255) / 256; ++q) acc[q] = 0.0;
  for (long long k0 = k_begin; k0 < k_end; k0 += KC) {
    for (int t = threadIdx.x; t < GRAM_MAX * KC; t += blockDim.x) {
      const int r = t / KC, k = t % KC;
      const long long kk = k0 + k;
      As[r][k] = (r < ra && kk < k_end) ? a[(long long)r * n + kk] : 0.0;
      Bs[r][k] = (r < rb && kk < k_end) ? b[(long long)r * n + kk] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < (GRAM_MAX * GRAM_MAX + 255) / 256; ++q) {
      const int p = threadIdx.x + q * 256;
      if (p < pairs) {
        const int i = p / rb, j = p % rb;
        double v = 0.0;
#pragma unroll 8
        for (int k = 0; k < KC; ++k) v += As[i][k] * Bs[j][k];
        acc[q] += v;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < (GRAM_MAX * GRAM_MAX + 255) / 256; ++q) {
    const int p = threadIdx.x + q * 256;
    if (p < pairs) partial[(long long)blockIdx.x * pairs + p] = acc[q];
  }
}

__global__ void gram_reduce_kernel(const double* __restrict__ partial, int pairs, int blocks, double* __restrict__ out) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < pairs; p += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < blocks; ++b) s += partial[(long long)b * pairs + p];
    out[p] = s;
  }
}
}  // namespace

extern "C" int tf_gram(const double* a_dev, int32_t ra, const double* b_dev, int32_t rb, int64_t n, double* out_dev,
                       double* scratch_dev, void* stream) {
  if (ra < 1 || rb < 1 || ra > GRAM_MAX || rb > GRAM_MAX || n < 1 || !a_dev || !b_dev || !out_dev || !scratch_dev)
    return TF_INVALID;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int blocks = static_cast<int>(std::min<long long>(GRAM_BLOCKS, (n + KC - 1) / KC));
  gram_partial_kernel<<<blocks, 256, 0, s>>>(a_dev, ra, b_dev, rb, n, scratch_dev);
  g_launch_count.fetch_add(1, std::memory_order_relaxed);
  if (cudaGetLastError() != cudaSuccess) return TF_CUDA;
  gram_reduce_kernel<<<(ra * rb + 255) / 256, 256, 0, s>>>(scratch_dev, ra * rb, blocks, out_dev);
  g_launch_count.fetch_add(1, std::memory_order_relaxed);
  if (cudaGetLastError() != cudaSuccess) return TF_CUDA;
  return TF_OK;
}

namespace tfb {
std::atomic<long long> g_launch_count{0};
}

extern "C" int64_t tf_launch_count(void) { return g_launch_count.load(); }

extern "C" int64_t tf_gram_scratch_size(int32_t ra, int32_t rb) {
  return (int64_t)GRAM_BLOCKS * ra * rb;
}
