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
#include <mutex>
#include <string>

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

// Count a launch and turn a launch error into TF_CUDA with the message tf_last_error(NULL) returns.
int launch_status(const char* name) {
  g_launch_count.fetch_add(1, std::memory_order_relaxed);
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return TF_OK;
  record_unhandled_error(std::string(name) + ": " + cudaGetErrorString(e));
  return TF_CUDA;
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
  if (ra < 1 || rb < 1 || ra > GRAM_MAX || rb > GRAM_MAX || n < 1 || !a_dev || !b_dev || !out_dev || !scratch_dev) {
    record_unhandled_error("tf_gram: need 1 <= ra, rb <= 64, n >= 1 and non-NULL pointers");
    return TF_INVALID;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int blocks = static_cast<int>(std::min<long long>(GRAM_BLOCKS, (n + KC - 1) / KC));
  gram_partial_kernel<<<blocks, 256, 0, s>>>(a_dev, ra, b_dev, rb, n, scratch_dev);
  int status = launch_status("tf_gram");
  if (status != TF_OK) return status;
  gram_reduce_kernel<<<(ra * rb + 255) / 256, 256, 0, s>>>(scratch_dev, ra * rb, blocks, out_dev);
  return launch_status("tf_gram");
}

namespace tfb {
std::atomic<long long> g_launch_count{0};
}

namespace {
// SIMP interpolation E = E0 (eps + (1 - eps) rho^p), dE/drho = E0 (1 - eps) p rho^(p-1), zero on
// inactive cells (topology_optimization.py:657-661), one cell per thread over the whole grid.
__global__ void __launch_bounds__(256) simp_kernel(const double* __restrict__ rho, long long n, double p, double eps, double young,
                                                   const uint8_t* __restrict__ active, double* __restrict__ moduli,
                                                   double* __restrict__ derivative) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const double r = rho[c];
    const bool on = active ? active[c] != 0 : true;
    moduli[c] = on ? young * (eps + (1.0 - eps) * pow(r, p)) : 0.0;
    if (derivative) derivative[c] = on ? young * (1.0 - eps) * p * pow(r, p - 1.0) : 0.0;
  }
}

// Sum of rho over the active cells (the volume row of topology_problem.py:345): one CTA, every
// thread a fixed stride of cells, then a fixed tree, so the value is bitwise reproducible.  It only
// streams rho and the flags (9 bytes per cell).
__global__ void __launch_bounds__(1024) volume_kernel(const double* __restrict__ rho, long long n, const uint8_t* __restrict__ active,
                                                      double* __restrict__ volume) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (long long c = threadIdx.x; c < n; c += blockDim.x)
    if (!active || active[c]) acc += rho[c];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    *volume = t;
  }
}

// out[j][i] = sum_c coef[c * ncomb + j] * u[c][i]: combinations of solution columns (the partial
// U v_i of the column-sharded lambda_max gradient).  HBM-bound: the columns are read once per
// group of 16 combinations (L1 serves the repeats), the outputs written once.
constexpr int COMBINE_MAX = 64;
constexpr int COMBINE_GROUP = 16;
__global__ void __launch_bounds__(256) combine_kernel(const double* __restrict__ u, int nrhs, long long n, const double* __restrict__ coef,
                                                      int ncomb, double* __restrict__ out) {
  __shared__ double c_s[COMBINE_MAX * COMBINE_MAX];
  for (int t = threadIdx.x; t < nrhs * ncomb; t += blockDim.x) c_s[t] = coef[t];
  __syncthreads();
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    for (int j0 = 0; j0 < ncomb; j0 += COMBINE_GROUP) {
      double acc[COMBINE_GROUP];
#pragma unroll
      for (int q = 0; q < COMBINE_GROUP; ++q) acc[q] = 0.0;
      for (int c = 0; c < nrhs; ++c) {
        const double v = u[(long long)c * n + i];
#pragma unroll
        for (int q = 0; q < COMBINE_GROUP; ++q)
          if (j0 + q < ncomb) acc[q] += c_s[c * ncomb + j0 + q] * v;
      }
#pragma unroll
      for (int q = 0; q < COMBINE_GROUP; ++q)
        if (j0 + q < ncomb) out[(long long)(j0 + q) * n + i] = acc[q];
    }
  }
}

}  // namespace

extern "C" int tf_simp(const double* rho_dev, int64_t n, double penalization, double min_stiffness_ratio, double young,
                       const uint8_t* active_dev, double* moduli_dev, double* derivative_dev, double* volume_dev, void* stream) {
  if (!rho_dev || !moduli_dev || n < 1 || !(penalization >= 1.0) || !(min_stiffness_ratio > 0.0 && min_stiffness_ratio < 1.0) ||
      !(young > 0.0)) {
    record_unhandled_error("tf_simp: invalid arguments");
    return TF_INVALID;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  simp_kernel<<<grid_for(n, 256), 256, 0, s>>>(rho_dev, n, penalization, min_stiffness_ratio, young, active_dev, moduli_dev,
                                               derivative_dev);
  int status = launch_status("tf_simp");
  if (status != TF_OK || !volume_dev) return status;
  volume_kernel<<<1, 1024, 0, s>>>(rho_dev, n, active_dev, volume_dev);
  return launch_status("tf_simp");
}

extern "C" int tf_combine(const double* u_dev, int32_t nrhs, int64_t n, const double* coef_dev, int32_t ncomb, double* out_dev,
                          void* stream) {
  if (nrhs < 1 || ncomb < 1 || nrhs > COMBINE_MAX || ncomb > COMBINE_MAX || n < 1 || !u_dev || !coef_dev || !out_dev) {
    record_unhandled_error("tf_combine: need 1 <= nrhs, ncomb <= 64, n >= 1 and non-NULL pointers");
    return TF_INVALID;
  }
  combine_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, static_cast<cudaStream_t>(stream)>>>(u_dev, nrhs, n, coef_dev, ncomb, out_dev);
  return launch_status("tf_combine");
}

extern "C" int64_t tf_launch_count(void) { return g_launch_count.load(); }

extern "C" int64_t tf_gram_scratch_size(int32_t ra, int32_t rb) {
  return (int64_t)GRAM_BLOCKS * ra * rb;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of tf_gram.
//
// Some callers cannot allocate device memory at the moment they need F: a
// host application that hands this library a fixed device-memory budget and
// owns every allocation itself, or an optimiser loop that runs inside such a
// host's callbacks, where neither cudaMalloc nor a caching allocator may be
// touched.  tf_gram_static takes no scratch argument: its per-CTA partials live
// in the file-scope array below, sized for at most TF_GRAM_STATIC_MAX_PAIRS
// (ra * rb) pairs.  The array is part of the library image, so every GPU that
// loads the library holds it (4.85 MB) until the process exits.
//
// Host code cannot pass the array's name to a kernel: on the host it is only a
// stand-in symbol, not a device address.  The first call on each device looks
// up the device address with cudaGetSymbolAddress (with that device current)
// and caches it; make that first call before any stream capture.  All calls
// share the one array, which keeps the last call's partials: the partial
// kernel writes every slot the reduction then reads, so nothing needs clearing,
// but calls that overlap on the GPU (different streams, no ordering) race on
// the array and must be serialised by the caller.
// ---------------------------------------------------------------------------
namespace {
constexpr int TF_GRAM_STATIC_MAX_PAIRS = 2048;   // e.g. 42 x 42 = 1764 fits
constexpr int TF_GRAM_STATIC_MAX_DEVICES = 64;
static __device__ __align__(256) double g_gram_static_scratch[GRAM_BLOCKS * TF_GRAM_STATIC_MAX_PAIRS];
std::mutex g_gram_static_mutex;
double* g_gram_static_ptr[TF_GRAM_STATIC_MAX_DEVICES] = {};
}  // namespace

extern "C" int tf_gram_static(const double* a_dev, int32_t ra, const double* b_dev, int32_t rb, int64_t n, double* out_dev,
                              void* stream) {
  if (ra < 1 || rb < 1 || ra > GRAM_MAX || rb > GRAM_MAX || n < 1 || !a_dev || !b_dev || !out_dev) {
    record_unhandled_error("tf_gram_static: need 1 <= ra, rb <= 64, n >= 1 and non-NULL pointers");
    return TF_INVALID;
  }
  if ((long long)ra * rb > TF_GRAM_STATIC_MAX_PAIRS) {
    record_unhandled_error("tf_gram_static: ra * rb = " + std::to_string((long long)ra * rb) +
                           " exceeds the static scratch limit of " + std::to_string(TF_GRAM_STATIC_MAX_PAIRS) +
                           " pairs; use tf_gram with a caller-provided scratch buffer");
    return TF_INVALID;
  }
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= TF_GRAM_STATIC_MAX_DEVICES) {
    record_unhandled_error("tf_gram_static: no usable current CUDA device");
    return TF_CUDA;
  }
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_gram_static_mutex);
    if (!g_gram_static_ptr[device]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_gram_static_scratch);
      if (e != cudaSuccess || !p) {
        record_unhandled_error(std::string("tf_gram_static: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
        return TF_CUDA;
      }
      g_gram_static_ptr[device] = static_cast<double*>(p);
    }
    scratch = g_gram_static_ptr[device];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int blocks = static_cast<int>(std::min<long long>(GRAM_BLOCKS, (n + KC - 1) / KC));
  gram_partial_kernel<<<blocks, 256, 0, s>>>(a_dev, ra, b_dev, rb, n, scratch);
  int status = launch_status("tf_gram_static");
  if (status != TF_OK) return status;
  gram_reduce_kernel<<<(ra * rb + 255) / 256, 256, 0, s>>>(scratch, ra * rb, blocks, out_dev);
  return launch_status("tf_gram_static");
}
