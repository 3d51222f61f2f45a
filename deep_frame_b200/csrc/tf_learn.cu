// Kernels of the learned initial guess: a small 3-D convolutional encoder / decoder trained on the
// solver's own (density, load, displacement) snapshots.  Convolutions are explicit im2col + a
// deterministic tiled SGEMM (FP32, split-K partial sums added in a fixed order), so forward and
// backward passes are bitwise reproducible; the remaining layers (bias + ReLU, 2x average pooling,
// 2x nearest upsampling, loss, Adam) are elementwise or fixed-order reductions.  Tensors are
// channel-major [C][nx][ny][nz] FP32 on a node grid; pooling halves each extent rounding up
// (missing children count as zero), upsampling copies a coarse value to its (up to 8) children.
#include <cmath>
#include <cuda_fp16.h>
#include <string>

#include "tf_b200.h"
#include "tf_common.h"
#include "tf_reduce.cuh"

using namespace tfb;

namespace {

thread_local std::string g_learn_error;

template <typename F>
int learn_guard(F&& f) {
  try {
    f();
    return TF_OK;
  } catch (const Error& e) {
    g_learn_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_learn_error = e.what();
    return TF_INTERNAL;
  }
}

struct Grid3 {
  int nx, ny, nz;
  __host__ __device__ long long n() const { return (long long)nx * ny * nz; }
};

// col[(c * 27 + t)][v] = in[c][v + offset(t)] (zero outside the grid)
__global__ void im2col_kernel(const float* __restrict__ in, int channels, Grid3 g, float* __restrict__ col) {
  const long long n = g.n();
  const long long total = (long long)channels * 27 * n;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
    const long long v = idx % n;
    const long long row = idx / n;
    const int t = static_cast<int>(row % 27), c = static_cast<int>(row / 27);
    const int k = static_cast<int>(v % g.nz);
    const long long r = v / g.nz;
    const int j = static_cast<int>(r % g.ny), i = static_cast<int>(r / g.ny);
    const int ii = i + t / 9 - 1, jj = j + (t / 3) % 3 - 1, kk = k + t % 3 - 1;
    float x = 0.0f;
    if ((unsigned)ii < (unsigned)g.nx && (unsigned)jj < (unsigned)g.ny && (unsigned)kk < (unsigned)g.nz)
      x = in[(long long)c * n + ((long long)ii * g.ny + jj) * g.nz + kk];
    col[idx] = x;
  }
}

// Adjoint of im2col: in[c][v] = sum_t col[(c * 27 + t)][v - offset(t)] (gather, fixed tap order)
__global__ void col2im_kernel(const float* __restrict__ col, int channels, Grid3 g, float* __restrict__ out) {
  const long long n = g.n();
  const long long total = (long long)channels * n;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
    const long long v = idx % n;
    const int c = static_cast<int>(idx / n);
    const int k = static_cast<int>(v % g.nz);
    const long long r = v / g.nz;
    const int j = static_cast<int>(r % g.ny), i = static_cast<int>(r / g.ny);
    float acc = 0.0f;
    for (int t = 0; t < 27; ++t) {
      const int ii = i - (t / 9 - 1), jj = j - ((t / 3) % 3 - 1), kk = k - (t % 3 - 1);
      if ((unsigned)ii < (unsigned)g.nx && (unsigned)jj < (unsigned)g.ny && (unsigned)kk < (unsigned)g.nz)
        acc += col[((long long)c * 27 + t) * n + ((long long)ii * g.ny + jj) * g.nz + kk];
    }
    out[idx] = acc;
  }
}

// C = alpha * op(A) op(B) + beta * C, row-major, op = transpose when flagged; split over K into
// `splits` slices whose partial tiles go to `work` and are summed in slice order by sum_splits_kernel.
constexpr int GT = 64, GK = 16;
__global__ void __launch_bounds__(256) sgemm_kernel(int ta, int tb, int M, int N, int K, const float* __restrict__ A, int lda,
                                                    const float* __restrict__ B, int ldb, float* __restrict__ out, int ldo,
                                                    int kchunk) {
  __shared__ float sa[GK][GT + 4];
  __shared__ float sb[GK][GT + 4];
  const int m0 = blockIdx.y * GT, n0 = blockIdx.x * GT;
  const int k_begin = blockIdx.z * kchunk, k_end = min(K, k_begin + kchunk);
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;   // 16 x 16 threads, 4 x 4 outputs each
  float acc[4][4] = {};
  for (int k0 = k_begin; k0 < k_end; k0 += GK) {
    // the contiguous dimension of each operand is the thread-fastest one (coalesced loads)
    for (int idx = threadIdx.x; idx < GK * GT; idx += 256) {
      const int kk = ta ? idx / GT : idx % GK, mm = ta ? idx % GT : idx / GK;
      const int m = m0 + mm, k = k0 + kk;
      float v = 0.0f;
      if (m < M && k < k_end) v = ta ? A[(long long)k * lda + m] : A[(long long)m * lda + k];
      sa[kk][mm] = v;
      const int kb = tb ? idx % GK : idx / GT, nn = tb ? idx / GK : idx % GT;
      const int nidx = n0 + nn, kbi = k0 + kb;
      float w = 0.0f;
      if (nidx < N && kbi < k_end) w = tb ? B[(long long)nidx * ldb + kbi] : B[(long long)kbi * ldb + nidx];
      sb[kb][nn] = w;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GK; ++kk) {
      float a4[4], b4[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) { a4[q] = sa[kk][ty * 4 + q]; b4[q] = sb[kk][tx * 4 + q]; }
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] = fmaf(a4[p], b4[q], acc[p][q]);
    }
    __syncthreads();
  }
  float* o = out + (long long)blockIdx.z * M * (long long)ldo;
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int m = m0 + ty * 4 + p;
    if (m >= M) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int nn = n0 + tx * 4 + q;
      if (nn < N) o[(long long)m * ldo + nn] = acc[p][q];
    }
  }
}

__global__ void sum_splits_kernel(const float* __restrict__ work, int splits, int M, int N, float alpha, float beta,
                                  float* __restrict__ C, int ldc) {
  const long long total = (long long)M * N;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
    const int m = static_cast<int>(idx / N), nn = static_cast<int>(idx % N);
    float s = 0.0f;
    for (int q = 0; q < splits; ++q) s += work[((long long)q * M + m) * N + nn];
    float* c = C + (long long)m * ldc + nn;
    *c = alpha * s + (beta != 0.0f ? beta * *c : 0.0f);
  }
}

// y[c][v] = max(x[c][v] + bias[c], 0) (relu != 0) or x + bias
__global__ void bias_act_kernel(float* __restrict__ x, const float* __restrict__ bias, int channels, long long n, int relu) {
  const long long total = (long long)channels * n;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
    float v = x[idx] + bias[idx / n];
    x[idx] = relu ? fmaxf(v, 0.0f) : v;
  }
}

// dx = dy * (y > 0) (relu) in place; db[c] = sum_v dx[c][v] (one CTA per channel, fixed order)
__global__ void __launch_bounds__(RED_THREADS) act_back_kernel(float* __restrict__ dy, const float* __restrict__ y, long long n,
                                                               int relu, float* __restrict__ db, int accumulate) {
  const int c = blockIdx.x;
  double s = 0.0, z = 0.0;
  for (long long v = threadIdx.x; v < n; v += blockDim.x) {
    const long long idx = (long long)c * n + v;
    float g = dy[idx];
    if (relu && !(y[idx] > 0.0f)) g = 0.0f;
    dy[idx] = g;
    s += g;
  }
  block_reduce2<0, 0>(s, z);
  if (threadIdx.x == 0) db[c] = (accumulate ? db[c] : 0.0f) + static_cast<float>(s);
}

__global__ void pool_kernel(const float* __restrict__ in, int channels, Grid3 f, Grid3 c, float* __restrict__ out) {
  const long long nc = c.n(), nf = f.n();
  const long long total = (long long)channels * nc;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
    const long long v = idx % nc;
    const int ch = static_cast<int>(idx / nc);
    const int k = static_cast<int>(v % c.nz);
    const long long r = v / c.nz;
    const int j = static_cast<int>(r % c.ny), i = static_cast<int>(r / c.ny);
    float s = 0.0f;
    for (int q = 0; q < 8; ++q) {
      const int ii = 2 * i + (q >> 2), jj = 2 * j + ((q >> 1) & 1), kk = 2 * k + (q & 1);
      if (ii < f.nx && jj < f.ny && kk < f.nz) s += in[(long long)ch * nf + ((long long)ii * f.ny + jj) * f.nz + kk];
    }
    out[idx] = 0.125f * s;
  }
}

// upsample (mode 0): fine[v] = coarse[parent(v)];  pool adjoint (mode 1): fine[v] = coarse[parent(v)] / 8
__global__ void spread_kernel(const float* __restrict__ coarse, int channels, Grid3 f, Grid3 c, float* __restrict__ fine, float scale) {
  const long long nc = c.n(), nf = f.n();
  const long long total = (long long)channels * nf;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
    const long long v = idx % nf;
    const int ch = static_cast<int>(idx / nf);
    const int k = static_cast<int>(v % f.nz);
    const long long r = v / f.nz;
    const int j = static_cast<int>(r % f.ny), i = static_cast<int>(r / f.ny);
    fine[idx] = scale * coarse[(long long)ch * nc + ((long long)(i / 2) * c.ny + j / 2) * c.nz + k / 2];
  }
}

// upsample adjoint: coarse[v] = sum of its children's gradients (fixed child order)
__global__ void gather_children_kernel(const float* __restrict__ fine, int channels, Grid3 f, Grid3 c, float* __restrict__ coarse) {
  const long long nc = c.n(), nf = f.n();
  const long long total = (long long)channels * nc;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
    const long long v = idx % nc;
    const int ch = static_cast<int>(idx / nc);
    const int k = static_cast<int>(v % c.nz);
    const long long r = v / c.nz;
    const int j = static_cast<int>(r % c.ny), i = static_cast<int>(r / c.ny);
    float s = 0.0f;
    for (int q = 0; q < 8; ++q) {
      const int ii = 2 * i + (q >> 2), jj = 2 * j + ((q >> 1) & 1), kk = 2 * k + (q & 1);
      if (ii < f.nx && jj < f.ny && kk < f.nz) s += fine[(long long)ch * nf + ((long long)ii * f.ny + jj) * f.nz + kk];
    }
    coarse[idx] = s;
  }
}

// loss = sum w (y - t)^2 / n_weighted ; dy = 2 w (y - t) / n_weighted ; partial sums per block, last block combines
__global__ void __launch_bounds__(RED_THREADS) mse_kernel(const float* __restrict__ y, const float* __restrict__ t,
                                                          const float* __restrict__ w, long long n, float inv_count,
                                                          float* __restrict__ dy, double* partial, unsigned* count,
                                                          double* loss) {
  double s = 0.0, z = 0.0;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
    const float wt = w ? w[idx] : 1.0f;
    const float d = y[idx] - t[idx];
    s += (double)wt * d * d;
    if (dy) dy[idx] = 2.0f * wt * d * inv_count;
  }
  block_reduce2<0, 0>(s, z);
  if (last_block_combine<0, 0>(s, z, partial, count, 0)) *loss = s * inv_count;
}

// Adam (bias-corrected), parameters FP32
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                            long long n, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
    const float gi = g[idx];
    const float mi = b1 * m[idx] + (1.0f - b1) * gi;
    const float vi = b2 * v[idx] + (1.0f - b2) * gi * gi;
    m[idx] = mi;
    v[idx] = vi;
    p[idx] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

Grid3 grid3(const int32_t s[3]) { return Grid3{s[0], s[1], s[2]}; }

// ---------------------------------------------------------------------------
// 3 x 3 x 3 convolution on the 5th-generation tensor cores (inference form of the network):
// y[o][v] = act(bias[o] + sum_{c,t} W[o][c * 27 + t] x[c][v + offset(t)]) as an implicit GEMM
// with M = 128 consecutive output nodes per CTA, N = the output channels padded to a multiple of
// 16 (W packed to FP16 [np][kp], kp a multiple of 64), K = input channels x 27 taps in chunks of
// 64.  Per chunk every thread gathers its node's 64 (channel, tap) inputs, rounds them to FP16 and
// writes them to shared memory in the UMMA K-major layout (16-byte rows of 8 values, core matrices
// of 8 rows); the weight chunk is copied beside it; one thread issues four tcgen05.mma kind::f16
// (K = 16 each) accumulating in FP32 in TMEM and commits them to the chunk buffer's mbarrier, so
// the gather of the next chunk (double-buffered) overlaps them.  The accumulators come back with
// tcgen05.ld, one TMEM lane (= output node) per thread.  Every wait is bounded; a timeout sets
// *err, waits (bounded) for the MMAs in flight and frees the TMEM.
// ---------------------------------------------------------------------------
constexpr int CV_M = 128, CV_KC = 64, CV_NMAX = 64, CV_THREADS = 128, CV_TMEM = 64;
constexpr unsigned CV_SPIN = 1u << 22;
constexpr int CV_A_BYTES = CV_M * CV_KC * 2;           // 16 KB per stage
constexpr int CV_B_BYTES = CV_NMAX * CV_KC * 2;        // 8 KB per stage
constexpr int CV_SMEM = 2 * CV_A_BYTES + 2 * CV_B_BYTES + 64;

__device__ __forceinline__ uint32_t cv_smem(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// UMMA shared-memory descriptor, K-major without swizzle (lbo: between 16-byte K columns of core
// matrices, sbo: between 8-row groups).
__device__ __forceinline__ uint64_t cv_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = static_cast<uint64_t>((addr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
  d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
  d |= static_cast<uint64_t>(1) << 46;
  return d;
}

__device__ __forceinline__ bool cv_wait(uint32_t bar, uint32_t parity) {
  for (unsigned it = 0; it < CV_SPIN; ++it) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
                 : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    if (ok) return true;
  }
  return false;
}

__global__ void __launch_bounds__(CV_THREADS) conv16_kernel(const float* __restrict__ x, int cin, Grid3 g, const __half* __restrict__ w16,
                                                           int cout, int np, int kp, const float* __restrict__ bias, int relu,
                                                           float* __restrict__ y, int* err) {
  extern __shared__ __align__(128) unsigned char cv_raw[];
  unsigned char* sA = cv_raw;                                  // [2][CV_KC / 8][CV_M][16 B]
  unsigned char* sB = cv_raw + 2 * CV_A_BYTES;                 // [2][CV_KC / 8][np][16 B]
  uint64_t* bars = reinterpret_cast<uint64_t*>(cv_raw + 2 * CV_A_BYTES + 2 * CV_B_BYTES);
  uint32_t* tbase = reinterpret_cast<uint32_t*>(bars + 2);
  int* abort_flag = reinterpret_cast<int*>(bars + 3);
  const int t = threadIdx.x, warp = t >> 5;
  const long long n = g.n();
  const long long v = (long long)blockIdx.x * CV_M + t;
  const bool live = v < n;
  int vi = 0, vj = 0, vk = 0;
  if (live) {
    vk = static_cast<int>(v % g.nz);
    const long long r = v / g.nz;
    vj = static_cast<int>(r % g.ny);
    vi = static_cast<int>(r / g.ny);
  }
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(cv_smem(&bars[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(cv_smem(&bars[1])));
    *abort_flag = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(cv_smem(tbase)), "r"(CV_TMEM));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tbase;
  const int K = cin * 27;
  const int chunks = kp / CV_KC;
  const uint32_t idesc = (1u << 4) | (uint32_t(np >> 3) << 17) | (uint32_t(CV_M >> 4) << 24);   // D FP32, A, B FP16, K-major
  uint32_t phases = 0u;   // bit s: the parity awaited next on stage s's barrier
  for (int q = 0; q < chunks; ++q) {
    const int st = q & 1;
    if (q >= 2) {   // the MMAs of chunk q - 2 have read this stage
      if (!cv_wait(cv_smem(&bars[st]), (phases >> st) & 1u)) *abort_flag = 1;
      phases ^= 1u << st;
      __syncthreads();
      if (*abort_flag) break;
    }
    unsigned char* a = sA + st * CV_A_BYTES;
    unsigned char* b = sB + st * CV_B_BYTES;
    // this thread's node: 64 (channel, tap) inputs of the chunk, 8 per 16-byte row
    int k = q * CV_KC;
    int c = k / 27, tap = k - 27 * (k / 27);
#pragma unroll 1
    for (int j = 0; j < CV_KC / 8; ++j) {
      uint32_t pk[4];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        float val = 0.0f;
        if (live && k < K) {
          const int ii = vi + tap / 9 - 1, jj = vj + (tap / 3) % 3 - 1, kk = vk + tap % 3 - 1;
          if ((unsigned)ii < (unsigned)g.nx && (unsigned)jj < (unsigned)g.ny && (unsigned)kk < (unsigned)g.nz)
            val = x[(long long)c * n + ((long long)ii * g.ny + jj) * g.nz + kk];
        }
        const uint32_t bits = __half_as_ushort(__float2half_rn(val));
        pk[e >> 1] = (e & 1) ? (pk[e >> 1] | (bits << 16)) : bits;   // element 2i in the low half
        ++k;
        if (++tap == 27) { tap = 0; ++c; }
      }
      *reinterpret_cast<uint4*>(a + (j * CV_M + t) * 16) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    }
    for (int piece = t; piece < np * (CV_KC / 8); piece += CV_THREADS) {
      const int row = piece / (CV_KC / 8), j = piece % (CV_KC / 8);
      *reinterpret_cast<uint4*>(b + (j * np + row) * 16) =
          *reinterpret_cast<const uint4*>(w16 + (long long)row * kp + q * CV_KC + 8 * j);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (t == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t aa = cv_smem(a), ba = cv_smem(b);
#pragma unroll
      for (int ks = 0; ks < CV_KC / 16; ++ks) {
        const uint64_t da = cv_desc(aa + 2 * ks * CV_M * 16, CV_M * 16, 128);
        const uint64_t db = cv_desc(ba + 2 * ks * np * 16, np * 16, 128);
        const uint32_t acc = (q > 0 || ks > 0) ? 1u : 0u;
        asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                     "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                     :: "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(cv_smem(&bars[st])) : "memory");
    }
  }
  if (!*abort_flag && chunks > 0) {
    // the last commit covers every MMA this thread issued
    const int st = (chunks - 1) & 1;
    if (!cv_wait(cv_smem(&bars[st]), (phases >> st) & 1u)) *abort_flag = 1;
    __syncthreads();
  }
  if (!*abort_flag) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    for (int c0 = 0; c0 < np; c0 += 16) {
      uint32_t r[16];
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                   : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
                     "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                   : "r"(tmem + (uint32_t(32 * warp) << 16) + c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (live) {
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          const int o = c0 + e;
          if (o < cout) {
            float val = __uint_as_float(r[e]) + bias[o];
            if (relu) val = fmaxf(val, 0.0f);
            y[(long long)o * n + v] = val;
          }
        }
      }
    }
  } else {
    if (t == 0) atomicExch(err, 1);
    // let MMAs still in flight finish before the TMEM is released (bounded)
    for (int st = 0; st < 2; ++st) cv_wait(cv_smem(&bars[st]), (phases >> st) & 1u);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(CV_TMEM));
}

// w16[o][k] = fp16(w[o][k]) for o < cout, k < K; zero padding up to [np][kp]
__global__ void pack16_kernel(const float* __restrict__ w, int cout, int K, __half* __restrict__ w16, int np, int kp) {
  const long long total = (long long)np * kp;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
    const int o = static_cast<int>(idx / kp), k = static_cast<int>(idx % kp);
    w16[idx] = __float2half_rn((o < cout && k < K) ? w[(long long)o * K + k] : 0.0f);
  }
}

}  // namespace

extern "C" const char* tf_nn_last_error(void) { return g_learn_error.c_str(); }

extern "C" int tf_nn_gemm(int32_t transa, int32_t transb, int32_t m, int32_t n, int32_t k, float alpha, const float* a, int32_t lda,
                          const float* b, int32_t ldb, float beta, float* c, int32_t ldc, float* work, int64_t work_floats,
                          void* stream) {
  return learn_guard([&] {
    require(m >= 0 && n >= 0 && k >= 0 && a && b && c && work, "tf_nn_gemm: invalid arguments");
    if (m == 0 || n == 0) return;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long tiles = (long long)((m + GT - 1) / GT) * ((n + GT - 1) / GT);
    int splits = 1;
    while (splits < 64 && tiles * splits < 2 * 148 && (long long)k / (2 * splits) >= 256) splits *= 2;
    while (splits > 1 && (long long)splits * m * n > work_floats) splits /= 2;
    require((long long)m * n <= work_floats, "tf_nn_gemm: workspace too small");
    const int kchunk = ((k + splits - 1) / splits + GK - 1) / GK * GK;
    dim3 grid((n + GT - 1) / GT, (m + GT - 1) / GT, splits);
    sgemm_kernel<<<grid, 256, 0, s>>>(transa, transb, m, n, k, a, lda, b, ldb, work, n, kchunk);
    TF_LAUNCH_CHECK("sgemm_kernel");
    sum_splits_kernel<<<grid_for((long long)m * n, 256), 256, 0, s>>>(work, splits, m, n, alpha, beta, c, ldc);
    TF_LAUNCH_CHECK("sum_splits_kernel");
  });
}

extern "C" int tf_nn_pack16(const float* w, int32_t cout, int32_t k, void* w16, int32_t np, int32_t kp, void* stream) {
  return learn_guard([&] {
    require(w && w16 && cout >= 1 && k >= 1, "tf_nn_pack16: invalid arguments");
    require(np >= cout && np % 16 == 0 && np <= CV_NMAX && kp >= k && kp % CV_KC == 0,
            "tf_nn_pack16: np must be a multiple of 16 in [cout, 64], kp a multiple of 64 >= k");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    pack16_kernel<<<grid_for((long long)np * kp, 256), 256, 0, s>>>(w, cout, k, static_cast<__half*>(w16), np, kp);
    TF_LAUNCH_CHECK("pack16_kernel");
  });
}

extern "C" int tf_nn_conv16(const float* x, int32_t cin, const int32_t shape[3], const void* w16, int32_t cout, int32_t np, int32_t kp,
                            const float* bias, int32_t relu, float* y, int32_t* err, void* stream) {
  return learn_guard([&] {
    require(x && shape && w16 && bias && y && err && cin >= 1 && cout >= 1, "tf_nn_conv16: invalid arguments");
    require(np >= cout && np % 16 == 0 && np <= CV_NMAX && kp >= 27 * cin && kp % CV_KC == 0,
            "tf_nn_conv16: np must be a multiple of 16 in [cout, 64], kp a multiple of 64 >= 27 cin");
    const Grid3 g = grid3(shape);
    require(g.nx >= 1 && g.ny >= 1 && g.nz >= 1, "tf_nn_conv16: empty grid");
    const long long blocks = (g.n() + CV_M - 1) / CV_M;
    require(blocks < (1LL << 31), "tf_nn_conv16: grid too large");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    static bool configured = false;
    if (!configured) {
      TF_CUDA_CHECK(cudaFuncSetAttribute(conv16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, CV_SMEM));
      configured = true;
    }
    conv16_kernel<<<(unsigned)blocks, CV_THREADS, CV_SMEM, s>>>(x, cin, g, static_cast<const __half*>(w16), cout, np, kp, bias, relu, y,
                                                                err);
    TF_LAUNCH_CHECK("conv16_kernel");
  });
}

extern "C" int tf_nn_im2col(const float* in, int32_t channels, const int32_t shape[3], float* col, void* stream) {
  return learn_guard([&] {
    require(in && col && shape && channels > 0, "tf_nn_im2col: invalid arguments");
    const Grid3 g = grid3(shape);
    im2col_kernel<<<grid_for((long long)channels * 27 * g.n(), 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(in, channels, g, col);
    TF_LAUNCH_CHECK("im2col_kernel");
  });
}

extern "C" int tf_nn_col2im(const float* col, int32_t channels, const int32_t shape[3], float* out, void* stream) {
  return learn_guard([&] {
    require(out && col && shape && channels > 0, "tf_nn_col2im: invalid arguments");
    const Grid3 g = grid3(shape);
    col2im_kernel<<<grid_for((long long)channels * g.n(), 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(col, channels, g, out);
    TF_LAUNCH_CHECK("col2im_kernel");
  });
}

extern "C" int tf_nn_bias_act(float* x, const float* bias, int32_t channels, int64_t n, int32_t relu, void* stream) {
  return learn_guard([&] {
    require(x && bias && channels > 0 && n >= 0, "tf_nn_bias_act: invalid arguments");
    bias_act_kernel<<<grid_for((long long)channels * n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(x, bias, channels, n, relu);
    TF_LAUNCH_CHECK("bias_act_kernel");
  });
}

extern "C" int tf_nn_act_back(float* dy, const float* y, int32_t channels, int64_t n, int32_t relu, float* dbias, int32_t accumulate,
                              void* stream) {
  return learn_guard([&] {
    require(dy && dbias && channels > 0 && (y || !relu), "tf_nn_act_back: invalid arguments");
    act_back_kernel<<<channels, RED_THREADS, 0, static_cast<cudaStream_t>(stream)>>>(dy, y, n, relu, dbias, accumulate);
    TF_LAUNCH_CHECK("act_back_kernel");
  });
}

extern "C" int tf_nn_pool(const float* in, int32_t channels, const int32_t fine[3], const int32_t coarse[3], float* out, void* stream) {
  return learn_guard([&] {
    const Grid3 f = grid3(fine), c = grid3(coarse);
    require(in && out && channels > 0 && c.nx == (f.nx + 1) / 2 && c.ny == (f.ny + 1) / 2 && c.nz == (f.nz + 1) / 2,
            "tf_nn_pool: invalid arguments");
    pool_kernel<<<grid_for((long long)channels * c.n(), 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(in, channels, f, c, out);
    TF_LAUNCH_CHECK("pool_kernel");
  });
}

/* mode 0: upsample forward; mode 1: pooling adjoint (fine = coarse / 8); mode 2: upsample adjoint (coarse = sum of children) */
extern "C" int tf_nn_resample(const float* in, int32_t channels, const int32_t fine[3], const int32_t coarse[3], int32_t mode, float* out,
                              void* stream) {
  return learn_guard([&] {
    const Grid3 f = grid3(fine), c = grid3(coarse);
    require(in && out && channels > 0 && mode >= 0 && mode <= 2 && c.nx == (f.nx + 1) / 2 && c.ny == (f.ny + 1) / 2 &&
            c.nz == (f.nz + 1) / 2, "tf_nn_resample: invalid arguments");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (mode == 2) {
      gather_children_kernel<<<grid_for((long long)channels * c.n(), 256), 256, 0, s>>>(in, channels, f, c, out);
      TF_LAUNCH_CHECK("gather_children_kernel");
    } else {
      spread_kernel<<<grid_for((long long)channels * f.n(), 256), 256, 0, s>>>(in, channels, f, c, out, mode == 1 ? 0.125f : 1.0f);
      TF_LAUNCH_CHECK("spread_kernel");
    }
  });
}

extern "C" int tf_nn_mse(const float* y, const float* target, const float* weight, int64_t n, double count, float* dy, double* scratch,
                         double* loss_dev, void* stream) {
  return learn_guard([&] {
    require(y && target && scratch && loss_dev && n > 0 && count > 0, "tf_nn_mse: invalid arguments");
    constexpr int BLOCKS = 296;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned* counter = reinterpret_cast<unsigned*>(scratch + 2 * BLOCKS);
    TF_CUDA_CHECK(cudaMemsetAsync(counter, 0, sizeof(unsigned), s));
    mse_kernel<<<BLOCKS, RED_THREADS, 0, s>>>(y, target, weight, n, static_cast<float>(1.0 / count), dy, scratch, counter, loss_dev);
    TF_LAUNCH_CHECK("mse_kernel");
  });
}

extern "C" int64_t tf_nn_mse_scratch_doubles(void) { return 2 * 296 + 1; }

extern "C" int tf_nn_adam(float* param, const float* grad, float* m, float* v, int64_t n, float lr, float beta1, float beta2, float eps,
                          int32_t step, void* stream) {
  return learn_guard([&] {
    require(param && grad && m && v && n >= 0 && step >= 1, "tf_nn_adam: invalid arguments");
    const float c1 = 1.0f - std::pow(beta1, (float)step), c2 = 1.0f - std::pow(beta2, (float)step);
    adam_kernel<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(param, grad, m, v, n, lr, beta1, beta2, eps, c1, c2);
    TF_LAUNCH_CHECK("adam_kernel");
  });
}
