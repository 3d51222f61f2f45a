// Deterministic block and grid reductions shared by the solver and the density kernels.
#pragma once
#include <cuda_runtime.h>

namespace tfb {

constexpr int RED_THREADS = 256;

// The block's place in its launch.  Kernel bodies shared by a plain launch and a batched one (one
// launch over the blocks of several solver instances) take it as a parameter and shadow the
// built-in blockIdx / gridDim with it (TF_VGRID), so the body reads the same either way.
struct VGrid {
  uint3 b;
  dim3 g;
};
__device__ __forceinline__ VGrid vgrid() { return VGrid{blockIdx, gridDim}; }
#define TF_VGRID(vg)                 \
  const uint3 blockIdx = (vg).b;     \
  const dim3 gridDim = (vg).g;       \
  (void)blockIdx;                    \
  (void)gridDim

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide reduction of two values (op 0 = sum, 1 = max); result valid in thread 0.
template <int OP0, int OP1>
__device__ __forceinline__ void block_reduce2(double& a, double& b) {
  __shared__ double sa[RED_THREADS / 32], sb[RED_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  a = OP0 ? warp_max(a) : warp_sum(a);
  b = OP1 ? warp_max(b) : warp_sum(b);
  if (lane == 0) { sa[warp] = a; sb[warp] = b; }
  __syncthreads();
  if (warp == 0) {
    a = lane < RED_THREADS / 32 ? sa[lane] : 0.0;
    b = lane < RED_THREADS / 32 ? sb[lane] : 0.0;
    a = OP0 ? warp_max(a) : warp_sum(a);
    b = OP1 ? warp_max(b) : warp_sum(b);
  }
  __syncthreads();
}

// Deterministic cross-block combine: every block stores its partial; the last
// block of the column sums the partials in block order.  Returns true in
// thread 0 of the last block, with the totals in a, b.
// bx, gx: the block's index and the block count along x of its (possibly batched) launch.
template <int OP0, int OP1>
__device__ __forceinline__ bool last_block_combine(double& a, double& b, double* partial, unsigned* count, int col, unsigned bx,
                                                   unsigned gx) {
  __shared__ bool is_last;
  if (threadIdx.x == 0) {
    double* p = partial + 2 * ((long long)col * gx + bx);
    p[0] = a;
    p[1] = b;
    __threadfence();
    const unsigned t = atomicAdd(&count[col], 1u);
    is_last = (t == gx - 1);
  }
  __syncthreads();
  if (!is_last) return false;
  if (threadIdx.x != 0) return false;
  __threadfence();
  double ta = 0.0, tb = 0.0;
  const double* p = partial + 2 * (long long)col * gx;
  for (unsigned q = 0; q < gx; ++q) {
    const double pa = __ldcg(p + 2 * q), pb = __ldcg(p + 2 * q + 1);
    ta = OP0 ? fmax(ta, pa) : ta + pa;
    tb = OP1 ? fmax(tb, pb) : tb + pb;
  }
  count[col] = 0;
  a = ta;
  b = tb;
  return true;
}
template <int OP0, int OP1>
__device__ __forceinline__ bool last_block_combine(double& a, double& b, double* partial, unsigned* count, int col) {
  return last_block_combine<OP0, OP1>(a, b, partial, count, col, blockIdx.x, gridDim.x);
}

// Three values (op 0 = sum, 1 = max), block-wide; result valid in thread 0.
template <int OP0, int OP1, int OP2>
__device__ __forceinline__ void block_reduce3(double& a, double& b, double& c) {
  __shared__ double sa[RED_THREADS / 32], sb[RED_THREADS / 32], sc[RED_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  a = OP0 ? warp_max(a) : warp_sum(a);
  b = OP1 ? warp_max(b) : warp_sum(b);
  c = OP2 ? warp_max(c) : warp_sum(c);
  if (lane == 0) { sa[warp] = a; sb[warp] = b; sc[warp] = c; }
  __syncthreads();
  if (warp == 0) {
    a = lane < RED_THREADS / 32 ? sa[lane] : 0.0;
    b = lane < RED_THREADS / 32 ? sb[lane] : 0.0;
    c = lane < RED_THREADS / 32 ? sc[lane] : 0.0;
    a = OP0 ? warp_max(a) : warp_sum(a);
    b = OP1 ? warp_max(b) : warp_sum(b);
    c = OP2 ? warp_max(c) : warp_sum(c);
  }
  __syncthreads();
}

// last_block_combine for three values; partials stored as [col][block][4].
template <int OP0, int OP1, int OP2>
__device__ __forceinline__ bool last_block_combine3(double& a, double& b, double& c, double* partial, unsigned* count, int col,
                                                    unsigned bx, unsigned gx) {
  __shared__ bool is_last;
  if (threadIdx.x == 0) {
    double* p = partial + 4 * ((long long)col * gx + bx);
    p[0] = a;
    p[1] = b;
    p[2] = c;
    __threadfence();
    const unsigned t = atomicAdd(&count[col], 1u);
    is_last = (t == gx - 1);
  }
  __syncthreads();
  if (!is_last) return false;
  if (threadIdx.x != 0) return false;
  __threadfence();
  double ta = 0.0, tb = 0.0, tc = 0.0;
  const double* p = partial + 4 * (long long)col * gx;
  for (unsigned q = 0; q < gx; ++q) {
    const double pa = __ldcg(p + 4 * q), pb = __ldcg(p + 4 * q + 1), pc = __ldcg(p + 4 * q + 2);
    ta = OP0 ? fmax(ta, pa) : ta + pa;
    tb = OP1 ? fmax(tb, pb) : tb + pb;
    tc = OP2 ? fmax(tc, pc) : tc + pc;
  }
  count[col] = 0;
  a = ta;
  b = tb;
  c = tc;
  return true;
}
template <int OP0, int OP1, int OP2>
__device__ __forceinline__ bool last_block_combine3(double& a, double& b, double& c, double* partial, unsigned* count, int col) {
  return last_block_combine3<OP0, OP1, OP2>(a, b, c, partial, count, col, blockIdx.x, gridDim.x);
}

}  // namespace tfb
