// One launch over the blocks of several independent solver instances.
//
// A batched launch concatenates the instances' own grids: instance i owns the flat blocks
// [begin[i], begin[i+1]) of a one-dimensional grid, and each block recovers its instance and its
// place in that instance's grid g[i] (batch_locate), then runs the same kernel body as a plain
// launch with that VGrid and the instance's arguments (rec[i]).  The records travel in the kernel
// parameter space (up to 32 KB on sm_70 and later with CUDA 12.1+), so a launch needs no device
// table and no copy.
#pragma once
#include <cuda_runtime.h>
#include <utility>
#include <vector>
#include "tf_common.h"
#include "tf_reduce.cuh"

namespace tfb {

constexpr int BATCH_MAX = 32;   // instances per launch; more are split into further launches

template <class Rec>
struct Batch {
  int n;
  unsigned begin[BATCH_MAX + 1];
  dim3 g[BATCH_MAX];
  Rec rec[BATCH_MAX];
};

template <class Rec>
__device__ __forceinline__ int batch_locate(const Batch<Rec>& b, VGrid& vg) {
  const unsigned X = blockIdx.x;
  int i = 0;
  while (i + 1 < b.n && X >= b.begin[i + 1]) ++i;
  const dim3 g = b.g[i];
  unsigned loc = X - b.begin[i];
  vg.b.x = loc % g.x;
  loc /= g.x;
  vg.b.y = loc % g.y;
  vg.b.z = loc / g.y;
  vg.g = g;
  return i;
}

template <class Rec>
using BatchKernel = void (*)(const Batch<Rec>);

// Launch `k` once per BATCH_MAX items: items[i] = (the instance's own grid, its arguments).
template <class Rec>
void launch_batched(BatchKernel<Rec> k, const std::vector<std::pair<dim3, Rec>>& items, dim3 block, size_t smem, cudaStream_t s,
                    const char* name) {
  static_assert(sizeof(Batch<Rec>) <= 32000, "batched launch records exceed the kernel parameter space");
  for (size_t s0 = 0; s0 < items.size(); s0 += BATCH_MAX) {
    Batch<Rec> b{};
    b.n = static_cast<int>(std::min<size_t>(BATCH_MAX, items.size() - s0));
    unsigned long long total = 0;
    for (int i = 0; i < b.n; ++i) {
      const dim3 g = items[s0 + i].first;
      b.begin[i] = static_cast<unsigned>(total);
      b.g[i] = g;
      b.rec[i] = items[s0 + i].second;
      total += (unsigned long long)g.x * g.y * g.z;
    }
    if (total == 0) continue;
    if (total > 0x7fffffffull) throw Error(TF_INVALID, std::string(name) + ": batched grid too large");
    b.begin[b.n] = static_cast<unsigned>(total);
    k<<<static_cast<unsigned>(total), block, smem, s>>>(b);
    TF_LAUNCH_CHECK(name);
  }
}

}  // namespace tfb
