// Shared host-side helpers of the sm_100a topology-optimisation library.
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

namespace tfb {

// Status codes returned by every extern "C" entry point (0 = ok).
enum Status : int {
  TF_OK = 0,
  TF_INVALID = 1,      // bad argument (maps to ValueError on the Python side)
  TF_CUDA = 2,         // CUDA runtime error
  TF_NOT_CONVERGED = 3,
  TF_NUMERIC = 4,      // numerical breakdown (non-SPD coarsest grid, NaN)
  TF_INTERNAL = 5,
};

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess)
    throw Error(TF_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
// Number of kernels this library has launched in the process (reported by tf_launch_count).
extern std::atomic<long long> g_launch_count;

#define TF_CUDA_CHECK(x) ::tfb::cuda_check((x), #x)
#define TF_LAUNCH_CHECK(name) \
  do {                                                  \
    ::tfb::g_launch_count.fetch_add(1, std::memory_order_relaxed); \
    ::tfb::cuda_check(cudaGetLastError(), name);        \
  } while (0)

// Store the message tf_last_error(NULL) returns (entry points without a handle).
void record_unhandled_error(const std::string& message);
// This thread's last such message (also what tf_filter/mma/chol_last_error(NULL) return).
const char* unhandled_error();

inline void require(bool ok, const std::string& m) {
  if (!ok) throw Error(TF_INVALID, m);
}

inline int grid_for(int64_t n, int block, int cap = 148 * 32) {
  int64_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return static_cast<int>(g);
}

// RAII device buffer.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  explicit DevBuf(size_t b) { alloc(b); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) { release(); p = o.p; bytes = o.bytes; o.p = nullptr; o.bytes = 0; }
    return *this;
  }
  ~DevBuf() { release(); }
  void alloc(size_t b) {
    release();
    if (b == 0) return;
    TF_CUDA_CHECK(cudaMalloc(&p, b));
    bytes = b;
  }
  // keep the current allocation when it already has exactly `b` bytes
  void ensure(size_t b) {
    if (p && bytes == b) return;
    alloc(b);
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

}  // namespace tfb
