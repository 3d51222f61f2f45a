// Cone density filter, its adjoint and the threshold projection (sm_100a).
//
// Replaces the reference's ConeFilter / DensityMap.filtered / .pullback /
// .project (deep_frame/topology_optimization.py:1082-1178).  The filter is a
// correlation with weights max(r - |offset * h|, 0) over the cells within the
// radius, restricted to allowed cells on both sides; the row sums are
// precomputed at creation (1 on forbidden cells).  One thread per cell reads its
// (2p+1)^3 neighbourhood through L1; a step is HBM-bound (about four FP64 streams
// per cell).
#include <cmath>
#include <string>
#include <vector>

#include "tf_b200.h"
#include "tf_common.h"

using namespace tfb;

namespace {
constexpr int PMAX = 4;                          // at most 9 x 9 x 9 taps
constexpr int WMAX = (2 * PMAX + 1) * (2 * PMAX + 1) * (2 * PMAX + 1);

struct FilterParam {
  double w[WMAX];
  int px, py, pz;
  int nx, ny, nz;
};

// out[i] = post[i] * sum_d w[d] * pre[i+d] * in[i+d] * in2[i+d]   (pre = allowed mask scaled, zero outside)
__global__ void filter_kernel(const __grid_constant__ FilterParam F, const double* __restrict__ in, const double* __restrict__ in2,
                              const double* __restrict__ pre, const double* __restrict__ post, double* __restrict__ out) {
  const long long total = (long long)F.nx * F.ny * F.nz;
  const int sy = 2 * F.py + 1, sz = 2 * F.pz + 1;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < total; c += (long long)gridDim.x * blockDim.x) {
    const int k = static_cast<int>(c % F.nz);
    const long long r = c / F.nz;
    const int j = static_cast<int>(r % F.ny), i = static_cast<int>(r / F.ny);
    double acc = 0.0;
    for (int a = -F.px; a <= F.px; ++a) {
      const int ii = i + a;
      if ((unsigned)ii >= (unsigned)F.nx) continue;
      for (int b = -F.py; b <= F.py; ++b) {
        const int jj = j + b;
        if ((unsigned)jj >= (unsigned)F.ny) continue;
        const double* wrow = F.w + ((a + F.px) * sy + (b + F.py)) * sz + F.pz;
        const long long base = ((long long)ii * F.ny + jj) * F.nz;
        for (int q = -F.pz; q <= F.pz; ++q) {
          const int kk = k + q;
          if ((unsigned)kk >= (unsigned)F.nz) continue;
          const double w = wrow[q];
          if (w == 0.0) continue;
          const long long s = base + kk;
          double v = pre[s] * in[s];
          if (in2) v *= in2[s];
          acc += w * v;
        }
      }
    }
    out[c] = post[c] * acc;
  }
}

// Threshold projection (DensityMap.project, topology_optimization.py:1152-1170).
__global__ void project_kernel(long long n, const double* __restrict__ filtered, const uint8_t* __restrict__ flags, double beta,
                               double eta, int robust, double* __restrict__ physical, double* __restrict__ derivative) {
  const double den = beta > 0.0 ? tanh(beta * eta) + tanh(beta * (1.0 - eta)) : 1.0;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const double f = filtered[c];
    double p, d;
    if (beta > 0.0 && robust) {
      const double shifted = beta * (f - eta);
      const double decay = exp(-2.0 * fabs(shifted));
      p = (tanh(beta * eta) + tanh(shifted)) / den;
      d = beta * 4.0 * decay / ((1.0 + decay) * (1.0 + decay)) / den;
    } else if (beta > 0.0) {
      const double t = tanh(beta * (f - eta));
      p = (tanh(beta * eta) + t) / den;
      d = beta * (1.0 - t * t) / den;
    } else {
      p = f;
      d = 1.0;
    }
    const unsigned fl = flags[c];   // bit 0 allowed, bit 1 preserve
    if (fl & 2u) p = 1.0;
    if (!(fl & 1u)) p = 0.0;
    if (!(fl & 1u) || (fl & 2u)) d = 0.0;
    physical[c] = fmin(fmax(p, 0.0), 1.0);
    if (derivative) derivative[c] = d;
  }
}
}  // namespace

struct tf_filter {
  FilterParam F{};
  long long n = 0;
  DevBuf mask, sums, post_fwd, post_adj, flags, ones;
  std::string err;
};

namespace {
template <typename Fn>
int filter_guard(tf_filter* h, Fn&& f) {
  try {
    f();
    return TF_OK;
  } catch (const Error& e) {
    if (h) h->err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    if (h) h->err = e.what();
    return TF_INTERNAL;
  }
}

__global__ void filter_post_kernel(long long n, const double* __restrict__ mask, const uint8_t* __restrict__ flags,
                                   double* __restrict__ sums, double* __restrict__ fwd, double* __restrict__ adj) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const bool allowed = flags[c] & 1u, preserve = flags[c] & 2u;
    const double s = allowed ? sums[c] : 1.0;
    sums[c] = s;
    fwd[c] = allowed ? 1.0 / s : 0.0;          // forward: mask / sums
    adj[c] = (allowed && !preserve) ? 1.0 : 0.0;   // pullback: free cells only
  }
}

__global__ void fill_kernel(double* __restrict__ v, long long n, double value) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) v[c] = value;
}
}  // namespace

extern "C" int tf_filter_create(const int64_t shape[3], const double spacing[3], double radius, const uint8_t* allowed,
                                const uint8_t* preserve, tf_filter** out) {
  if (!out) return TF_INVALID;
  *out = nullptr;
  tf_filter* h = new tf_filter();
  int rc = filter_guard(h, [&] {
    require(shape && spacing && allowed, "shape, spacing and allowed must not be NULL");
    require(std::isfinite(radius) && radius > 0, "filter radius must be finite and positive");
    int pads[3];
    for (int d = 0; d < 3; ++d) {
      require(shape[d] >= 1 && std::isfinite(spacing[d]) && spacing[d] > 0, "invalid filter grid");
      pads[d] = static_cast<int>(std::floor(radius / spacing[d]));
      require(pads[d] <= PMAX, "filter radius spans more than 4 cells; not supported");
    }
    FilterParam& F = h->F;
    F.px = pads[0]; F.py = pads[1]; F.pz = pads[2];
    F.nx = static_cast<int>(shape[0]); F.ny = static_cast<int>(shape[1]); F.nz = static_cast<int>(shape[2]);
    const int sy = 2 * F.py + 1, sz = 2 * F.pz + 1;
    for (int a = -F.px; a <= F.px; ++a)
      for (int b = -F.py; b <= F.py; ++b)
        for (int c = -F.pz; c <= F.pz; ++c) {
          const double dist = std::sqrt(std::pow(a * spacing[0], 2) + std::pow(b * spacing[1], 2) + std::pow(c * spacing[2], 2));
          F.w[((a + F.px) * sy + (b + F.py)) * sz + (c + F.pz)] = std::max(radius - dist, 0.0);
        }
    h->n = (long long)F.nx * F.ny * F.nz;
    const long long n = h->n;
    std::vector<uint8_t> fl(n);
    std::vector<double> m(n);
    for (long long c = 0; c < n; ++c) {
      const bool al = allowed[c] != 0, pr = preserve ? preserve[c] != 0 : false;
      require(!pr || al, "preserved cells must be allowed");
      fl[c] = static_cast<uint8_t>((al ? 1 : 0) | (pr ? 2 : 0));
      m[c] = al ? 1.0 : 0.0;
    }
    h->flags.alloc(n);
    h->mask.alloc(sizeof(double) * n);
    h->sums.alloc(sizeof(double) * n);
    h->post_fwd.alloc(sizeof(double) * n);
    h->post_adj.alloc(sizeof(double) * n);
    h->ones.alloc(sizeof(double) * n);
    TF_CUDA_CHECK(cudaMemcpy(h->flags.p, fl.data(), n, cudaMemcpyHostToDevice));
    TF_CUDA_CHECK(cudaMemcpy(h->mask.p, m.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    fill_kernel<<<grid_for(n, 256), 256>>>(h->ones.as<double>(), n, 1.0);
    TF_LAUNCH_CHECK("fill_kernel");
    // sums = mask * (W (mask * 1))
    filter_kernel<<<grid_for(n, 256), 256>>>(F, h->ones.as<double>(), nullptr, h->mask.as<double>(), h->mask.as<double>(),
                                             h->sums.as<double>());
    TF_LAUNCH_CHECK("filter_kernel");
    filter_post_kernel<<<grid_for(n, 256), 256>>>(n, h->mask.as<double>(), h->flags.as<uint8_t>(), h->sums.as<double>(),
                                                  h->post_fwd.as<double>(), h->post_adj.as<double>());
    TF_LAUNCH_CHECK("filter_post_kernel");
    TF_CUDA_CHECK(cudaDeviceSynchronize());
    std::vector<double> sums(n);
    TF_CUDA_CHECK(cudaMemcpy(sums.data(), h->sums.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
    for (double v : sums) require(v > 0.0, "Density filter contains an empty allowed-cell neighborhood");
  });
  if (rc != TF_OK) {
    record_unhandled_error(h->err);
    delete h;
    return rc;
  }
  *out = h;
  return TF_OK;
}

extern "C" int tf_filter_apply(tf_filter* h, const double* in_dev, const double* in2_dev, double* out_dev, int32_t adjoint,
                               void* stream) {
  if (!h) return TF_INVALID;
  return filter_guard(h, [&] {
    require(in_dev && out_dev && in_dev != out_dev, "tf_filter_apply: invalid buffers");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!adjoint) {
      // filtered = mask * (W (mask * x)) / sums    (DensityMap.filtered)
      filter_kernel<<<grid_for(h->n, 256), 256, 0, s>>>(h->F, in_dev, in2_dev, h->mask.as<double>(), h->post_fwd.as<double>(), out_dev);
    } else {
      // pullback = free * (W (mask * g * in2 / sums))   (DensityMap.pullback)
      filter_kernel<<<grid_for(h->n, 256), 256, 0, s>>>(h->F, in_dev, in2_dev, h->post_fwd.as<double>(), h->post_adj.as<double>(), out_dev);
    }
    TF_LAUNCH_CHECK("filter_kernel");
  });
}

extern "C" int tf_filter_sums(const tf_filter* h, double* sums_dev, void* stream) {
  if (!h || !sums_dev) return TF_INVALID;
  if (cudaMemcpyAsync(sums_dev, h->sums.p, sizeof(double) * h->n, cudaMemcpyDeviceToDevice, static_cast<cudaStream_t>(stream)) != cudaSuccess)
    return TF_CUDA;
  return TF_OK;
}

extern "C" int tf_filter_project(tf_filter* h, const double* filtered_dev, double beta, double eta, int32_t robust,
                                 double* physical_dev, double* derivative_dev, void* stream) {
  if (!h) return TF_INVALID;
  return filter_guard(h, [&] {
    require(filtered_dev && physical_dev, "tf_filter_project: NULL buffer");
    require(std::isfinite(beta) && beta >= 0 && eta > 0 && eta < 1, "invalid projection settings");
    project_kernel<<<grid_for(h->n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        h->n, filtered_dev, h->flags.as<uint8_t>(), beta, eta, robust, physical_dev, derivative_dev);
    TF_LAUNCH_CHECK("project_kernel");
  });
}

extern "C" int tf_filter_destroy(tf_filter* h) {
  if (h) {
    cudaDeviceSynchronize();
    delete h;
  }
  return TF_OK;
}

extern "C" const char* tf_filter_last_error(const tf_filter* h) { return h ? h->err.c_str() : ""; }
