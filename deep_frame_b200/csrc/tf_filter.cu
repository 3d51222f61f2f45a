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
#include "tf_reduce.cuh"

using namespace tfb;

namespace {
constexpr int PMAX = 4;                          // at most 9 x 9 x 9 taps
constexpr int WMAX = (2 * PMAX + 1) * (2 * PMAX + 1) * (2 * PMAX + 1);

struct FilterParam {
  double w[WMAX];
  int px, py, pz;
  int nx, ny, nz;
};

// sum_d w[d] * pre[i+d] * in[i+d] * in2[i+d] over the cone neighbourhood of cell c (zero outside the grid).
__device__ __forceinline__ double cone_sum(const FilterParam& F, long long c, const double* __restrict__ in,
                                           const double* __restrict__ in2, const double* __restrict__ pre) {
  const int sy = 2 * F.py + 1, sz = 2 * F.pz + 1;
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
  return acc;
}

// out[i] = post[i] * sum_d w[d] * pre[i+d] * in[i+d] * in2[i+d]   (pre = allowed mask scaled, zero outside)
__global__ void filter_kernel(const __grid_constant__ FilterParam F, const double* __restrict__ in, const double* __restrict__ in2,
                              const double* __restrict__ pre, const double* __restrict__ post, double* __restrict__ out) {
  const long long total = (long long)F.nx * F.ny * F.nz;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < total; c += (long long)gridDim.x * blockDim.x)
    out[c] = post[c] * cone_sum(F, c, in, in2, pre);
}

// Threshold projection of one cell (DensityMap.project, topology_optimization.py:1152-1170):
// single tanh, robust tanh (derivative through exp(-2|shift|) so it stays positive at high beta)
// or identity at beta = 0; preserves forced to 1, forbidden cells to 0, derivative zero off the free cells.
__device__ __forceinline__ double project_cell(double f, unsigned fl, double beta, double eta, int robust, double den, double* deriv) {
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
  if (fl & 2u) p = 1.0;              // bit 0 allowed, bit 1 preserve
  if (!(fl & 1u)) p = 0.0;
  if (!(fl & 1u) || (fl & 2u)) d = 0.0;
  if (deriv) *deriv = d;
  return fmin(fmax(p, 0.0), 1.0);
}

__device__ __forceinline__ double projection_denominator(double beta, double eta) {
  return beta > 0.0 ? tanh(beta * eta) + tanh(beta * (1.0 - eta)) : 1.0;
}

__global__ void project_kernel(long long n, const double* __restrict__ filtered, const uint8_t* __restrict__ flags, double beta,
                               double eta, int robust, double* __restrict__ physical, double* __restrict__ derivative) {
  const double den = projection_denominator(beta, eta);
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    double d;
    physical[c] = project_cell(filtered[c], flags[c], beta, eta, robust, den, &d);
    if (derivative) derivative[c] = d;
  }
}

// ---------------------------------------------------------------------------------------------
// Optimality-criteria update (_oc_update, topology_optimization.py:1197-1233), device resident.
// The bisection on the volume multiplier runs as a state machine in device memory: every round is
// one proposal kernel and one fused filter + projection + weighted-sum kernel whose last block
// (deterministic combine) compares the volume with the target and moves the bracket.  The host
// launches rounds in chunks and reads the phase once per chunk.
constexpr int OC_BLOCKS = 296;                    // fixed grid: the reductions are bitwise reproducible
enum OcPhase { OC_LOWEST = 0, OC_BRACKET = 1, OC_BISECT = 2, OC_DONE = 3 };
enum OcError { OC_OK = 0, OC_BAD_SENSITIVITY = 1, OC_NO_BRACKET = 2 };

struct OcState {
  double lower, upper, mult, maxdv, maxratio, volume;
  int phase, count, evaluations, lowest, error, pad;
};

__device__ __forceinline__ bool is_free(unsigned fl) { return (fl & 1u) && !(fl & 2u); }

// Validity of the sensitivities on the free cells and max(dV) (:1199-1202).
__global__ void __launch_bounds__(RED_THREADS) oc_check_kernel(long long n, const uint8_t* __restrict__ flags,
                                                               const double* __restrict__ df0, const double* __restrict__ dv,
                                                               double* partial, unsigned* count, OcState* st) {
  double mx = 0.0, bad = 0.0;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    if (!is_free(flags[c])) continue;
    const double v = dv[c], g = df0[c];
    if (!(isfinite(v) && v >= 0.0) || !isfinite(g)) bad = 1.0;
    else mx = fmax(mx, v);
  }
  block_reduce2<1, 1>(mx, bad);
  if (last_block_combine<1, 1>(mx, bad, partial, count, 0)) {
    st->maxdv = mx;
    st->error = (bad > 0.0 || !(mx > 0.0)) ? OC_BAD_SENSITIVITY : OC_OK;
  }
}

// ratios = max(1e-30, -dC / max(dV, 1e-12 max dV)), move-limited bounds (:1202-1205).
__global__ void __launch_bounds__(RED_THREADS) oc_prepare_kernel(long long n, const uint8_t* __restrict__ flags,
                                                                 const double* __restrict__ x, const double* __restrict__ df0,
                                                                 const double* __restrict__ dv, double minimum, double move,
                                                                 double* __restrict__ ratio, double* __restrict__ lo,
                                                                 double* __restrict__ hi, double* partial, unsigned* count,
                                                                 OcState* st) {
  if (st->error) return;
  const double floor_dv = 1e-12 * st->maxdv;
  double mr = 0.0, z = 0.0;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    if (!is_free(flags[c])) continue;
    const double r = fmax(1e-30, -df0[c] / fmax(dv[c], floor_dv));
    ratio[c] = r;
    lo[c] = fmax(minimum, x[c] - move);
    hi[c] = fmin(1.0, x[c] + move);
    mr = fmax(mr, r);
  }
  block_reduce2<1, 0>(mr, z);
  if (last_block_combine<1, 0>(mr, z, partial, count, 0)) {
    st->maxratio = mr;
    st->phase = OC_LOWEST;
  }
}

// proposal(multiplier): free cells clip(x sqrt(ratio / max(multiplier, 1e-100)), lo, hi) (:1206-1209);
// the lowest design (free cells at lo) in the first round; final = 1 writes the accepted candidate.
__global__ void oc_proposal_kernel(long long n, const uint8_t* __restrict__ flags, const double* __restrict__ x,
                                   const double* __restrict__ ratio, const double* __restrict__ lo, const double* __restrict__ hi,
                                   const OcState* st, double* __restrict__ out, int final) {
  const int phase = st->phase;
  if (st->error || (!final && phase == OC_DONE)) return;
  const bool lowest = final ? st->lowest != 0 : phase == OC_LOWEST;
  const double m = fmax(final ? st->upper : st->mult, 1e-100);
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    if (!is_free(flags[c])) {
      out[c] = x[c];
    } else {
      out[c] = lowest ? lo[c] : fmin(fmax(x[c] * sqrt(ratio[c] / m), lo[c]), hi[c]);
    }
  }
}

// Weighted volume sum(w * project(filtered(p), eta)) (DensityMap.volume, :1146-1151), fused; with a state
// it also advances the multiplier search (:1210-1232).
__global__ void __launch_bounds__(RED_THREADS) volume_kernel(const __grid_constant__ FilterParam F, long long n,
                                                             const uint8_t* __restrict__ flags, const double* __restrict__ mask,
                                                             const double* __restrict__ post, const double* __restrict__ p,
                                                             const double* __restrict__ weights, double beta, double eta, int robust,
                                                             double target, double* partial, unsigned* count, OcState* st,
                                                             double* out) {
  if (st && (st->error || st->phase == OC_DONE)) return;
  const double den = projection_denominator(beta, eta);
  double acc = 0.0, z = 0.0;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const double f = post[c] * cone_sum(F, c, p, nullptr, mask);
    const double ph = project_cell(f, flags[c], beta, eta, robust, den, nullptr);
    acc += (weights ? weights[c] : 1.0) * ph;
  }
  block_reduce2<0, 0>(acc, z);
  if (!last_block_combine<0, 0>(acc, z, partial, count, 0)) return;
  if (!st) {
    *out = acc;
    return;
  }
  OcState& s = *st;
  s.volume = acc;
  s.evaluations += 1;
  if (s.phase == OC_LOWEST) {
    if (acc > target) {                       // even the lowest design is too heavy: take it
      s.lowest = 1;
      s.phase = OC_DONE;
    } else {
      s.upper = fmax(s.maxratio, 1e-12);
      s.count = 0;
      s.mult = s.upper;
      s.phase = OC_BRACKET;
    }
  } else if (s.phase == OC_BRACKET) {         // double the multiplier until the volume fits
    if (acc <= target + 1e-9) {
      s.lower = 0.0;
      s.count = 0;
      s.mult = (s.lower + s.upper) / 2;
      s.phase = OC_BISECT;
    } else {
      s.upper *= 2.0;
      s.count += 1;
      if (s.count >= 100) {
        s.error = OC_NO_BRACKET;
        s.phase = OC_DONE;
      } else {
        s.mult = s.upper;
      }
    }
  } else {                                    // bisection; the candidate is proposal(upper)
    if (acc > target) s.lower = s.mult;
    else s.upper = s.mult;
    s.count += 1;
    if ((s.upper - s.lower) / fmax(s.upper + s.lower, 1e-100) < 1e-8 || s.count >= 70) s.phase = OC_DONE;
    else s.mult = (s.lower + s.upper) / 2;
  }
}
}  // namespace

struct tf_filter {
  FilterParam F{};
  long long n = 0;
  DevBuf mask, sums, post_fwd, post_adj, flags, ones;
  DevBuf ratio, lo, hi, proposal, state, partial, count;   // optimality-criteria workspace
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

extern "C" const char* tf_filter_last_error(const tf_filter* h) { return h ? h->err.c_str() : unhandled_error(); }

namespace {
void ensure_reduction(tf_filter* h, cudaStream_t s) {
  if (!h->partial.p) {
    h->partial.alloc(sizeof(double) * 2 * OC_BLOCKS);
    h->count.alloc(sizeof(unsigned));
    h->state.alloc(sizeof(OcState));
    TF_CUDA_CHECK(cudaMemsetAsync(h->count.p, 0, sizeof(unsigned), s));
  }
}
}  // namespace

extern "C" int tf_filter_volume(tf_filter* h, const double* design_dev, const double* weights_dev, double beta, double eta,
                                int32_t robust, double* volume_dev, void* stream) {
  if (!h) return TF_INVALID;
  return filter_guard(h, [&] {
    require(design_dev && volume_dev, "tf_filter_volume: NULL buffer");
    require(std::isfinite(beta) && beta >= 0 && eta > 0 && eta < 1, "invalid projection settings");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ensure_reduction(h, s);
    volume_kernel<<<OC_BLOCKS, RED_THREADS, 0, s>>>(h->F, h->n, h->flags.as<uint8_t>(), h->mask.as<double>(),
                                                    h->post_fwd.as<double>(), design_dev, weights_dev, beta, eta, robust, 0.0,
                                                    h->partial.as<double>(), h->count.as<unsigned>(), nullptr, volume_dev);
    TF_LAUNCH_CHECK("volume_kernel");
  });
}

extern "C" int tf_oc_update(tf_filter* h, const double* design_dev, const double* objective_derivative_dev,
                            const double* volume_derivative_dev, const double* weights_dev, double target, double minimum_density,
                            double move_limit, double beta, double eta, int32_t robust, double* candidate_dev, tf_oc_report* report,
                            void* stream) {
  if (!h) return TF_INVALID;
  return filter_guard(h, [&] {
    require(design_dev && objective_derivative_dev && volume_derivative_dev && candidate_dev, "tf_oc_update: NULL buffer");
    require(candidate_dev != design_dev, "tf_oc_update: candidate must not alias the design");
    require(std::isfinite(target), "tf_oc_update: target must be finite");
    require(std::isfinite(minimum_density) && minimum_density >= 0 && minimum_density < 1, "invalid minimum_design_density");
    require(std::isfinite(move_limit) && move_limit > 0 && move_limit <= 1, "invalid move limit");
    require(std::isfinite(beta) && beta >= 0 && eta > 0 && eta < 1, "invalid projection settings");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long n = h->n;
    ensure_reduction(h, s);
    h->ratio.ensure(sizeof(double) * n);
    h->lo.ensure(sizeof(double) * n);
    h->hi.ensure(sizeof(double) * n);
    h->proposal.ensure(sizeof(double) * n);
    OcState* st = h->state.as<OcState>();
    const uint8_t* fl = h->flags.as<uint8_t>();
    TF_CUDA_CHECK(cudaMemsetAsync(st, 0, sizeof(OcState), s));
    oc_check_kernel<<<OC_BLOCKS, RED_THREADS, 0, s>>>(n, fl, objective_derivative_dev, volume_derivative_dev,
                                                      h->partial.as<double>(), h->count.as<unsigned>(), st);
    TF_LAUNCH_CHECK("oc_check_kernel");
    oc_prepare_kernel<<<OC_BLOCKS, RED_THREADS, 0, s>>>(n, fl, design_dev, objective_derivative_dev, volume_derivative_dev,
                                                        minimum_density, move_limit, h->ratio.as<double>(), h->lo.as<double>(),
                                                        h->hi.as<double>(), h->partial.as<double>(), h->count.as<unsigned>(), st);
    TF_LAUNCH_CHECK("oc_prepare_kernel");
    // 1 lowest-design check + at most 100 bracketing and 70 bisection rounds (:1213-1232)
    constexpr int MAX_ROUNDS = 171, CHUNK = 8;
    OcState host{};
    for (int done = 0; done < MAX_ROUNDS;) {
      const int rounds = std::min(CHUNK, MAX_ROUNDS - done);
      for (int r = 0; r < rounds; ++r) {
        oc_proposal_kernel<<<OC_BLOCKS, RED_THREADS, 0, s>>>(n, fl, design_dev, h->ratio.as<double>(), h->lo.as<double>(),
                                                             h->hi.as<double>(), st, h->proposal.as<double>(), 0);
        TF_LAUNCH_CHECK("oc_proposal_kernel");
        volume_kernel<<<OC_BLOCKS, RED_THREADS, 0, s>>>(h->F, n, fl, h->mask.as<double>(), h->post_fwd.as<double>(),
                                                        h->proposal.as<double>(), weights_dev, beta, eta, robust, target,
                                                        h->partial.as<double>(), h->count.as<unsigned>(), st, nullptr);
        TF_LAUNCH_CHECK("volume_kernel");
      }
      done += rounds;
      TF_CUDA_CHECK(cudaMemcpyAsync(&host, st, sizeof(OcState), cudaMemcpyDeviceToHost, s));
      TF_CUDA_CHECK(cudaStreamSynchronize(s));
      if (host.error || host.phase == OC_DONE) break;
    }
    if (host.error == OC_BAD_SENSITIVITY) throw Error(TF_NUMERIC, "Invalid OC sensitivities");
    if (host.error == OC_NO_BRACKET) throw Error(TF_NUMERIC, "OC could not bracket the volume multiplier");
    if (host.phase != OC_DONE) throw Error(TF_INTERNAL, "OC multiplier search did not finish");
    oc_proposal_kernel<<<OC_BLOCKS, RED_THREADS, 0, s>>>(n, fl, design_dev, h->ratio.as<double>(), h->lo.as<double>(),
                                                         h->hi.as<double>(), st, candidate_dev, 1);
    TF_LAUNCH_CHECK("oc_proposal_kernel");
    if (report) {
      report->multiplier = host.lowest ? 0.0 : host.upper;
      report->lower = host.lower;
      report->volume = host.volume;
      report->evaluations = host.evaluations;
      report->lowest = host.lowest;
    }
  });
}
