// Method of moving asymptotes: one subproblem step on the device (sm_100a).
//
// Replaces mmapy.mmasub as called from deep_frame/topology_optimizers.py:61-63
// (asymptotes, move limits, convex approximations and the primal-dual
// interior-point subproblem solver of K. Svanberg's method).  Every per-variable
// quantity (x, the asymptotes, p0/q0, P/Q, the dual slacks xsi/eta, Newton
// directions) lives in HBM; each Newton iteration is three passes over the n
// variables whose per-constraint sums (m <= TF_MMA_MAX_M) are reduced in a
// fixed order, so the step is bitwise reproducible.  The (m+1) x (m+1) dual
// system and the m-sized variables stay on the host.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "tf_b200.h"
#include "tf_common.h"

using namespace tfb;

namespace {
constexpr int MMAX = TF_MMA_MAX_M;               // constraints handled by the device path
constexpr int NSUM = 2 * MMAX + MMAX * (MMAX + 1) / 2;
constexpr int MMA_BLOCKS = 296;
constexpr int MMA_THREADS = 256;

struct Duals {
  double lam[MMAX];
  double dlam[MMAX];
  int m;
  double epsi;
  double step;
};

// Block sum of K values per thread into partial[blockIdx.x][K] (thread 0 writes).
template <int K>
__device__ __forceinline__ void block_sums(double (&v)[K], double* partial) {
  __shared__ double sh[MMA_THREADS / 32][K];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < K; ++q) {
    double x = v[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) sh[warp][q] = x;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < K; q += blockDim.x) {
    double x = 0.0;
    for (int w = 0; w < MMA_THREADS / 32; ++w) x += sh[w][q];
    partial[(long long)blockIdx.x * K + q] = x;
  }
}

template <int K>
__device__ __forceinline__ void block_maxes(double (&v)[K], double* partial) {
  __shared__ double sh[MMA_THREADS / 32][K];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < K; ++q) {
    double x = v[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
    if (lane == 0) sh[warp][q] = x;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < K; q += blockDim.x) {
    double x = -INFINITY;
    for (int w = 0; w < MMA_THREADS / 32; ++w) x = fmax(x, sh[w][q]);
    partial[(long long)blockIdx.x * K + q] = x;
  }
}

__global__ void combine_kernel(const double* __restrict__ partial, int blocks, int k, int use_max, double* __restrict__ out) {
  for (int q = threadIdx.x; q < k; q += blockDim.x) {
    double s = use_max ? -INFINITY : 0.0;
    for (int b = 0; b < blocks; ++b) {
      const double v = partial[(long long)b * k + q];
      s = use_max ? fmax(s, v) : s + v;
    }
    out[q] = s;
  }
}

struct Vec {
  double *x, *xmin, *xmax, *xold1, *xold2, *low, *upp, *df0dx, *alfa, *beta, *p0, *q0, *P, *Q, *xsi, *eta, *xo, *xsio, *etao,
      *delx, *diagx, *dx, *dxsi, *deta;
  long long n;
};

// Asymptotes, move limits and the convex approximation; partial sums of b = P/ux + Q/xl.
__global__ void __launch_bounds__(MMA_THREADS) mma_setup_kernel(Vec v, const double* __restrict__ dfdx, int m, int iteration,
                                                                 double move, double asyinit, double asydecr, double asyincr,
                                                                 double asymin, double asymax, double raa0, double albefa,
                                                                 double* partial) {
  double acc[MMAX];
#pragma unroll
  for (int i = 0; i < MMAX; ++i) acc[i] = 0.0;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < v.n; j += (long long)gridDim.x * blockDim.x) {
    const double x = v.x[j], xmin = v.xmin[j], xmax = v.xmax[j];
    const double span = xmax - xmin;
    double low, upp;
    if (iteration <= 2) {
      low = x - asyinit * span;
      upp = x + asyinit * span;
    } else {
      const double o1 = v.xold1[j], o2 = v.xold2[j];
      const double trend = (x - o1) * (o1 - o2);
      const double f = trend > 0.0 ? asyincr : (trend < 0.0 ? asydecr : 1.0);
      low = x - f * (o1 - v.low[j]);
      upp = x + f * (v.upp[j] - o1);
      low = fmin(fmax(low, x - asymax * span), x - asymin * span);
      upp = fmin(fmax(upp, x + asymin * span), x + asymax * span);
    }
    v.low[j] = low;
    v.upp[j] = upp;
    const double alfa = fmax(fmax(low + albefa * (x - low), x - move * span), xmin);
    const double beta = fmin(fmin(upp - albefa * (upp - x), x + move * span), xmax);
    v.alfa[j] = alfa;
    v.beta[j] = beta;
    const double ux1 = upp - x, xl1 = x - low, ux2 = ux1 * ux1, xl2 = xl1 * xl1;
    const double raa = raa0 / fmax(span, 1e-5);
    const double g0 = v.df0dx[j];
    double p0 = fmax(g0, 0.0), q0 = fmax(-g0, 0.0);
    const double pq0 = 0.001 * (p0 + q0) + raa;
    v.p0[j] = (p0 + pq0) * ux2;
    v.q0[j] = (q0 + pq0) * xl2;
    for (int i = 0; i < m; ++i) {
      const double g = dfdx[(long long)i * v.n + j];
      const double p = fmax(g, 0.0), q = fmax(-g, 0.0);
      const double pq = 0.001 * (p + q) + raa;
      const double P = (p + pq) * ux2, Q = (q + pq) * xl2;
      v.P[(long long)i * v.n + j] = P;
      v.Q[(long long)i * v.n + j] = Q;
      acc[i] += P / ux1 + Q / xl1;
    }
    // subproblem start point (Svanberg's subsolv initialisation)
    const double xs = 0.5 * (alfa + beta);
    v.x[j] = xs;   // x now holds the subproblem iterate; the caller keeps xval separately
    v.xsi[j] = fmax(1.0 / (xs - alfa), 1.0);
    v.eta[j] = fmax(1.0 / (beta - xs), 1.0);
  }
  block_sums<MMAX>(acc, partial);
}

// KKT residual terms over the n variables: sum of squares and max |.| of
// rex, rexsi, reeta, and the constraint sums gvec_i = sum P_ij/ux + Q_ij/xl.
__global__ void __launch_bounds__(MMA_THREADS) mma_residual_kernel(Vec v, Duals d, double* partial) {
  double acc[MMAX + 2];
#pragma unroll
  for (int i = 0; i < MMAX + 2; ++i) acc[i] = 0.0;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < v.n; j += (long long)gridDim.x * blockDim.x) {
    const double x = v.x[j];
    const double ux1 = v.upp[j] - x, xl1 = x - v.low[j];
    const double uxi = 1.0 / ux1, xli = 1.0 / xl1;
    double plam = v.p0[j], qlam = v.q0[j];
    for (int i = 0; i < d.m; ++i) {
      const double P = v.P[(long long)i * v.n + j], Q = v.Q[(long long)i * v.n + j];
      plam += d.lam[i] * P;
      qlam += d.lam[i] * Q;
      acc[i] += P * uxi + Q * xli;
    }
    const double dpsidx = plam * uxi * uxi - qlam * xli * xli;
    const double xsi = v.xsi[j], eta = v.eta[j];
    const double rex = dpsidx - xsi + eta;
    const double rexsi = xsi * (x - v.alfa[j]) - d.epsi;
    const double reeta = eta * (v.beta[j] - x) - d.epsi;
    acc[MMAX] += rex * rex + rexsi * rexsi + reeta * reeta;
    acc[MMAX + 1] = fmax(acc[MMAX + 1], fmax(fabs(rex), fmax(fabs(rexsi), fabs(reeta))));
  }
  // the max slot is reduced as a sum of per-thread maxima would be wrong: reduce it separately
  double sums[MMAX + 1];
#pragma unroll
  for (int i = 0; i < MMAX + 1; ++i) sums[i] = acc[i];
  block_sums<MMAX + 1>(sums, partial);
  __syncthreads();
  double mx[1] = {acc[MMAX + 1]};
  block_maxes<1>(mx, partial + (long long)gridDim.x * (MMAX + 1));
}

// Newton system terms: delx, diagx per variable (kept), and the sums
// gvec_i, (GG delx/diagx)_i and (GG diag(1/diagx) GG^T)_ik.  Saves the start point.
__global__ void __launch_bounds__(MMA_THREADS) mma_newton_kernel(Vec v, Duals d, double* partial) {
  double acc[NSUM];
#pragma unroll
  for (int i = 0; i < NSUM; ++i) acc[i] = 0.0;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < v.n; j += (long long)gridDim.x * blockDim.x) {
    const double x = v.x[j];
    v.xo[j] = x;
    v.xsio[j] = v.xsi[j];
    v.etao[j] = v.eta[j];
    const double ux1 = v.upp[j] - x, xl1 = x - v.low[j];
    const double ux2 = ux1 * ux1, xl2 = xl1 * xl1, ux3 = ux1 * ux2, xl3 = xl1 * xl2;
    double plam = v.p0[j], qlam = v.q0[j];
    double gg[MMAX];
#pragma unroll
    for (int i = 0; i < MMAX; ++i) {
      gg[i] = 0.0;
      if (i < d.m) {
        const double P = v.P[(long long)i * v.n + j], Q = v.Q[(long long)i * v.n + j];
        plam += d.lam[i] * P;
        qlam += d.lam[i] * Q;
        acc[i] += P / ux1 + Q / xl1;
        gg[i] = P / ux2 - Q / xl2;
      }
    }
    const double xa = x - v.alfa[j], bx = v.beta[j] - x;
    const double dpsidx = plam / ux2 - qlam / xl2;
    const double delx = dpsidx - d.epsi / xa + d.epsi / bx;
    const double diagx = 2.0 * (plam / ux3 + qlam / xl3) + v.xsi[j] / xa + v.eta[j] / bx;
    v.delx[j] = delx;
    v.diagx[j] = diagx;
    const double t = delx / diagx;
    int q = 2 * MMAX;
#pragma unroll
    for (int i = 0; i < MMAX; ++i) {
      if (i < d.m) acc[MMAX + i] += gg[i] * t;
#pragma unroll
      for (int k = 0; k <= i; ++k, ++q)
        if (i < d.m) acc[q] += gg[i] * gg[k] / diagx;
    }
  }
  block_sums<NSUM>(acc, partial);
}

// dx, dxsi, deta and the step-length maxima.
__global__ void __launch_bounds__(MMA_THREADS) mma_direction_kernel(Vec v, Duals d, double* partial) {
  double mx[1] = {-INFINITY};
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < v.n; j += (long long)gridDim.x * blockDim.x) {
    const double x = v.x[j];
    const double ux1 = v.upp[j] - x, xl1 = x - v.low[j];
    const double ux2 = ux1 * ux1, xl2 = xl1 * xl1;
    double gtd = 0.0;
    for (int i = 0; i < d.m; ++i) {
      const double gg = v.P[(long long)i * v.n + j] / ux2 - v.Q[(long long)i * v.n + j] / xl2;
      gtd += gg * d.dlam[i];
    }
    const double diagx = v.diagx[j];
    const double dx = -v.delx[j] / diagx - gtd / diagx;
    const double xa = x - v.alfa[j], bx = v.beta[j] - x;
    const double xsi = v.xsi[j], eta = v.eta[j];
    const double dxsi = -xsi + d.epsi / xa - xsi * dx / xa;
    const double deta = -eta + d.epsi / bx + eta * dx / bx;
    v.dx[j] = dx;
    v.dxsi[j] = dxsi;
    v.deta[j] = deta;
    mx[0] = fmax(mx[0], fmax(fmax(-1.01 * dxsi / xsi, -1.01 * deta / eta), fmax(-1.01 * dx / xa, 1.01 * dx / bx)));
  }
  block_maxes<1>(mx, partial);
}

__global__ void mma_trial_kernel(Vec v, double step) {
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < v.n; j += (long long)gridDim.x * blockDim.x) {
    v.x[j] = v.xo[j] + step * v.dx[j];
    v.xsi[j] = v.xsio[j] + step * v.dxsi[j];
    v.eta[j] = v.etao[j] + step * v.deta[j];
  }
}

// Dense (m+1) solve with partial pivoting on the host.
bool solve_small(std::vector<double>& a, std::vector<double>& b, int n) {
  for (int c = 0; c < n; ++c) {
    int p = c;
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(a[r * n + c]) > std::fabs(a[p * n + c])) p = r;
    if (a[p * n + c] == 0.0) return false;
    if (p != c) {
      for (int k = 0; k < n; ++k) std::swap(a[c * n + k], a[p * n + k]);
      std::swap(b[c], b[p]);
    }
    for (int r = c + 1; r < n; ++r) {
      const double f = a[r * n + c] / a[c * n + c];
      for (int k = c; k < n; ++k) a[r * n + k] -= f * a[c * n + k];
      b[r] -= f * b[c];
    }
  }
  for (int c = n - 1; c >= 0; --c) {
    double s = b[c];
    for (int k = c + 1; k < n; ++k) s -= a[c * n + k] * b[k];
    b[c] = s / a[c * n + c];
  }
  return true;
}

}  // namespace

struct tf_mma {
  int m = 0;
  long long n = 0;
  DevBuf x, xmin, xmax, xold1, xold2, low, upp, df0dx, alfa, beta, p0, q0, P, Q, xsi, eta, xo, xsio, etao, delx, diagx, dx, dxsi,
      deta, partial, sums;
  double* host = nullptr;   // pinned reduction results
  std::string err;
  ~tf_mma() {
    if (host) cudaFreeHost(host);
  }
  Vec vec() {
    Vec v;
    v.x = x.as<double>(); v.xmin = xmin.as<double>(); v.xmax = xmax.as<double>(); v.xold1 = xold1.as<double>();
    v.xold2 = xold2.as<double>(); v.low = low.as<double>(); v.upp = upp.as<double>(); v.df0dx = df0dx.as<double>();
    v.alfa = alfa.as<double>(); v.beta = beta.as<double>(); v.p0 = p0.as<double>(); v.q0 = q0.as<double>();
    v.P = P.as<double>(); v.Q = Q.as<double>(); v.xsi = xsi.as<double>(); v.eta = eta.as<double>(); v.xo = xo.as<double>();
    v.xsio = xsio.as<double>(); v.etao = etao.as<double>(); v.delx = delx.as<double>(); v.diagx = diagx.as<double>();
    v.dx = dx.as<double>(); v.dxsi = dxsi.as<double>(); v.deta = deta.as<double>(); v.n = n;
    return v;
  }
};

namespace {
template <typename F>
int mma_guard(tf_mma* h, F&& f) {
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

int blocks_for(long long n) { return static_cast<int>(std::max<long long>(1, std::min<long long>(MMA_BLOCKS, (n + MMA_THREADS - 1) / MMA_THREADS))); }

// Reduce `k` per-block values (sum or max) and copy them to the pinned host buffer.
void fetch(tf_mma* h, int blocks, int k, int use_max, long long offset, double* dst, cudaStream_t s) {
  combine_kernel<<<1, 256, 0, s>>>(h->partial.as<double>() + offset, blocks, k, use_max, h->sums.as<double>());
  TF_LAUNCH_CHECK("combine_kernel");
  TF_CUDA_CHECK(cudaMemcpyAsync(dst, h->sums.p, sizeof(double) * k, cudaMemcpyDeviceToHost, s));
}
}  // namespace

extern "C" int tf_mma_create(int32_t m, int64_t n, tf_mma** out) {
  if (!out) return TF_INVALID;
  *out = nullptr;
  tf_mma* h = new tf_mma();
  int rc = mma_guard(h, [&] {
    require(m >= 1 && m <= MMAX, "the device MMA handles 1 to 8 constraints");
    require(n >= 1, "n must be positive");
    h->m = m;
    h->n = n;
    const size_t nb = sizeof(double) * n;
    for (DevBuf* b : {&h->x, &h->xmin, &h->xmax, &h->xold1, &h->xold2, &h->low, &h->upp, &h->df0dx, &h->alfa, &h->beta, &h->p0,
                      &h->q0, &h->xsi, &h->eta, &h->xo, &h->xsio, &h->etao, &h->delx, &h->diagx, &h->dx, &h->dxsi, &h->deta})
      b->alloc(nb);
    h->P.alloc(nb * m);
    h->Q.alloc(nb * m);
    h->partial.alloc(sizeof(double) * MMA_BLOCKS * (NSUM + 2));
    h->sums.alloc(sizeof(double) * (NSUM + 2));
    TF_CUDA_CHECK(cudaMallocHost(&h->host, sizeof(double) * 4 * (NSUM + 2)));
  });
  if (rc != TF_OK) {
    record_unhandled_error(h->err);
    delete h;
    return rc;
  }
  *out = h;
  return TF_OK;
}

extern "C" int tf_mma_destroy(tf_mma* h) {
  if (h) {
    cudaDeviceSynchronize();
    delete h;
  }
  return TF_OK;
}

extern "C" const char* tf_mma_last_error(const tf_mma* h) { return h ? h->err.c_str() : unhandled_error(); }

extern "C" int tf_mma_step(tf_mma* h, int32_t iteration, const double* xval, const double* xmin, const double* xmax,
                           const double* xold1, const double* xold2, const double* df0dx, const double* fval, const double* dfdx,
                           double* low, double* upp, double a0, const double* a, const double* c, const double* d,
                           const tf_mma_settings* settings, double* xnew, double* y_out, double* z_out, double* lam_out,
                           int32_t* newton_iterations, void* stream) {
  if (!h) return TF_INVALID;
  return mma_guard(h, [&] {
    require(xval && xmin && xmax && xold1 && xold2 && df0dx && fval && dfdx && low && upp && a && c && d && xnew,
            "tf_mma_step: NULL argument");
    tf_mma_settings s = settings ? *settings : tf_mma_settings{0.5, 0.5, 0.7, 1.2, 0.01, 10.0, 1e-5, 0.1, 1e-7};
    const int m = h->m;
    const long long n = h->n;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t nb = sizeof(double) * n;
    TF_CUDA_CHECK(cudaMemcpyAsync(h->x.p, xval, nb, cudaMemcpyDeviceToDevice, st));
    TF_CUDA_CHECK(cudaMemcpyAsync(h->xmin.p, xmin, nb, cudaMemcpyDeviceToDevice, st));
    TF_CUDA_CHECK(cudaMemcpyAsync(h->xmax.p, xmax, nb, cudaMemcpyDeviceToDevice, st));
    TF_CUDA_CHECK(cudaMemcpyAsync(h->xold1.p, xold1, nb, cudaMemcpyDeviceToDevice, st));
    TF_CUDA_CHECK(cudaMemcpyAsync(h->xold2.p, xold2, nb, cudaMemcpyDeviceToDevice, st));
    TF_CUDA_CHECK(cudaMemcpyAsync(h->low.p, low, nb, cudaMemcpyDeviceToDevice, st));
    TF_CUDA_CHECK(cudaMemcpyAsync(h->upp.p, upp, nb, cudaMemcpyDeviceToDevice, st));
    TF_CUDA_CHECK(cudaMemcpyAsync(h->df0dx.p, df0dx, nb, cudaMemcpyDeviceToDevice, st));
    Vec v = h->vec();
    const int blocks = blocks_for(n);
    mma_setup_kernel<<<blocks, MMA_THREADS, 0, st>>>(v, dfdx, m, iteration, s.move, s.asyinit, s.asydecr, s.asyincr, s.asymin,
                                                     s.asymax, s.raa0, s.albefa, h->partial.as<double>());
    TF_LAUNCH_CHECK("mma_setup_kernel");
    double* hb = h->host;
    fetch(h, blocks, MMAX, 0, 0, hb, st);
    TF_CUDA_CHECK(cudaStreamSynchronize(st));
    std::vector<double> b(m), A(m), C(m), D(m);
    for (int i = 0; i < m; ++i) {
      b[i] = hb[i] - fval[i];
      A[i] = a[i];
      C[i] = c[i];
      D[i] = d[i];
    }
    // subproblem start point
    std::vector<double> y(m, 1.0), lam(m, 1.0), mu(m), sv(m, 1.0);
    for (int i = 0; i < m; ++i) mu[i] = std::max(1.0, 0.5 * C[i]);
    double z = 1.0, zet = 1.0, epsi = 1.0;
    Duals du{};
    du.m = m;
    auto residual = [&](double& norm, double& rmax) {
      du.epsi = epsi;
      for (int i = 0; i < m; ++i) du.lam[i] = lam[i];
      mma_residual_kernel<<<blocks, MMA_THREADS, 0, st>>>(v, du, h->partial.as<double>());
      TF_LAUNCH_CHECK("mma_residual_kernel");
      fetch(h, blocks, MMAX + 1, 0, 0, hb, st);
      fetch(h, blocks, 1, 1, (long long)blocks * (MMAX + 1), hb + MMAX + 1, st);
      TF_CUDA_CHECK(cudaStreamSynchronize(st));
      double ss = hb[MMAX], mx = hb[MMAX + 1];
      double alam = 0.0;
      for (int i = 0; i < m; ++i) alam += A[i] * lam[i];
      auto add = [&](double r) { ss += r * r; mx = std::max(mx, std::fabs(r)); };
      for (int i = 0; i < m; ++i) add(C[i] + D[i] * y[i] - mu[i] - lam[i]);
      add(a0 - zet - alam);
      for (int i = 0; i < m; ++i) add(hb[i] - A[i] * z - y[i] + sv[i] - b[i]);
      for (int i = 0; i < m; ++i) add(mu[i] * y[i] - epsi);
      add(zet * z - epsi);
      for (int i = 0; i < m; ++i) add(lam[i] * sv[i] - epsi);
      norm = std::sqrt(ss);
      rmax = mx;
    };
    int total = 0;
    std::vector<double> sums(NSUM);
    while (epsi > s.epsimin) {
      double norm, rmax;
      residual(norm, rmax);
      int inner = 0;
      while (rmax > 0.9 * epsi && inner < 200) {
        ++inner;
        ++total;
        du.epsi = epsi;
        for (int i = 0; i < m; ++i) du.lam[i] = lam[i];
        mma_newton_kernel<<<blocks, MMA_THREADS, 0, st>>>(v, du, h->partial.as<double>());
        TF_LAUNCH_CHECK("mma_newton_kernel");
        fetch(h, blocks, NSUM, 0, 0, hb, st);
        TF_CUDA_CHECK(cudaStreamSynchronize(st));
        std::copy(hb, hb + NSUM, sums.begin());
        double alam = 0.0;
        for (int i = 0; i < m; ++i) alam += A[i] * lam[i];
        std::vector<double> dely(m), diagy(m), dellam(m), blam(m);
        const double delz = a0 - alam - epsi / z;
        std::vector<double> AA((m + 1) * (m + 1), 0.0), rhs(m + 1);
        for (int i = 0; i < m; ++i) {
          dely[i] = C[i] + D[i] * y[i] - lam[i] - epsi / y[i];
          diagy[i] = D[i] + mu[i] / y[i];
          dellam[i] = sums[i] - A[i] * z - y[i] - b[i] + epsi / lam[i];
          blam[i] = dellam[i] + dely[i] / diagy[i] - sums[MMAX + i];
          rhs[i] = blam[i];
        }
        rhs[m] = delz;
        int q = 2 * MMAX;
        for (int i = 0; i < MMAX; ++i)
          for (int k = 0; k <= i; ++k, ++q)
            if (i < m) {
              AA[i * (m + 1) + k] = sums[q];
              AA[k * (m + 1) + i] = sums[q];
            }
        for (int i = 0; i < m; ++i) {
          AA[i * (m + 1) + i] += sv[i] / lam[i] + 1.0 / diagy[i];
          AA[i * (m + 1) + m] = A[i];
          AA[m * (m + 1) + i] = A[i];
        }
        AA[m * (m + 1) + m] = -zet / z;
        if (!solve_small(AA, rhs, m + 1)) throw Error(TF_NUMERIC, "MMA dual Newton system is singular");
        std::vector<double> dlam(rhs.begin(), rhs.begin() + m);
        const double dz = rhs[m];
        std::vector<double> dy(m), dmu(m), ds(m);
        for (int i = 0; i < m; ++i) {
          dy[i] = -dely[i] / diagy[i] + dlam[i] / diagy[i];
          dmu[i] = -mu[i] + epsi / y[i] - mu[i] * dy[i] / y[i];
          ds[i] = -sv[i] + epsi / lam[i] - sv[i] * dlam[i] / lam[i];
          du.dlam[i] = dlam[i];
        }
        const double dzet = -zet + epsi / z - zet * dz / z;
        mma_direction_kernel<<<blocks, MMA_THREADS, 0, st>>>(v, du, h->partial.as<double>());
        TF_LAUNCH_CHECK("mma_direction_kernel");
        fetch(h, blocks, 1, 1, 0, hb, st);
        TF_CUDA_CHECK(cudaStreamSynchronize(st));
        double stm = std::max(hb[0], 1.0);
        auto upd = [&](double dv, double val) { stm = std::max(stm, -1.01 * dv / val); };
        for (int i = 0; i < m; ++i) {
          upd(dy[i], y[i]);
          upd(dlam[i], lam[i]);
          upd(dmu[i], mu[i]);
          upd(ds[i], sv[i]);
        }
        upd(dz, z);
        upd(dzet, zet);
        double step = 1.0 / stm;
        const std::vector<double> y0 = y, lam0 = lam, mu0 = mu, s0 = sv;
        const double z0 = z, zet0 = zet;
        int tries = 0;
        double new_norm = 2.0 * norm, new_max = rmax;
        while (new_norm > norm && tries < 50) {
          ++tries;
          mma_trial_kernel<<<blocks, MMA_THREADS, 0, st>>>(v, step);
          TF_LAUNCH_CHECK("mma_trial_kernel");
          for (int i = 0; i < m; ++i) {
            y[i] = y0[i] + step * dy[i];
            lam[i] = lam0[i] + step * dlam[i];
            mu[i] = mu0[i] + step * dmu[i];
            sv[i] = s0[i] + step * ds[i];
          }
          z = z0 + step * dz;
          zet = zet0 + step * dzet;
          residual(new_norm, new_max);
          step *= 0.5;
        }
        norm = new_norm;
        rmax = new_max;
      }
      epsi *= 0.1;
    }
    TF_CUDA_CHECK(cudaMemcpyAsync(xnew, h->x.p, nb, cudaMemcpyDeviceToDevice, st));
    TF_CUDA_CHECK(cudaMemcpyAsync(low, h->low.p, nb, cudaMemcpyDeviceToDevice, st));
    TF_CUDA_CHECK(cudaMemcpyAsync(upp, h->upp.p, nb, cudaMemcpyDeviceToDevice, st));
    TF_CUDA_CHECK(cudaStreamSynchronize(st));
    for (int i = 0; i < m; ++i) {
      if (y_out) y_out[i] = y[i];
      if (lam_out) lam_out[i] = lam[i];
    }
    if (z_out) *z_out = z;
    if (newton_iterations) *newton_iterations = total;
  });
}
