// Hierarchy set-up kernels and the device-side PCG vector kernels.
#pragma once
#include "tf_kernels.cuh"
#include "tf_reduce.cuh"

namespace tfb {

struct PcgState {
  double* bnorm;
  double* rho;
  double* alpha;
  double* rel;
  double* scale;
  double* rzo;
  double* beta;
  double* wscale;          // scale the preconditioner output w was formed with: z = wscale * w
  double* rtrue;           // true relative residual at the last FP64 residual recomputation
  int* active;
  int* cand;
  int* iters;
  int* flags;              // [0] any candidate this step, [1] number of active columns
  unsigned long long* hist;  // bit patterns of non-negative doubles, one per step
  double* partial;         // [ncol][blocks][2] (two-value reductions) or [4] (three-value)
  unsigned* count;         // [ncol]
  int ncol;
};

// ---------------------------------------------------------------- set-up ----

// Live-dof mask of the finest level: a node is live when an adjacent element
// has E > 0 (topology_multigrid.py:138-144); fixed dofs are cleared.
__global__ void fine_mask_kernel(Geo g, const double* __restrict__ E, const uint8_t* __restrict__ fixedbits,
                                 uint8_t* __restrict__ mask) {
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < g.nnode; n += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    node_coords(n, g, i, j, k);
    bool live = false;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int ei = i - 1 + (e >> 2), ej = j - 1 + ((e >> 1) & 1), ek = k - 1 + (e & 1);
      if ((unsigned)ei < (unsigned)g.ex && (unsigned)ej < (unsigned)g.ey && (unsigned)ek < (unsigned)g.ez)
        live |= E[((long long)ei * g.ey + ej) * g.ez + ek] > 0.0;
    }
    mask[n] = live ? static_cast<uint8_t>(7u & ~static_cast<unsigned>(fixedbits[n])) : uint8_t(0);
  }
}

// Diagonal of the finest operator, sum_e E_e K0_ii (topology_multigrid.py:118-124), times the mask.
__global__ void fine_diag_kernel(Geo g, const double* __restrict__ E, const uint8_t* __restrict__ mask,
                                 const double* __restrict__ k0diag, double* __restrict__ diag) {
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < g.nnode; n += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    node_coords(n, g, i, j, k);
    double d[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int ox = e >> 2, oy = (e >> 1) & 1, oz = e & 1;
      const int ei = i - 1 + ox, ej = j - 1 + oy, ek = k - 1 + oz;
      if ((unsigned)ei < (unsigned)g.ex && (unsigned)ej < (unsigned)g.ey && (unsigned)ek < (unsigned)g.ez) {
        const double w = E[((long long)ei * g.ey + ej) * g.ez + ek];
        const int cn = corner_id(1 - ox, 1 - oy, 1 - oz);
#pragma unroll
        for (int a = 0; a < 3; ++a) d[a] += w * k0diag[3 * cn + a];
      }
    }
    const unsigned m = mask[n];
#pragma unroll
    for (int a = 0; a < 3; ++a) diag[3 * n + a] = ((m >> a) & 1u) ? d[a] : 0.0;
  }
}

// Diagonal of a Galerkin level: sum_e B_e[ii].
__global__ void block_diag_kernel(Geo g, const double* __restrict__ B, double* __restrict__ diag) {
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < g.nnode; n += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    node_coords(n, g, i, j, k);
    double d[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int ox = e >> 2, oy = (e >> 1) & 1, oz = e & 1;
      const int ei = i - 1 + ox, ej = j - 1 + oy, ek = k - 1 + oz;
      if ((unsigned)ei < (unsigned)g.ex && (unsigned)ej < (unsigned)g.ey && (unsigned)ek < (unsigned)g.ez) {
        const double* b = B + (((long long)ei * g.ey + ej) * g.ez + ek) * 576;
        const int cn = corner_id(1 - ox, 1 - oy, 1 - oz);
#pragma unroll
        for (int a = 0; a < 3; ++a) d[a] += b[(3 * cn + a) * 25];
      }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) diag[3 * n + a] = d[a];
  }
}

// max over an array (single column reduction into out[0])
__global__ void amax_kernel(const double* __restrict__ v, long long n, double* partial, unsigned* count, double* out) {
  double a = 0.0, b = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    a = fmax(a, fabs(v[t]));
  block_reduce2<1, 0>(a, b);
  if (last_block_combine<1, 0>(a, b, partial, count, 0)) out[0] = a;
}

// Dead-dof mask and inverse diagonal of a Galerkin level (topology_multigrid.py:180-186).
template <typename T>
__global__ void coarse_mask_inv_kernel(long long nnode, const double* __restrict__ diag, const double* __restrict__ dmax,
                                       double ratio, uint8_t* __restrict__ mask, double* __restrict__ inv64, T* __restrict__ invw) {
  const double thr = ratio * dmax[0];
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < nnode; n += (long long)gridDim.x * blockDim.x) {
    unsigned m = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double d = diag[3 * n + a];
      const bool live = d > thr;
      m |= live ? (1u << a) : 0u;
      const double iv = live ? 1.0 / (d > 0.0 ? d : 1.0) : 0.0;
      inv64[3 * n + a] = iv;
      if (invw) invw[3 * n + a] = static_cast<T>(iv);
    }
    mask[n] = static_cast<uint8_t>(m);
  }
}

template <typename T>
__global__ void fine_inv_kernel(long long nnode, const double* __restrict__ diag, const uint8_t* __restrict__ mask,
                                double* __restrict__ inv64, T* __restrict__ invw) {
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < nnode; n += (long long)gridDim.x * blockDim.x) {
    const unsigned m = mask[n];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double d = diag[3 * n + a];
      const double iv = ((m >> a) & 1u) ? 1.0 / (d > 0.0 ? d : 1.0) : 0.0;
      inv64[3 * n + a] = iv;
      if (invw) invw[3 * n + a] = static_cast<T>(iv);
    }
  }
}

// Galerkin coarse blocks  B_C = sym( sum_c P_c^T K_c P_c )  (topology_multigrid.py:125-137,175-179).
// P_c = W_c (x) I3 with W_c[r][s] the trilinear weight of coarse corner s at
// child corner r.  From the finest level K_c = E_c g g^T o K0 (g = live mask of
// the child's 24 dofs); children without a dead dof take the precomputed
// Q_c = P_c^T K0 P_c.  Deeper levels use the previous level's blocks.
struct GalerkinParam { double W[8][8][8]; };

__global__ void __launch_bounds__(128) galerkin_kernel(const __grid_constant__ GalerkinParam P, Geo cg, Geo fg, int from_fine,
                                                       const double* __restrict__ E, const uint8_t* __restrict__ fmask,
                                                       const double* __restrict__ K0, const double* __restrict__ Q,
                                                       const double* __restrict__ child_blocks, double* __restrict__ out) {
  __shared__ double Kc[576];
  __shared__ double Tm[576];
  __shared__ double acc[576];
  __shared__ int gbits[24];
  __shared__ int fast;
  const long long ncoarse = (long long)cg.ex * cg.ey * cg.ez;
  for (long long ce = blockIdx.x; ce < ncoarse; ce += gridDim.x) {
    const int K = static_cast<int>(ce % cg.ez);
    const long long r1 = ce / cg.ez;
    const int J = static_cast<int>(r1 % cg.ey);
    const int I = static_cast<int>(r1 / cg.ey);
    for (int t = threadIdx.x; t < 576; t += blockDim.x) acc[t] = 0.0;
    __syncthreads();
    for (int c = 0; c < 8; ++c) {
      const int fi = 2 * I + (c >> 2), fj = 2 * J + ((c >> 1) & 1), fk = 2 * K + (c & 1);
      const long long fe = ((long long)fi * fg.ey + fj) * fg.ez + fk;
      double Ec = 0.0;
      if (from_fine) {
        Ec = E[fe];
        if (threadIdx.x < 24) {
          const int corner = threadIdx.x / 3, comp = threadIdx.x % 3;
          const int cx = (corner == 1 || corner == 2 || corner == 5 || corner == 6) ? 1 : 0;
          const int cy = (corner == 2 || corner == 3 || corner == 6 || corner == 7) ? 1 : 0;
          const int cz = corner >> 2;
          const long long node = ((long long)(fi + cx) * fg.ny + (fj + cy)) * fg.nz + (fk + cz);
          gbits[threadIdx.x] = (fmask[node] >> comp) & 1;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
          int all = 1;
          for (int q = 0; q < 24; ++q) all &= gbits[q];
          fast = all;
        }
        __syncthreads();
        if (Ec == 0.0) { __syncthreads(); continue; }
        if (fast) {
          const double* q = Q + c * 576;
          for (int t = threadIdx.x; t < 576; t += blockDim.x) acc[t] += Ec * q[t];
          __syncthreads();
          continue;
        }
        for (int t = threadIdx.x; t < 576; t += blockDim.x) {
          const int a = t / 24, b = t % 24;
          Kc[t] = (gbits[a] && gbits[b]) ? Ec * K0[t] : 0.0;
        }
      } else {
        const double* src = child_blocks + fe * 576;
        for (int t = threadIdx.x; t < 576; t += blockDim.x) Kc[t] = src[t];
      }
      __syncthreads();
      // Tm = Kc P_c :  Tm[i][3s+y] = sum_r Kc[i][3r+y] W[c][r][s]
      for (int t = threadIdx.x; t < 576; t += blockDim.x) {
        const int i = t / 24, col = t % 24, s = col / 3, y = col % 3;
        double v = 0.0;
#pragma unroll
        for (int r = 0; r < 8; ++r) v += Kc[i * 24 + 3 * r + y] * P.W[c][r][s];
        Tm[t] = v;
      }
      __syncthreads();
      // acc += P_c^T Tm :  acc[3s+x][j] += sum_r W[c][r][s] Tm[3r+x][j]
      for (int t = threadIdx.x; t < 576; t += blockDim.x) {
        const int row = t / 24, j = t % 24, s = row / 3, x = row % 3;
        double v = 0.0;
#pragma unroll
        for (int r = 0; r < 8; ++r) v += P.W[c][r][s] * Tm[(3 * r + x) * 24 + j];
        acc[t] += v;
      }
      __syncthreads();
    }
    double* o = out + ce * 576;
    for (int t = threadIdx.x; t < 576; t += blockDim.x) {
      const int a = t / 24, b = t % 24;
      o[t] = 0.5 * (acc[t] + acc[b * 24 + a]);
    }
    __syncthreads();
  }
}

// Assembled 27-point stencil of a Galerkin level from its [nelem][576] FP64 element blocks (block row
// 3 corner + q, column 3 corner + r): one thread per (neighbour offset d, node) sums the 3 x 3 blocks
// coupling the node (corner cn of element e) with node + d (corner cm of e) over the elements holding
// both, in a fixed element order.  Output entry-major [243][nnode] in FP64, and in FP32 when s32 is set.
__global__ void stencil_assemble_kernel(Geo g, const double* __restrict__ blocks, double* __restrict__ s64,
                                        float* __restrict__ s32) {
  const long long nnode = g.nnode;
  const long long total = 27 * nnode;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int d = static_cast<int>(t / nnode);
    const long long n = t % nnode;
    const int k = static_cast<int>(n % g.nz);
    const long long r1 = n / g.nz;
    const int j = static_cast<int>(r1 % g.ny), i = static_cast<int>(r1 / g.ny);
    const int di = d / 9 - 1, dj = (d / 3) % 3 - 1, dk = d % 3 - 1;
    double acc[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) acc[q] = 0.0;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int ox = e >> 2, oy = (e >> 1) & 1, oz = e & 1;
      const int cx = 1 - ox + di, cy = 1 - oy + dj, cz = 1 - oz + dk;
      if (cx < 0 || cx > 1 || cy < 0 || cy > 1 || cz < 0 || cz > 1) continue;
      const int ei = i - 1 + ox, ej = j - 1 + oy, ek = k - 1 + oz;
      if (!((unsigned)ei < (unsigned)g.ex && (unsigned)ej < (unsigned)g.ey && (unsigned)ek < (unsigned)g.ez)) continue;
      const int cn = corner_id(1 - ox, 1 - oy, 1 - oz);
      const int cm = corner_id(cx, cy, cz);
      const double* bp = blocks + (((long long)ei * g.ey + ej) * g.ez + ek) * 576 + (3 * cn) * 24 + 3 * cm;
#pragma unroll
      for (int q = 0; q < 3; ++q)
#pragma unroll
        for (int rr = 0; rr < 3; ++rr) acc[3 * q + rr] += bp[q * 24 + rr];
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      const long long o = (long long)(d * 9 + q) * nnode + n;
      s64[o] = acc[q];
      if (s32) s32[o] = static_cast<float>(acc[q]);
    }
  }
}

// [nelem][576] FP64 blocks -> entry-major [576][nelem] copy in T (tiled through shared memory).
template <typename T>
__global__ void blocks_soa_kernel(const double* __restrict__ aos, T* __restrict__ soa, long long nelem) {
  __shared__ double tile[32][65];
  const long long e0 = (long long)blockIdx.x * 32;
  const int r0 = blockIdx.y * 64;
  for (int t = threadIdx.x; t < 32 * 64; t += blockDim.x) {
    const int el = t / 64, r = t % 64;
    const long long e = e0 + el;
    tile[el][r] = (e < nelem && r0 + r < 576) ? aos[e * 576 + r0 + r] : 0.0;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < 32 * 64; t += blockDim.x) {
    const int r = t / 32, el = t % 32;
    const long long e = e0 + el;
    if (e < nelem && r0 + r < 576) soa[(long long)(r0 + r) * nelem + e] = static_cast<T>(tile[el][r]);
  }
}

template <typename T>
__global__ void cast_kernel(const double* __restrict__ src, T* __restrict__ dst, long long n) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    dst[t] = static_cast<T>(src[t]);
}

// Deterministic uniform(-0.5, 0.5) start vector of the power iteration, masked.
__device__ __forceinline__ double hash_uniform(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  x ^= x >> 31;
  return (double)(x >> 11) * (1.0 / 9007199254740992.0);
}

template <typename T>
__global__ void power_init_kernel(long long nnode, const uint8_t* __restrict__ mask, T* __restrict__ v) {
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < nnode; n += (long long)gridDim.x * blockDim.x) {
    const unsigned m = mask[n];
#pragma unroll
    for (int a = 0; a < 3; ++a)
      v[3 * n + a] = ((m >> a) & 1u) ? static_cast<T>(hash_uniform(3 * n + a) - 0.5) : T(0);
  }
}

// y <- inv o y, out = ||y||
template <typename T>
__global__ void power_scale_kernel(long long ndof, const T* __restrict__ inv, T* __restrict__ y, double* partial,
                                   unsigned* count, double* out) {
  double a = 0.0, b = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < ndof; t += (long long)gridDim.x * blockDim.x) {
    const T v = inv[t] * y[t];
    y[t] = v;
    a += (double)v * (double)v;
  }
  block_reduce2<0, 0>(a, b);
  if (last_block_combine<0, 0>(a, b, partial, count, 0)) out[0] = sqrt(a);
}

template <typename T>
__global__ void power_norm_kernel(long long ndof, const T* __restrict__ y, const double* __restrict__ est, T* __restrict__ v) {
  const double s = 1.0 / est[0];
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < ndof; t += (long long)gridDim.x * blockDim.x)
    v[t] = static_cast<T>((double)y[t] * s);
}

// Dense coarsest matrix of the live dofs, assembled node by node (deterministic).
__global__ void coarsest_assemble_kernel(Geo g, const double* __restrict__ B, const int* __restrict__ live_of_dof,
                                         const long long* __restrict__ live_dofs, int n, double* __restrict__ A) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const long long dof = live_dofs[t];
    const long long node = dof / 3;
    const int a = static_cast<int>(dof % 3);
    int i, j, k;
    node_coords(node, g, i, j, k);
    double* row = A + t * (long long)n;
    for (int di = -1; di <= 1; ++di)
      for (int dj = -1; dj <= 1; ++dj)
        for (int dk = -1; dk <= 1; ++dk) {
          const int ni = i + di, nj = j + dj, nk = k + dk;
          if (!((unsigned)ni < (unsigned)g.nx && (unsigned)nj < (unsigned)g.ny && (unsigned)nk < (unsigned)g.nz)) continue;
          const long long m = ((long long)ni * g.ny + nj) * g.nz + nk;
          double v[3] = {0.0, 0.0, 0.0};
          for (int e = 0; e < 8; ++e) {
            const int ox = e >> 2, oy = (e >> 1) & 1, oz = e & 1;
            const int cx = 1 - ox + di, cy = 1 - oy + dj, cz = 1 - oz + dk;
            if (cx < 0 || cx > 1 || cy < 0 || cy > 1 || cz < 0 || cz > 1) continue;
            const int ei = i - 1 + ox, ej = j - 1 + oy, ek = k - 1 + oz;
            if (!((unsigned)ei < (unsigned)g.ex && (unsigned)ej < (unsigned)g.ey && (unsigned)ek < (unsigned)g.ez)) continue;
            const double* b = B + (((long long)ei * g.ey + ej) * g.ez + ek) * 576;
            const int cn = corner_id(1 - ox, 1 - oy, 1 - oz), cm = corner_id(cx, cy, cz);
            for (int q = 0; q < 3; ++q) v[q] += b[(3 * cn + a) * 24 + 3 * cm + q];
          }
          for (int q = 0; q < 3; ++q) {
            const int col = live_of_dof[3 * m + q];
            if (col >= 0) row[col] = v[q];
          }
        }
  }
}

// The same coarsest Galerkin matrix in band storage (the lower band of (A + A^T) / 2:
// AB[c * (bw + 1) + (r - c)] = A[r][c] for 0 <= r - c <= bw, live-dof numbering), for coarsest grids
// too large for a dense factor.  Thread r forms row r's entries left of the diagonal and their
// transposed counterparts, so every band entry is written once (no atomics, deterministic).
__global__ void coarsest_assemble_band_kernel(Geo g, const double* __restrict__ B, const int* __restrict__ live_of_dof,
                                              const long long* __restrict__ live_dofs, int n, int bw, double* __restrict__ AB) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const long long dof = live_dofs[t];
    const long long node = dof / 3;
    const int a = static_cast<int>(dof % 3);
    int i, j, k;
    node_coords(node, g, i, j, k);
    for (int di = -1; di <= 1; ++di)
      for (int dj = -1; dj <= 1; ++dj)
        for (int dk = -1; dk <= 1; ++dk) {
          const int ni = i + di, nj = j + dj, nk = k + dk;
          if (!((unsigned)ni < (unsigned)g.nx && (unsigned)nj < (unsigned)g.ny && (unsigned)nk < (unsigned)g.nz)) continue;
          const long long m = ((long long)ni * g.ny + nj) * g.nz + nk;
          double v[3] = {0.0, 0.0, 0.0}, vt[3] = {0.0, 0.0, 0.0};
          for (int e = 0; e < 8; ++e) {
            const int ox = e >> 2, oy = (e >> 1) & 1, oz = e & 1;
            const int cx = 1 - ox + di, cy = 1 - oy + dj, cz = 1 - oz + dk;
            if (cx < 0 || cx > 1 || cy < 0 || cy > 1 || cz < 0 || cz > 1) continue;
            const int ei = i - 1 + ox, ej = j - 1 + oy, ek = k - 1 + oz;
            if (!((unsigned)ei < (unsigned)g.ex && (unsigned)ej < (unsigned)g.ey && (unsigned)ek < (unsigned)g.ez)) continue;
            const double* b = B + (((long long)ei * g.ey + ej) * g.ez + ek) * 576;
            const int cn = corner_id(1 - ox, 1 - oy, 1 - oz), cm = corner_id(cx, cy, cz);
            for (int q = 0; q < 3; ++q) {
              v[q] += b[(3 * cn + a) * 24 + 3 * cm + q];
              vt[q] += b[(3 * cm + q) * 24 + 3 * cn + a];
            }
          }
          for (int q = 0; q < 3; ++q) {
            const int col = live_of_dof[3 * m + q];
            if (col < 0 || col > t || t - col > bw) continue;
            AB[(long long)col * (bw + 1) + (t - col)] = col == t ? v[q] : 0.5 * (v[q] + vt[q]);
          }
        }
  }
}

// gather live coarsest dofs of the active columns into FP64 [ncol][n]
template <typename T>
__device__ __forceinline__ void coarsest_gather_body(const VGrid vg_,const T* __restrict__ src, long long stride, const long long* __restrict__ live, int n,
                                       double* __restrict__ dst, const int* __restrict__ active) {
  TF_VGRID(vg_);
  const int col = blockIdx.y;
  if (active && !active[col]) return;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    dst[(long long)col * n + t] = static_cast<double>(src[col * stride + live[t]]);
}
template <typename T>
__global__ void coarsest_gather_kernel(const T* __restrict__ src, long long stride, const long long* __restrict__ live, int n,
                                       double* __restrict__ dst, const int* __restrict__ active) {
  coarsest_gather_body<T>(vgrid(), src, stride, live, n, dst, active);
}

template <typename T>
__device__ __forceinline__ void coarsest_scatter_body(const VGrid vg_,const double* __restrict__ src, const long long* __restrict__ live, int n,
                                        T* __restrict__ dst, long long stride, const int* __restrict__ active, int round) {
  TF_VGRID(vg_);
  const int col = blockIdx.y;
  if (active && !active[col]) return;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    dst[col * stride + live[t]] = round_store(static_cast<T>(src[(long long)col * n + t]), round);
}
template <typename T>
__global__ void coarsest_scatter_kernel(const double* __restrict__ src, const long long* __restrict__ live, int n,
                                        T* __restrict__ dst, long long stride, const int* __restrict__ active, int round) {
  coarsest_scatter_body<T>(vgrid(), src, live, n, dst, stride, active, round);
}

// ----------------------------------------------------------- elementwise ----

template <typename T>
__device__ __forceinline__ void zero_cols_body(const VGrid vg_,T* __restrict__ v, long long stride, const int* __restrict__ active) {
  TF_VGRID(vg_);
  const int col = blockIdx.y;
  if (active && !active[col]) return;
  T* p = v + col * stride;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < stride; t += (long long)gridDim.x * blockDim.x) p[t] = T(0);
}
template <typename T>
__global__ void zero_cols_kernel(T* __restrict__ v, long long stride, const int* __restrict__ active) {
  zero_cols_body<T>(vgrid(), v, stride, active);
}

// x = s * inv * b   (first Jacobi sweep from a zero guess)
template <typename T>
__device__ __forceinline__ void jacobi_first_body(const VGrid vg_,long long ndof, const T* __restrict__ inv, const T* __restrict__ b, T* __restrict__ x, T s,
                                    const int* __restrict__ active, int round) {
  TF_VGRID(vg_);
  const int col = blockIdx.y;
  if (active && !active[col]) return;
  const long long off = (long long)col * ndof;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < ndof; t += (long long)gridDim.x * blockDim.x)
    x[off + t] = round_store(s * inv[t] * b[off + t], round);
}
template <typename T>
__global__ void jacobi_first_kernel(long long ndof, const T* __restrict__ inv, const T* __restrict__ b, T* __restrict__ x, T s,
                                    const int* __restrict__ active, int round) {
  jacobi_first_body<T>(vgrid(), ndof, inv, b, x, s, active, round);
}

// Chebyshev start from a zero guess: res = b, d = inv * res / theta, x = d (with has_x: x += d, res
// kept).  Without write_rd only x is written: a one-sweep smoother reads neither res nor d again.
template <typename T>
__device__ __forceinline__ void cheb_first_body(const VGrid vg_,long long ndof, const T* __restrict__ inv, const T* __restrict__ b, T* __restrict__ res,
                                  T* __restrict__ d, T* __restrict__ x, T inv_theta, int has_x, int write_rd,
                                  const int* __restrict__ active, int round) {
  TF_VGRID(vg_);
  const int col = blockIdx.y;
  if (active && !active[col]) return;
  const long long off = (long long)col * ndof;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < ndof; t += (long long)gridDim.x * blockDim.x) {
    const T r = has_x ? res[off + t] : b[off + t];
    const T dv = round_store(inv[t] * r * inv_theta, round);
    if (write_rd) {
      res[off + t] = r;
      d[off + t] = dv;
    }
    x[off + t] = has_x ? round_store(x[off + t] + dv, round) : dv;
  }
}
template <typename T>
__global__ void cheb_first_kernel(long long ndof, const T* __restrict__ inv, const T* __restrict__ b, T* __restrict__ res,
                                  T* __restrict__ d, T* __restrict__ x, T inv_theta, int has_x, int write_rd,
                                  const int* __restrict__ active, int round) {
  cheb_first_body<T>(vgrid(), ndof, inv, b, res, d, x, inv_theta, has_x, write_rd, active, round);
}

// --------------------------------------------------------------- PCG -------

constexpr int PCG_BLOCKS = 64;   // reduction blocks per column

// bnorm = ||b||; r = b; x = 0 (or r = b - A x computed elsewhere)
__device__ __forceinline__ void pcg_norm_body(const VGrid vg_,const double* __restrict__ b, long long n, PcgState st, double* out, int take_sqrt) {
  TF_VGRID(vg_);
  const int col = blockIdx.y;
  if (!st.active[col]) return;
  const double* p = b + (long long)col * n;
  double a = 0.0, z = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) a += p[t] * p[t];
  block_reduce2<0, 0>(a, z);
  if (last_block_combine<0, 0>(a, z, st.partial, st.count, col, blockIdx.x, gridDim.x)) out[col] = take_sqrt ? sqrt(a) : a;
}
__global__ void pcg_norm_kernel(const double* __restrict__ b, long long n, PcgState st, double* out, int take_sqrt) {
  pcg_norm_body(vgrid(), b, n, st, out, take_sqrt);
}

// alpha = rho / (p . q).  R is the type of the PCG vectors: double for the FP64 PCG, float for the
// FP32 iterations of the mixed PCG (dot products accumulate in double either way).
template <typename R>
__global__ void pcg_alpha_kernel(const R* __restrict__ p, const R* __restrict__ q, long long n, PcgState st) {
  const int col = blockIdx.y;
  if (!st.active[col]) return;
  const long long off = (long long)col * n;
  double a = 0.0, z = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    a += static_cast<double>(p[off + t]) * static_cast<double>(q[off + t]);
  block_reduce2<0, 0>(a, z);
  if (last_block_combine<0, 0>(a, z, st.partial, st.count, col, blockIdx.x, gridDim.x)) st.alpha[col] = st.rho[col] / a;
}

// alpha = rho / (p . K p) from the per-warp partials that the FP64 finest-level operator wrote while
// it formed q = K p (LevelArgs::dot_out): one block per column sums its partials in a fixed order,
// so the result does not depend on scheduling.
__device__ __forceinline__ void pcg_alpha_sum_body(const VGrid vg_,const double* __restrict__ part, long long per_col, PcgState st) {
  TF_VGRID(vg_);
  const int col = blockIdx.x;
  if (!st.active[col]) return;
  const double* pc = part + (long long)col * per_col;
  double a = 0.0, z = 0.0;
  for (long long t = threadIdx.x; t < per_col; t += blockDim.x) a += pc[t];
  block_reduce2<0, 0>(a, z);
  if (threadIdx.x == 0) st.alpha[col] = st.rho[col] / a;
}
__global__ void pcg_alpha_sum_kernel(const double* __restrict__ part, long long per_col, PcgState st) {
  pcg_alpha_sum_body(vgrid(), part, per_col, st);
}

// x += alpha p; r -= alpha q; rel = ||r|| / ||b||; candidate when rel < tol (topology_multigrid.py:424-430).
// The same pass forms the next preconditioner inputs, scale = max|r| (clamped at 1e-300) and
// rzo = r . z_old (topology_multigrid.py:320, :446), with z_old = wscale * w rebuilt from the
// work-precision preconditioner output: z itself is never stored.  x is always FP64.  With
// reliable > 0 (the mixed PCG) a column whose iterated residual fell below reliable times its
// last true residual also asks for the FP64 residual recomputation (a reliable update).
template <typename T, typename R>
__device__ __forceinline__ void pcg_update_body(const VGrid vg_,double* __restrict__ x, R* __restrict__ r, const R* __restrict__ p,
                                  const R* __restrict__ q, const T* __restrict__ w, long long n, PcgState st, double tol,
                                  int step, double reliable) {
  TF_VGRID(vg_);
  const int col = blockIdx.y;
  if (!st.active[col]) return;
  const long long off = (long long)col * n;
  const double al = st.alpha[col];
  const double zs = st.wscale[col];
  double a = 0.0, mx = 0.0, d = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    x[off + t] += al * static_cast<double>(p[off + t]);
    const R rv = static_cast<R>(static_cast<double>(r[off + t]) - al * static_cast<double>(q[off + t]));
    r[off + t] = rv;
    const double rd = static_cast<double>(rv);
    a += rd * rd;
    mx = fmax(mx, fabs(rd));
    d += rd * (static_cast<double>(w[off + t]) * zs);
  }
  block_reduce3<0, 1, 0>(a, mx, d);
  if (last_block_combine3<0, 1, 0>(a, mx, d, st.partial, st.count, col, blockIdx.x, gridDim.x)) {
    const double rel = sqrt(a) / st.bnorm[col];
    st.rel[col] = rel;
    st.scale[col] = fmax(mx, 1e-300);
    st.rzo[col] = d;
    if (!isfinite(rel)) {
      st.cand[col] = 4;   // breakdown (a non-finite residual): the column stops and is reported unconverged
      return;
    }
    atomicMax(&st.hist[step - 1], static_cast<unsigned long long>(__double_as_longlong(rel)));
    if (rel < tol || (reliable > 0.0 && rel < reliable * st.rtrue[col])) { st.cand[col] = 1; atomicExch(&st.flags[0], 1); }
  }
}
template <typename T, typename R>
__global__ void pcg_update_kernel(double* __restrict__ x, R* __restrict__ r, const R* __restrict__ p,
                                  const R* __restrict__ q, const T* __restrict__ w, long long n, PcgState st, double tol,
                                  int step, double reliable) {
  pcg_update_body<T, R>(vgrid(), x, r, p, q, w, n, st, tol, step, reliable);
}

// True-residual recheck (topology_multigrid.py:431-437): when any column is a
// candidate, every active column's residual is recomputed as t = b - K x; a
// column converges when ||t|| / ||b|| < tol, the others continue from t.
__device__ __forceinline__ void pcg_truecheck_body(const VGrid vg_,const double* __restrict__ t_res, long long n, PcgState st, double tol, int step) {
  TF_VGRID(vg_);
  const int col = blockIdx.y;
  if (!st.flags[0] || !st.active[col] || st.cand[col] == 4) return;
  const long long off = (long long)col * n;
  double a = 0.0, z = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const double v = t_res[off + t];
    a += v * v;
  }
  block_reduce2<0, 0>(a, z);
  if (last_block_combine<0, 0>(a, z, st.partial, st.count, col, blockIdx.x, gridDim.x)) {
    const double rel = sqrt(a) / st.bnorm[col];
    st.rel[col] = rel;
    st.rtrue[col] = rel;
    st.cand[col] = (rel < tol) ? 2 : 3;   // 2 = converged, 3 = continue from the true residual
  }
}
__global__ void pcg_truecheck_kernel(const double* __restrict__ t_res, long long n, PcgState st, double tol, int step) {
  pcg_truecheck_body(vgrid(), t_res, n, st, tol, step);
}

// Columns that continue from the true residual (cand 3): r <- t, and the preconditioner inputs
// scale = max|t| and rzo = t . z_old are formed again from the new r.
template <typename T, typename R>
__device__ __forceinline__ void pcg_retire_body(const VGrid vg_,const double* __restrict__ t_res, R* __restrict__ r, const T* __restrict__ w, long long n,
                                  PcgState st) {
  TF_VGRID(vg_);
  const int col = blockIdx.y;
  if (!st.active[col] || st.cand[col] != 3) return;
  const long long off = (long long)col * n;
  const double zs = st.wscale[col];
  double mx = 0.0, d = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const double v = t_res[off + t];
    r[off + t] = static_cast<R>(v);
    mx = fmax(mx, fabs(v));
    d += v * (static_cast<double>(w[off + t]) * zs);
  }
  block_reduce2<1, 0>(mx, d);
  if (last_block_combine<1, 0>(mx, d, st.partial, st.count, col, blockIdx.x, gridDim.x)) {
    st.scale[col] = fmax(mx, 1e-300);
    st.rzo[col] = d;
  }
}
template <typename T, typename R>
__global__ void pcg_retire_kernel(const double* __restrict__ t_res, R* __restrict__ r, const T* __restrict__ w, long long n,
                                  PcgState st) {
  pcg_retire_body<T, R>(vgrid(), t_res, r, w, n, st);
}

__device__ __forceinline__ void pcg_flags_body(const VGrid vg_,PcgState st, int step) {
  TF_VGRID(vg_);
  // single block: finalize column states for this step
  int n_active = 0;
  for (int col = threadIdx.x; col < st.ncol; col += blockDim.x) {
    if (st.active[col]) {
      if (st.cand[col] == 2 || st.cand[col] == 4) {   // converged, or broken down (its rel stays non-finite)
        st.active[col] = 0;
        st.iters[col] = step;
      }
    }
    st.cand[col] = 0;
    n_active += st.active[col];
  }
  __shared__ int tot;
  if (threadIdx.x == 0) tot = 0;
  __syncthreads();
  atomicAdd(&tot, n_active);
  __syncthreads();
  if (threadIdx.x == 0) {
    st.flags[1] = tot;
    st.flags[0] = 0;
  }
}
__global__ void pcg_flags_kernel(PcgState st, int step) {
  pcg_flags_body(vgrid(), st, step);
}

// The starting residual: r = t (t = b, or b - K x0 for a warm start), scale = max|t| (clamped at
// 1e-300; topology_multigrid.py:320) and rtrue = ||t|| / ||b||, the reference of the first
// reliable update.
template <typename R>
__device__ __forceinline__ void pcg_take_body(const VGrid vg_,const double* __restrict__ t_res, R* __restrict__ r, long long n, PcgState st) {
  TF_VGRID(vg_);
  const int col = blockIdx.y;
  if (!st.active[col]) return;
  const long long off = (long long)col * n;
  double mx = 0.0, a = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const double v = t_res[off + t];
    r[off + t] = static_cast<R>(v);
    mx = fmax(mx, fabs(v));
    a += v * v;
  }
  block_reduce2<1, 0>(mx, a);
  if (last_block_combine<1, 0>(mx, a, st.partial, st.count, col, blockIdx.x, gridDim.x)) {
    st.scale[col] = fmax(mx, 1e-300);
    st.rtrue[col] = sqrt(a) / st.bnorm[col];
  }
}
template <typename R>
__global__ void pcg_take_kernel(const double* __restrict__ t_res, R* __restrict__ r, long long n, PcgState st) {
  pcg_take_body<R>(vgrid(), t_res, r, n, st);
}

// scale = max|r| (clamped at 1e-300) before the first preconditioner application (topology_multigrid.py:320)
template <typename R>
__global__ void pcg_prep_kernel(const R* __restrict__ r, long long n, PcgState st) {
  const int col = blockIdx.y;
  if (!st.active[col]) return;
  const long long off = (long long)col * n;
  double mx = 0.0, d = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    mx = fmax(mx, fabs(static_cast<double>(r[off + t])));
  block_reduce2<1, 0>(mx, d);
  if (last_block_combine<1, 0>(mx, d, st.partial, st.count, col, blockIdx.x, gridDim.x)) st.scale[col] = fmax(mx, 1e-300);
}

template <typename T, typename R>
__device__ __forceinline__ void pcg_to_work_body(const VGrid vg_,const R* __restrict__ r, long long n, PcgState st, T* __restrict__ w, int round) {
  TF_VGRID(vg_);
  const int col = blockIdx.y;
  if (!st.active[col]) return;
  const long long off = (long long)col * n;
  const double s = 1.0 / st.scale[col];
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    w[off + t] = round_store(static_cast<T>(static_cast<double>(r[off + t]) * s), round);
}
template <typename T, typename R>
__global__ void pcg_to_work_kernel(const R* __restrict__ r, long long n, PcgState st, T* __restrict__ w, int round) {
  pcg_to_work_body<T, R>(vgrid(), r, n, st, w, round);
}

// rz = r . z with z = scale * w (w: the work-precision preconditioner output); beta = (rz - rzo) / rho
// (flexible Polak-Ribiere, topology_multigrid.py:445-448).  z is written out only when asked for (z != nullptr).
template <typename T, typename R>
__device__ __forceinline__ void pcg_from_work_body(const VGrid vg_,const T* __restrict__ w, const R* __restrict__ r, double* __restrict__ z, long long n,
                                     PcgState st, int initial) {
  TF_VGRID(vg_);
  const int col = blockIdx.y;
  if (!st.active[col]) return;
  const long long off = (long long)col * n;
  const double s = st.scale[col];
  double d = 0.0, zz = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const double v = static_cast<double>(w[off + t]) * s;
    if (z) z[off + t] = v;
    d += static_cast<double>(r[off + t]) * v;
  }
  block_reduce2<0, 0>(d, zz);
  if (last_block_combine<0, 0>(d, zz, st.partial, st.count, col, blockIdx.x, gridDim.x)) {
    st.beta[col] = initial ? 0.0 : (d - st.rzo[col]) / st.rho[col];
    st.rho[col] = d;
    st.wscale[col] = s;
  }
}
template <typename T, typename R>
__global__ void pcg_from_work_kernel(const T* __restrict__ w, const R* __restrict__ r, double* __restrict__ z, long long n,
                                     PcgState st, int initial) {
  pcg_from_work_body<T, R>(vgrid(), w, r, z, n, st, initial);
}

// p = z + beta p, z = wscale * w
template <typename T, typename R>
__device__ __forceinline__ void pcg_direction_body(const VGrid vg_,const T* __restrict__ w, R* __restrict__ p, long long n, PcgState st, int initial) {
  TF_VGRID(vg_);
  const int col = blockIdx.y;
  if (!st.active[col]) return;
  const long long off = (long long)col * n;
  const double be = st.beta[col], s = st.wscale[col];
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const double z = static_cast<double>(w[off + t]) * s;
    p[off + t] = static_cast<R>(initial ? z : z + be * static_cast<double>(p[off + t]));
  }
}
template <typename T, typename R>
__global__ void pcg_direction_kernel(const T* __restrict__ w, R* __restrict__ p, long long n, PcgState st, int initial) {
  pcg_direction_body<T, R>(vgrid(), w, p, n, st, initial);
}

// ------------------------------------------------------- layout copies ----

// padded[c][node_p] <- mask * flat[c][node] for nodes inside the unpadded grid (0 elsewhere)
__global__ void pad_kernel(const double* __restrict__ flat, long long fstride, Geo un, Geo pd, const uint8_t* __restrict__ mask,
                           double* __restrict__ out, const int* __restrict__ colmap) {
  const int col = blockIdx.y;
  const int src = colmap ? colmap[col] : col;
  const double* f = flat + (long long)src * fstride;
  double* o = out + (long long)col * 3 * pd.nnode;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < pd.nnode; n += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    node_coords(n, pd, i, j, k);
    const bool inside = i < un.nx && j < un.ny && k < un.nz;
    const unsigned m = mask ? mask[n] : 7u;
    const long long s = inside ? ((long long)i * un.ny + j) * un.nz + k : 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) o[3 * n + a] = (inside && ((m >> a) & 1u)) ? f[3 * s + a] : 0.0;
  }
}

__global__ void unpad_kernel(const double* __restrict__ padded, Geo un, Geo pd, double* __restrict__ flat, long long fstride,
                             const int* __restrict__ colmap) {
  const int col = blockIdx.y;
  const int dst = colmap ? colmap[col] : col;
  const double* p = padded + (long long)col * 3 * pd.nnode;
  double* f = flat + (long long)dst * fstride;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < un.nnode; n += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    node_coords(n, un, i, j, k);
    const long long s = ((long long)i * pd.ny + j) * pd.nz + k;
#pragma unroll
    for (int a = 0; a < 3; ++a) f[3 * n + a] = p[3 * s + a];
  }
}

// per-column norms of a flat block (host decides which columns are zero)
__global__ void colnorm_kernel(const double* __restrict__ v, long long n, double* __restrict__ out, double* partial, unsigned* count) {
  const int col = blockIdx.y;
  double a = 0.0, z = 0.0;
  const double* p = v + (long long)col * n;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) a += p[t] * p[t];
  block_reduce2<0, 0>(a, z);
  if (last_block_combine<0, 0>(a, z, partial, count, col)) out[col] = sqrt(a);
}

__global__ void zero_flat_cols_kernel(double* __restrict__ v, long long n, const int* __restrict__ cols) {
  double* p = v + (long long)cols[blockIdx.y] * n;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) p[t] = 0.0;
}

}  // namespace tfb
