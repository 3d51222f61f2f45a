// Device kernels of the hex8 SIMP / geometric-multigrid path (sm_100a).
//
// Vector layout in HBM: a block of R columns is [R][nx][ny][nz][3] in the work
// precision, i.e. every column is the reference's flat dof vector
// (dof = 3 * node + component, node in C order) of a padded level grid.
// Element fields are [ex][ey][ez].  A node-centric formulation is used for
// every operator: thread n computes its own 3 outputs from the (up to) 8
// elements around it, so no atomics and no scatter conflicts are needed and
// every write is coalesced along z.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace tfb {

struct Geo {
  int ex, ey, ez;   // elements
  int nx, ny, nz;   // nodes = elements + 1
  long long nnode;  // nx * ny * nz
};

template <typename T> struct K0Param { T k[576]; };

// corner numbering of the reference element (deep_frame/topology_optimization.py:246-249)
__host__ __device__ constexpr int corner_id(int x, int y, int z) {
  return z * 4 + (y ? (x ? 2 : 3) : (x ? 1 : 0));
}

__device__ __forceinline__ void node_coords(long long n, const Geo& g, int& i, int& j, int& k) {
  k = static_cast<int>(n % g.nz);
  long long r = n / g.nz;
  j = static_cast<int>(r % g.ny);
  i = static_cast<int>(r / g.ny);
}

template <typename T>
__device__ __forceinline__ void load_masked(const T* __restrict__ u, const uint8_t* __restrict__ mask,
                                            long long node, T& u0, T& u1, T& u2) {
  const T* p = u + 3 * node;
  const unsigned m = mask ? mask[node] : 7u;
  u0 = (m & 1u) ? p[0] : T(0);
  u1 = (m & 2u) ? p[1] : T(0);
  u2 = (m & 4u) ? p[2] : T(0);
}

// ---------------------------------------------------------------------------
// Fine-level operator at one node: out = sum_e E_e K0[c_n(e), :] (mask*u)_e.
// The 27 neighbours are visited once; each neighbour's 3 values feed the
// per-element accumulators of every element it shares with the node.  All
// K0 indices are compile-time constants, so K0 is read from the kernel's
// constant bank.  64 (neighbour, element) pairs x 9 FMA = 576 FMA per node.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void fine_node(const K0Param<T>& K, const Geo& g, const T* __restrict__ E,
                                          const uint8_t* __restrict__ mask, const T* __restrict__ u,
                                          int i, int j, int k, T out[3]) {
  T acc[8][3];
#pragma unroll
  for (int e = 0; e < 8; ++e) { acc[e][0] = T(0); acc[e][1] = T(0); acc[e][2] = T(0); }
#pragma unroll
  for (int di = -1; di <= 1; ++di) {
#pragma unroll
    for (int dj = -1; dj <= 1; ++dj) {
#pragma unroll
      for (int dk = -1; dk <= 1; ++dk) {
        const int ni = i + di, nj = j + dj, nk = k + dk;
        T u0 = T(0), u1 = T(0), u2 = T(0);
        if ((unsigned)ni < (unsigned)g.nx && (unsigned)nj < (unsigned)g.ny && (unsigned)nk < (unsigned)g.nz)
          load_masked(u, mask, ((long long)ni * g.ny + nj) * g.nz + nk, u0, u1, u2);
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int ox = e >> 2, oy = (e >> 1) & 1, oz = e & 1;     // element (i-1+ox, j-1+oy, k-1+oz)
          const int cx = 1 - ox + di, cy = 1 - oy + dj, cz = 1 - oz + dk;
          if (cx < 0 || cx > 1 || cy < 0 || cy > 1 || cz < 0 || cz > 1) continue;
          const int cn = corner_id(1 - ox, 1 - oy, 1 - oz);
          const int cm = corner_id(cx, cy, cz);
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            const int row = (3 * cn + a) * 24 + 3 * cm;
            acc[e][a] += K.k[row] * u0 + K.k[row + 1] * u1 + K.k[row + 2] * u2;
          }
        }
      }
    }
  }
  out[0] = out[1] = out[2] = T(0);
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    const int ei = i - 1 + (e >> 2), ej = j - 1 + ((e >> 1) & 1), ek = k - 1 + (e & 1);
    if ((unsigned)ei < (unsigned)g.ex && (unsigned)ej < (unsigned)g.ey && (unsigned)ek < (unsigned)g.ez) {
      const T w = E[((long long)ei * g.ey + ej) * g.ez + ek];
      out[0] += w * acc[e][0];
      out[1] += w * acc[e][1];
      out[2] += w * acc[e][2];
    }
  }
}

// ---------------------------------------------------------------------------
// Coarse-level (Galerkin block) operator at one node for CB columns at once:
// out[c] = sum_e B_e[c_n(e) rows, :] (mask*u_c)_e.  Each block value loaded is
// reused for CB columns.  Blocks are stored entry-major ([576][nelem]), so the
// threads of a warp (consecutive nodes along z) read consecutive elements and
// every block load is one coalesced transaction.
// ---------------------------------------------------------------------------
template <typename T, int CB>
__device__ __forceinline__ void block_node(const Geo& g, const T* __restrict__ B, const uint8_t* __restrict__ mask,
                                           const T* __restrict__ u, long long colstride, int ncol,
                                           int i, int j, int k, T out[CB][3]) {
#pragma unroll
  for (int c = 0; c < CB; ++c) { out[c][0] = T(0); out[c][1] = T(0); out[c][2] = T(0); }
  long long ebase[8];
  bool evalid[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    const int ei = i - 1 + (e >> 2), ej = j - 1 + ((e >> 1) & 1), ek = k - 1 + (e & 1);
    evalid[e] = (unsigned)ei < (unsigned)g.ex && (unsigned)ej < (unsigned)g.ey && (unsigned)ek < (unsigned)g.ez;
    ebase[e] = evalid[e] ? (((long long)ei * g.ey + ej) * g.ez + ek) : 0;
  }
#pragma unroll
  for (int di = -1; di <= 1; ++di) {
#pragma unroll
    for (int dj = -1; dj <= 1; ++dj) {
#pragma unroll
      for (int dk = -1; dk <= 1; ++dk) {
        const int ni = i + di, nj = j + dj, nk = k + dk;
        if (!((unsigned)ni < (unsigned)g.nx && (unsigned)nj < (unsigned)g.ny && (unsigned)nk < (unsigned)g.nz)) continue;
        const long long node = ((long long)ni * g.ny + nj) * g.nz + nk;
        T uv[CB][3];
#pragma unroll
        for (int c = 0; c < CB; ++c) {
          if (c < ncol) load_masked(u + c * colstride, mask, node, uv[c][0], uv[c][1], uv[c][2]);
          else { uv[c][0] = uv[c][1] = uv[c][2] = T(0); }
        }
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int ox = e >> 2, oy = (e >> 1) & 1, oz = e & 1;
          const int cx = 1 - ox + di, cy = 1 - oy + dj, cz = 1 - oz + dk;
          if (cx < 0 || cx > 1 || cy < 0 || cy > 1 || cz < 0 || cz > 1) continue;
          if (!evalid[e]) continue;
          const int cn = corner_id(1 - ox, 1 - oy, 1 - oz);
          const int cm = corner_id(cx, cy, cz);
          const long long est = (long long)g.ex * g.ey * g.ez;
          const T* bp = B + ebase[e] + (long long)((3 * cn) * 24 + 3 * cm) * est;
          T b[9];
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            b[3 * a + 0] = bp[(a * 24 + 0) * est];
            b[3 * a + 1] = bp[(a * 24 + 1) * est];
            b[3 * a + 2] = bp[(a * 24 + 2) * est];
          }
#pragma unroll
          for (int c = 0; c < CB; ++c) {
#pragma unroll
            for (int a = 0; a < 3; ++a)
              out[c][a] += b[3 * a] * uv[c][0] + b[3 * a + 1] * uv[c][1] + b[3 * a + 2] * uv[c][2];
          }
        }
      }
    }
  }
}

// Epilogue modes of the level operators.
enum ApplyMode : int {
  MODE_APPLY = 0,   // y = mask * A u
  MODE_RESID = 1,   // y = mask * (b - A u)
  MODE_JACOBI = 2,  // y = u + s * inv * (b - A u)
  MODE_CHEB = 3,    // res -= A u; dnew = c1 * u + c2 * inv * res; x += dnew   (u is the direction d)
};

template <typename T>
struct LevelArgs {
  Geo g;
  const T* E;            // fine: element moduli [ex][ey][ez]; coarse: blocks entry-major [576][nelem]
  const uint8_t* mask;   // per-node 3-bit live mask
  const T* inv;          // inverse diagonal [ndof] (Jacobi / Chebyshev)
  const T* u;            // operator input, [R][ndof]
  const T* b;            // right-hand side (RESID / JACOBI)
  T* y;                  // output (APPLY / RESID / JACOBI) or new direction (CHEB)
  T* res;                // CHEB residual, updated in place
  T* x;                  // CHEB solution, updated in place
  long long colstride;   // = 3 * nnode (columns are contiguous)
  int ncol;
  const int* active;     // optional per-column flag; inactive columns are skipped
  const int* gate;       // optional device flag; the whole launch is skipped while *gate == 0
  T s, c1, c2;           // epilogue scalars
};

template <typename T>
__device__ __forceinline__ void epilogue(const LevelArgs<T>& a, int mode, long long col_off, long long node,
                                         unsigned m, const T av[3]) {
  const long long d0 = col_off + 3 * node;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const bool live = (m >> q) & 1u;
    const long long d = d0 + q;
    if (mode == MODE_APPLY) {
      a.y[d] = live ? av[q] : T(0);
    } else if (mode == MODE_RESID) {
      a.y[d] = live ? (a.b[d] - av[q]) : T(0);
    } else if (mode == MODE_JACOBI) {
      a.y[d] = a.u[d] + a.s * a.inv[3 * node + q] * (a.b[d] - (live ? av[q] : T(0)));
    } else {  // MODE_CHEB
      const T r = a.res[d] - (live ? av[q] : T(0));
      const T dn = a.c1 * a.u[d] + a.c2 * a.inv[3 * node + q] * r;
      a.res[d] = r;
      a.y[d] = dn;
      a.x[d] += dn;
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) fine_level_kernel(const __grid_constant__ K0Param<T> K, const LevelArgs<T> a, int mode) {
  const int col = blockIdx.y;
  if (a.gate && !*a.gate) return;
  if (a.active && !a.active[col]) return;
  const long long off = (long long)col * a.colstride;
  const T* u = a.u + off;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < a.g.nnode; n += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    node_coords(n, a.g, i, j, k);
    T av[3];
    fine_node<T>(K, a.g, a.E, a.mask, u, i, j, k, av);
    const unsigned m = a.mask ? a.mask[n] : 7u;
    epilogue(a, mode, off, n, m, av);
  }
}

template <typename T, int CB>
__global__ void __launch_bounds__(128) block_level_kernel(const LevelArgs<T> a, int mode) {
  const int c0 = blockIdx.y * CB;
  if (a.gate && !*a.gate) return;
  const int nc = min(CB, a.ncol - c0);
  bool any = false;
  for (int c = 0; c < nc; ++c) any |= (!a.active || a.active[c0 + c]);
  if (!any) return;
  const long long off = (long long)c0 * a.colstride;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < a.g.nnode; n += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    node_coords(n, a.g, i, j, k);
    T av[CB][3];
    block_node<T, CB>(a.g, a.E, a.mask, a.u + off, a.colstride, nc, i, j, k, av);
    const unsigned m = a.mask ? a.mask[n] : 7u;
#pragma unroll
    for (int c = 0; c < CB; ++c) {
      if (c < nc && (!a.active || a.active[c0 + c])) epilogue(a, mode, off + c * a.colstride, n, m, av[c]);
    }
  }
}

// ---------------------------------------------------------------------------
// Element energies u_e^T K0 u_e.  With comb == nullptr, column r contributes
// coef[r] * u_r,e^T K0 u_r,e; otherwise combination j forms w = U comb[:, j]
// on the fly and contributes coef[j] * w_e^T K0 w_e.  out[e] = scale[e] * sum
// (+ out[e] when accumulate).  With per_column set, out is [R][nelem] and
// holds the plain energies of every column.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(128) energy_kernel(const __grid_constant__ K0Param<T> K, Geo g, const T* __restrict__ u,
                                                     long long colstride, int ncol, const double* __restrict__ comb, int ncomb,
                                                     const double* __restrict__ coef, const double* __restrict__ scale,
                                                     double* __restrict__ out, int accumulate, int per_column) {
  const long long nelem = (long long)g.ex * g.ey * g.ez;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nelem; e += (long long)gridDim.x * blockDim.x) {
    const int ek = static_cast<int>(e % g.ez);
    const long long r1 = e / g.ez;
    const int ej = static_cast<int>(r1 % g.ey);
    const int ei = static_cast<int>(r1 / g.ey);
    long long nodes[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int cx = (c == 1 || c == 2 || c == 5 || c == 6) ? 1 : 0;
      const int cy = (c == 2 || c == 3 || c == 6 || c == 7) ? 1 : 0;
      const int cz = c >> 2;
      nodes[c] = ((long long)(ei + cx) * g.ny + (ej + cy)) * g.nz + (ek + cz);
    }
    const int terms = comb ? ncomb : ncol;
    double total = 0.0;
    for (int t = 0; t < terms; ++t) {
      T w[24];
      if (comb) {
#pragma unroll
        for (int q = 0; q < 24; ++q) w[q] = T(0);
        for (int r = 0; r < ncol; ++r) {
          const T cr = static_cast<T>(comb[(long long)r * ncomb + t]);
          if (cr == T(0)) continue;
          const T* ur = u + r * colstride;
#pragma unroll
          for (int c = 0; c < 8; ++c) {
            w[3 * c + 0] += cr * ur[3 * nodes[c] + 0];
            w[3 * c + 1] += cr * ur[3 * nodes[c] + 1];
            w[3 * c + 2] += cr * ur[3 * nodes[c] + 2];
          }
        }
      } else {
        const T* ur = u + t * colstride;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          w[3 * c + 0] = ur[3 * nodes[c] + 0];
          w[3 * c + 1] = ur[3 * nodes[c] + 1];
          w[3 * c + 2] = ur[3 * nodes[c] + 2];
        }
      }
      T q = T(0);
#pragma unroll
      for (int r = 0; r < 24; ++r) {
        T kr = T(0);
#pragma unroll
        for (int c = 0; c < 24; ++c) kr += K.k[r * 24 + c] * w[c];
        q += w[r] * kr;
      }
      if (per_column) {
        out[(long long)t * nelem + e] = static_cast<double>(q);
      } else {
        total += (coef ? coef[t] : 1.0) * static_cast<double>(q);
      }
    }
    if (!per_column) {
      const double v = (scale ? scale[e] : 1.0) * total;
      out[e] = accumulate ? out[e] + v : v;
    }
  }
}

// ---------------------------------------------------------------------------
// Full-weighting restriction (conv3d with (x)[1/2, 1, 1/2], stride 2, padding 1,
// deep_frame/topology_multigrid.py:314) and its transpose, the trilinear
// prolongation (:316).  Columns on blockIdx.y.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void restrict_kernel(Geo fine, Geo coarse, const T* __restrict__ r, long long fstride, T* __restrict__ out,
                                long long cstride, const uint8_t* __restrict__ cmask, const int* __restrict__ active) {
  const int col = blockIdx.y;
  if (active && !active[col]) return;
  const T* rc = r + col * fstride;
  T* oc = out + col * cstride;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < coarse.nnode; n += (long long)gridDim.x * blockDim.x) {
    int I, J, Kc;
    node_coords(n, coarse, I, J, Kc);
    T acc0 = T(0), acc1 = T(0), acc2 = T(0);
#pragma unroll
    for (int di = -1; di <= 1; ++di) {
      const int fi = 2 * I + di;
      if ((unsigned)fi >= (unsigned)fine.nx) continue;
#pragma unroll
      for (int dj = -1; dj <= 1; ++dj) {
        const int fj = 2 * J + dj;
        if ((unsigned)fj >= (unsigned)fine.ny) continue;
#pragma unroll
        for (int dk = -1; dk <= 1; ++dk) {
          const int fk = 2 * Kc + dk;
          if ((unsigned)fk >= (unsigned)fine.nz) continue;
          const T w = T((di ? 0.5 : 1.0) * (dj ? 0.5 : 1.0) * (dk ? 0.5 : 1.0));
          const T* p = rc + 3 * (((long long)fi * fine.ny + fj) * fine.nz + fk);
          acc0 += w * p[0]; acc1 += w * p[1]; acc2 += w * p[2];
        }
      }
    }
    const unsigned m = cmask ? cmask[n] : 7u;
    oc[3 * n + 0] = (m & 1u) ? acc0 : T(0);
    oc[3 * n + 1] = (m & 2u) ? acc1 : T(0);
    oc[3 * n + 2] = (m & 4u) ? acc2 : T(0);
  }
}

// x_fine += mask * P c  (P = transpose of the restriction)
template <typename T>
__global__ void prolong_add_kernel(Geo fine, Geo coarse, const T* __restrict__ c, long long cstride, T* __restrict__ x,
                                   long long fstride, const uint8_t* __restrict__ fmask, const int* __restrict__ active) {
  const int col = blockIdx.y;
  if (active && !active[col]) return;
  const T* cc = c + col * cstride;
  T* xc = x + col * fstride;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < fine.nnode; n += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    node_coords(n, fine, i, j, k);
    int I0[3], I1[3];
    T w0[3], w1[3];
    const int idx[3] = {i, j, k};
    const int lim[3] = {coarse.nx, coarse.ny, coarse.nz};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if ((idx[d] & 1) == 0) { I0[d] = idx[d] >> 1; w0[d] = T(1); I1[d] = -1; w1[d] = T(0); }
      else { I0[d] = (idx[d] - 1) >> 1; w0[d] = T(0.5); I1[d] = (idx[d] + 1) >> 1; w1[d] = T(0.5); }
      if (I1[d] >= lim[d]) { I1[d] = -1; }
    }
    T acc0 = T(0), acc1 = T(0), acc2 = T(0);
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      const int ci = a ? I1[0] : I0[0];
      const T wa = a ? w1[0] : w0[0];
      if (ci < 0) continue;
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const int cj = b ? I1[1] : I0[1];
        const T wb = b ? w1[1] : w0[1];
        if (cj < 0) continue;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int ck = q ? I1[2] : I0[2];
          const T wq = q ? w1[2] : w0[2];
          if (ck < 0) continue;
          const T w = wa * wb * wq;
          const T* p = cc + 3 * (((long long)ci * coarse.ny + cj) * coarse.nz + ck);
          acc0 += w * p[0]; acc1 += w * p[1]; acc2 += w * p[2];
        }
      }
    }
    const unsigned m = fmask ? fmask[n] : 7u;
    if (m & 1u) xc[3 * n + 0] += acc0;
    if (m & 2u) xc[3 * n + 1] += acc1;
    if (m & 4u) xc[3 * n + 2] += acc2;
  }
}

}  // namespace tfb
