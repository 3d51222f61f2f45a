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
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>
#include "tf_reduce.cuh"

namespace tfb {

struct Geo {
  int ex, ey, ez;   // elements
  int nx, ny, nz;   // nodes = elements + 1
  long long nnode;  // nx * ny * nz
};

// corner numbering of the reference element (deep_frame/topology_optimization.py:246-249)
__host__ __device__ constexpr int corner_id(int x, int y, int z) {
  return z * 4 + (y ? (x ? 2 : 3) : (x ? 1 : 0));
}

template <typename T> struct K0Param { T k[576]; };

// Element stiffness of the finest level in constant memory.  A handle claims one
// of K0_SLOTS slots (per distinct K0); the operator kernels are instantiated per
// slot so every coefficient is a compile-time constant-bank operand of its FMA.
constexpr int K0_SLOTS = 2;
__constant__ float c_k0f[K0_SLOTS][576];
__constant__ double c_k0d[K0_SLOTS][576];
// For a box element with an axis-aligned orthotropic (or isotropic) material,
// K0 is invariant under the 8 reflections of the element: with R the corner
// bits of the row corner c,  K0[3c+a][3d+b] = s_a s_b K0[a][3(d xor R)+b]
// (s = -1 on reflected axes).  Only the 72 coefficients of corner 0's rows are
// distinct, and every index and sign is a compile-time constant.
__constant__ float c_kcf[K0_SLOTS][72];
__constant__ double c_kcd[K0_SLOTS][72];

__host__ __device__ constexpr int corner_x(int c) { return (c == 1 || c == 2 || c == 5 || c == 6) ? 1 : 0; }
__host__ __device__ constexpr int corner_y(int c) { return (c == 2 || c == 3 || c == 6 || c == 7) ? 1 : 0; }
__host__ __device__ constexpr int corner_z(int c) { return c >> 2; }

template <typename T, int SLOT, bool REFLECT> struct K0Const;
template <int SLOT> struct K0Const<float, SLOT, false> {
  __device__ __forceinline__ float operator()(int cn, int a, int cm, int b) const { return c_k0f[SLOT][(3 * cn + a) * 24 + 3 * cm + b]; }
};
template <int SLOT> struct K0Const<double, SLOT, false> {
  __device__ __forceinline__ double operator()(int cn, int a, int cm, int b) const { return c_k0d[SLOT][(3 * cn + a) * 24 + 3 * cm + b]; }
};
template <typename T, int SLOT>
__device__ __forceinline__ T reflected_k0(const T (&table)[K0_SLOTS][72], int cn, int a, int cm, int b) {
  const int rx = corner_x(cn), ry = corner_y(cn), rz = corner_z(cn);
  const int d = corner_id(corner_x(cm) ^ rx, corner_y(cm) ^ ry, corner_z(cm) ^ rz);
  const int ra = a == 0 ? rx : (a == 1 ? ry : rz);
  const int rb = b == 0 ? rx : (b == 1 ? ry : rz);
  const T v = table[SLOT][(a * 8 + d) * 3 + b];
  return (ra ^ rb) ? -v : v;
}
template <int SLOT> struct K0Const<float, SLOT, true> {
  __device__ __forceinline__ float operator()(int cn, int a, int cm, int b) const { return reflected_k0<float, SLOT>(c_kcf, cn, a, cm, b); }
};
template <int SLOT> struct K0Const<double, SLOT, true> {
  __device__ __forceinline__ double operator()(int cn, int a, int cm, int b) const { return reflected_k0<double, SLOT>(c_kcd, cn, a, cm, b); }
};


// Node counts stay below 2^31 (tf_create checks it), so 32-bit division suffices: a 64-bit one is
// a long instruction sequence per call.
__device__ __forceinline__ void node_coords(long long n, const Geo& g, int& i, int& j, int& k) {
  const unsigned u = static_cast<unsigned>(n), nz = static_cast<unsigned>(g.nz), ny = static_cast<unsigned>(g.ny);
  const unsigned r = u / nz;
  k = static_cast<int>(u - r * nz);
  const unsigned ii = r / ny;
  j = static_cast<int>(r - ii * ny);
  i = static_cast<int>(ii);
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

// Storage rounding of the work-precision V-cycle vectors: 0 none, 1 bfloat16, 2 float16.  With a
// 16-bit storage precision every V-cycle vector value is rounded to that format (round to nearest)
// when it is stored, while the arithmetic stays FP32: the vectors then hold exactly what 16-bit
// buffers would, so the solver's iteration counts are those of 16-bit storage (the buffers
// themselves stay FP32).
__device__ __forceinline__ float round_store(float v, int mode) {
  if (mode == 1) return __bfloat162float(__float2bfloat16_rn(v));
  if (mode == 2) return __half2float(__float2half_rn(v));
  return v;
}
__device__ __forceinline__ double round_store(double v, int) { return v; }
// compile-time form for the level operators: RND = 0 compiles to a plain store
template <int RND, typename T>
__device__ __forceinline__ T rs(T v) {
  if constexpr (RND == 0) return v;
  else return round_store(v, RND);
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
  int round;             // storage rounding of the outputs (round_store mode; selects the RND instantiation)
  // Fused PCG curvature (finest level, FP64 operator, MODE_APPLY): every warp writes the sum of
  // u . y over its nodes of column c to dot_out[(c * gridDim.x + blockIdx.x) * warps + warp]
  double* dot_out;
};

template <typename T, int RND>
__device__ __forceinline__ void epilogue(const LevelArgs<T>& a, int mode, long long col_off, long long node,
                                         unsigned m, const T av[3]) {
  const long long d0 = col_off + 3 * node;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const bool live = (m >> q) & 1u;
    const long long d = d0 + q;
    if (mode == MODE_APPLY) {
      a.y[d] = rs<RND>(live ? av[q] : T(0));
    } else if (mode == MODE_RESID) {
      a.y[d] = rs<RND>(live ? (a.b[d] - av[q]) : T(0));
    } else if (mode == MODE_JACOBI) {
      a.y[d] = rs<RND>(a.u[d] + a.s * a.inv[3 * node + q] * (a.b[d] - (live ? av[q] : T(0))));
    } else {  // MODE_CHEB
      const T r = rs<RND>(a.res[d] - (live ? av[q] : T(0)));
      const T dn = rs<RND>(a.c1 * a.u[d] + a.c2 * a.inv[3 * node + q] * r);
      a.res[d] = r;
      a.y[d] = dn;
      a.x[d] = rs<RND>(a.x[d] + dn);
    }
  }
}

// Per-column epilogue inputs besides A u (b; res and x for the Chebyshev update), loaded before the
// operator so that their latency overlaps its arithmetic.  The other inputs (the direction u and
// the inverse diagonal, the same for every column) are read afterwards.
template <typename T>
struct EpiPre {
  T v[2][3];
};

template <typename T>
__device__ __forceinline__ void epilogue_load(const LevelArgs<T>& a, int mode, long long col_off, long long node, EpiPre<T>& in) {
  const long long d0 = col_off + 3 * node;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    if (mode == MODE_RESID || mode == MODE_JACOBI) {
      in.v[0][q] = a.b[d0 + q];
    } else if (mode == MODE_CHEB) {
      in.v[0][q] = a.res[d0 + q];
      in.v[1][q] = a.x[d0 + q];
    }
  }
}

// epilogue() from prefetched inputs (the same arithmetic)
template <typename T, int RND>
__device__ __forceinline__ void epilogue_pre(const LevelArgs<T>& a, int mode, long long col_off, long long node, unsigned m,
                                             const T av[3], const EpiPre<T>& in) {
  const long long d0 = col_off + 3 * node;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const bool live = (m >> q) & 1u;
    const long long d = d0 + q;
    if (mode == MODE_APPLY) {
      a.y[d] = rs<RND>(live ? av[q] : T(0));
    } else if (mode == MODE_RESID) {
      a.y[d] = rs<RND>(live ? (in.v[0][q] - av[q]) : T(0));
    } else if (mode == MODE_JACOBI) {
      a.y[d] = rs<RND>(a.u[d] + a.s * a.inv[3 * node + q] * (in.v[0][q] - (live ? av[q] : T(0))));
    } else {  // MODE_CHEB
      const T r = rs<RND>(in.v[0][q] - (live ? av[q] : T(0)));
      const T dn = rs<RND>(a.c1 * a.u[d] + a.c2 * a.inv[3 * node + q] * r);
      a.res[d] = r;
      a.y[d] = dn;
      a.x[d] = rs<RND>(in.v[1][q] + dn);
    }
  }
}

// ---------------------------------------------------------------------------
// Shared-memory tiled level operators.  A CTA owns a tile of TX x TY x tz
// output nodes (tz <= TZMAX chosen per grid so that the z extent is covered
// with little waste) and stages the tile's input nodes with a one-node halo,
// already masked and zero-padded outside the grid, in a fixed-pitch shared
// array: every neighbour offset of the 27-point stencil is then a
// compile-time immediate and the inner loop has no bounds or mask tests.
// The element moduli (finest level) are staged the same way, with zeros for
// elements outside the grid.
// ---------------------------------------------------------------------------
constexpr int TX = 4, TY = 8, TZMAX = 9;
constexpr int HX = TX + 2, HY = TY + 2, HZ = TZMAX + 2;   // halo tile pitch (nodes)
constexpr int EX = TX + 1, EY = TY + 1, EZ = TZMAX + 1;   // element tile pitch
constexpr int HALO = HX * HY * HZ;

struct TileMap {
  int tiles_x, tiles_y, tiles_z, tz;
};

__host__ inline TileMap tile_map(const Geo& g) {
  TileMap m;
  const int nzt = (g.nz + TZMAX - 1) / TZMAX;
  m.tz = (g.nz + nzt - 1) / nzt;
  m.tiles_x = (g.nx + TX - 1) / TX;
  m.tiles_y = (g.ny + TY - 1) / TY;
  m.tiles_z = (g.nz + m.tz - 1) / m.tz;
  return m;
}

template <typename T, int CB>
constexpr size_t stencil_smem_bytes() {
  return sizeof(T) * 3 * (size_t)HALO * CB;
}

// Stage the masked input tiles of nc <= CB columns in one pass over the halo: the mask is read once
// per node and the columns' loads are issued together, independent of the mask load (the mask is
// applied when storing).
template <typename T, int CB>
__device__ __forceinline__ void stage_tiles(T* __restrict__ s, const Geo& g, const T* __restrict__ u, long long colstride, int nc,
                                            const uint8_t* __restrict__ mask, int x0, int y0, int z0, int tz) {
  const int hz = tz + 2;
  const int count = HX * HY * hz;
  for (int t = threadIdx.x; t < count; t += blockDim.x) {
    const int cz = t % hz, r = t / hz, cy = r % HY, cx = r / HY;
    const int gx = x0 - 1 + cx, gy = y0 - 1 + cy, gz = z0 - 1 + cz;
    const bool in = (unsigned)gx < (unsigned)g.nx && (unsigned)gy < (unsigned)g.ny && (unsigned)gz < (unsigned)g.nz;
    const long long node = in ? ((long long)gx * g.ny + gy) * g.nz + gz : 0;
    const unsigned m = in ? (mask ? mask[node] : 7u) : 0u;
    T v[CB][3];
#pragma unroll
    for (int c = 0; c < CB; ++c) {
      v[c][0] = v[c][1] = v[c][2] = T(0);
      if (in && c < nc) {
        const T* p = u + c * colstride + 3 * node;
        v[c][0] = p[0];
        v[c][1] = p[1];
        v[c][2] = p[2];
      }
    }
    const int so = 3 * ((cx * HY + cy) * HZ + cz);
#pragma unroll
    for (int c = 0; c < CB; ++c) {
      if (c < nc) {
        T* d = s + c * HALO * 3 + so;
        d[0] = (m & 1u) ? v[c][0] : T(0);
        d[1] = (m & 2u) ? v[c][1] : T(0);
        d[2] = (m & 4u) ? v[c][2] : T(0);
      }
    }
  }
}

// Finest-level tile.  The thread block is (TZ, TY, FTXT) and every thread owns
// NPT nodes adjacent in x, so a CTA covers (FTXT * NPT) x TY x TZ output nodes.
// Inputs are staged component-planar with a row pitch chosen so that a warp
// reads distinct banks; no index needs a runtime division.
constexpr int FTXT = 4;   // threads along x
template <typename T, int TZ> struct FineTile {
  // row pitch (elements): conflict-free warp reads for 8-high tiles; 7- and 9-high tiles mix x rows
  // in a warp and reach two-way conflicts at best (7 high: rows packed, P = 9)
  static constexpr int P = TZ == 7 ? 9 : (sizeof(T) == 4 ? (TZ == 8 ? 24 : 41) : (TZ == 8 ? 24 : 25));
};

template <typename T, int NPT, typename KC>
__device__ __forceinline__ void fine_tile_nodes(const KC& K, const T* __restrict__ su, const T* __restrict__ sE, int plane, int hy, int p,
                                                int ey, int ez, int lx, int ly, int lz, T out[NPT][3]) {
  T acc[NPT][8][3];
#pragma unroll
  for (int q = 0; q < NPT; ++q)
#pragma unroll
    for (int e = 0; e < 8; ++e) { acc[q][e][0] = T(0); acc[q][e][1] = T(0); acc[q][e][2] = T(0); }
  const int x0 = lx * NPT;   // first node of this thread in the tile
  const T* base = su + ((x0 + 1) * hy + (ly + 1)) * p + (lz + 1);
#pragma unroll
  for (int px = -1; px <= NPT; ++px) {
#pragma unroll
    for (int dj = -1; dj <= 1; ++dj) {
#pragma unroll
      for (int dk = -1; dk <= 1; ++dk) {
        const T* ptr = base + (px * hy + dj) * p + dk;
        const T u0 = ptr[0], u1 = ptr[plane], u2 = ptr[2 * plane];
#pragma unroll
        for (int q = 0; q < NPT; ++q) {
          const int di = px - q;
          if (di < -1 || di > 1) continue;
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            const int ox = e >> 2, oy = (e >> 1) & 1, oz = e & 1;
            const int cx = 1 - ox + di, cy = 1 - oy + dj, cz = 1 - oz + dk;
            if (cx < 0 || cx > 1 || cy < 0 || cy > 1 || cz < 0 || cz > 1) continue;
            const int cn = corner_id(1 - ox, 1 - oy, 1 - oz);
            const int cm = corner_id(cx, cy, cz);
#pragma unroll
            for (int a = 0; a < 3; ++a) {
              T t = fma(K(cn, a, cm, 0), u0, acc[q][e][a]);
              t = fma(K(cn, a, cm, 1), u1, t);
              acc[q][e][a] = fma(K(cn, a, cm, 2), u2, t);
            }
          }
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < NPT; ++q) {
    const T* eb = sE + ((x0 + q) * ey + ly) * ez + lz;
    out[q][0] = out[q][1] = out[q][2] = T(0);
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const T w = eb[((e >> 2) * ey + ((e >> 1) & 1)) * ez + (e & 1)];
      out[q][0] = fma(w, acc[q][e][0], out[q][0]);
      out[q][1] = fma(w, acc[q][e][1], out[q][1]);
      out[q][2] = fma(w, acc[q][e][2], out[q][2]);
    }
  }
}

// One CTA handles one tile for `cpb` (<= 64) consecutive columns: the element
// moduli, the halo's global indices and live bits, the owned nodes' live bits and
// the chunk's active-column mask are read once; while column c is computed from
// one shared-memory halo buffer, column c+1's halo is loading into registers and
// then goes to the other buffer, so the global-load latency overlaps the FMAs and
// one barrier per column suffices.
//
// PCG (FP64 only, MODE_APPLY): the curvature partials of LevelArgs::dot_out, in their own
// instantiation so that the plain applies keep their registers.
template <typename T, int SLOT, bool REFLECT, int TZ, int NPT, int RND, bool PCG>
__device__ __forceinline__ void fine_level_body(const VGrid vg_, const LevelArgs<T>& a, int mode, TileMap tm, int cpb) {
  TF_VGRID(vg_);
  static_assert(!PCG || sizeof(T) == 8, "the fused PCG step is an FP64 operator");
  constexpr int TXN = FTXT * NPT;                 // tile nodes along x
  constexpr int SHX = TXN + 2, SHY = TY + 2;      // staged halo extents
  constexpr int FMAXH = (SHX * SHY * (TZ + 2) + FTXT * TY * TZ - 1) / (FTXT * TY * TZ);   // halo nodes staged per thread
  constexpr int P = FineTile<T, TZ>::P;
  constexpr int PLANE = SHX * SHY * P;
  constexpr int SEX = TXN + 1, SEY = TY + 1, SEZ = TZ + 1;
  constexpr int NT = FTXT * TY * TZ;
  constexpr int HALO_N = SHX * SHY * (TZ + 2);
  static_assert(HALO_N <= FMAXH * NT, "halo exceeds the per-thread staging slots");
  extern __shared__ __align__(16) unsigned char fine_smem[];
  T* su = reinterpret_cast<T*>(fine_smem);   // two halo buffers of 3 * PLANE
  T* sE = su + 6 * PLANE;
  const K0Const<T, SLOT, REFLECT> K;
  if (a.gate && !*a.gate) return;
  const int c_begin = blockIdx.y * cpb;
  const int c_end = min(a.ncol, c_begin + cpb);
  const Geo& g = a.g;
  const int b = blockIdx.x;
  const int bz = b % tm.tiles_z, r = b / tm.tiles_z, by = r % tm.tiles_y, bx = r / tm.tiles_y;
  const int x0 = bx * TXN, y0 = by * TY, z0 = bz * TZ;
  const int lz = threadIdx.x, ly = threadIdx.y, lx = threadIdx.z;
  const int tid = (lx * TY + ly) * TZ + lz;
  // halo slots of this thread: shared offset, global node index (-1 outside) and live bits
  int soff[FMAXH], gnode[FMAXH];
  unsigned live[FMAXH];
#pragma unroll
  for (int h = 0; h < FMAXH; ++h) {
    const int t = tid + h * NT;
    soff[h] = -1;
    gnode[h] = -1;
    live[h] = 0;
    if (t < HALO_N) {
      const int cz = t % (TZ + 2), rr = t / (TZ + 2), cy = rr % SHY, cx = rr / SHY;
      soff[h] = (cx * SHY + cy) * P + cz;
      const int gx = x0 - 1 + cx, gy = y0 - 1 + cy, gz = z0 - 1 + cz;
      if ((unsigned)gx < (unsigned)g.nx && (unsigned)gy < (unsigned)g.ny && (unsigned)gz < (unsigned)g.nz) {
        gnode[h] = (gx * g.ny + gy) * g.nz + gz;
        live[h] = a.mask ? a.mask[gnode[h]] : 7u;
      }
    }
  }
  for (int cx = lx; cx < SEX; cx += FTXT) {
    const int gx = x0 - 1 + cx;
    for (int cy = ly; cy < SEY; cy += TY) {
      const int gy = y0 - 1 + cy;
      for (int cz = lz; cz < SEZ; cz += TZ) {
        const int gz = z0 - 1 + cz;
        T v = T(0);
        if ((unsigned)gx < (unsigned)g.ex && (unsigned)gy < (unsigned)g.ey && (unsigned)gz < (unsigned)g.ez)
          v = a.E[((long long)gx * g.ey + gy) * g.ez + gz];
        sE[(cx * SEY + cy) * SEZ + cz] = v;
      }
    }
  }
  T pre[FMAXH][3];
  auto fetch = [&](int c) {
    const T* u = a.u + (long long)c * a.colstride;
#pragma unroll
    for (int h = 0; h < FMAXH; ++h) {
      pre[h][0] = pre[h][1] = pre[h][2] = T(0);
      if (gnode[h] >= 0) {
        const T* p = u + 3 * (long long)gnode[h];
        if (live[h] & 1u) pre[h][0] = p[0];
        if (live[h] & 2u) pre[h][1] = p[1];
        if (live[h] & 4u) pre[h][2] = p[2];
      }
    }
  };
  // two halo buffers: column c is computed from one while column c+1's halo is stored into the other,
  // so one barrier per column separates them
  auto store = [&](T* buf) {
#pragma unroll
    for (int h = 0; h < FMAXH; ++h) {
      if (soff[h] >= 0) {
        buf[soff[h]] = pre[h][0];
        buf[soff[h] + PLANE] = pre[h][1];
        buf[soff[h] + 2 * PLANE] = pre[h][2];
      }
    }
  };
  // the chunk's active columns as a bit mask (cpb <= 64), read once
  unsigned long long act = 0ull;
  for (int q = c_begin; q < c_end; ++q)
    if (!a.active || a.active[q]) act |= 1ull << (q - c_begin);
  if (!act) return;
  auto next_active = [&](int from) {
    const unsigned long long rest = from - c_begin < 64 ? act >> (from - c_begin) : 0ull;
    return rest ? from + __ffsll(static_cast<long long>(rest)) - 1 : c_end;
  };
  int c = next_active(c_begin);
  T* cur = su;
  T* other = su + 3 * PLANE;
  fetch(c);
  store(cur);
  __syncthreads();
  const int j = y0 + ly, k = z0 + lz;
  const bool owner = j < g.ny && k < g.nz;
  // per-node quantities that do not depend on the column: node index and live bits
  long long node[NPT];
  unsigned mq[NPT];
#pragma unroll
  for (int q = 0; q < NPT; ++q) {
    const int i = x0 + lx * NPT + q;
    node[q] = -1;
    mq[q] = 0u;
    if (owner && i < g.nx) {
      node[q] = ((long long)i * g.ny + j) * g.nz + k;
      mq[q] = a.mask ? a.mask[node[q]] : 7u;
    }
  }
  double dot = 0.0;
  while (c < c_end) {
    const int next = next_active(c + 1);
    if (next < c_end) fetch(next);
    if (owner) {
      const long long off = (long long)c * a.colstride;
      if constexpr (sizeof(T) == 4) {
        // work-precision smoother: the epilogue inputs are fetched before the operator
        EpiPre<T> ep[NPT];
#pragma unroll
        for (int q = 0; q < NPT; ++q)
          if (node[q] >= 0) epilogue_load(a, mode, off, node[q], ep[q]);
        T av[NPT][3];
        fine_tile_nodes<T, NPT>(K, cur, sE, PLANE, SHY, P, SEY, SEZ, lx, ly, lz, av);
#pragma unroll
        for (int q = 0; q < NPT; ++q)
          if (node[q] >= 0) epilogue_pre<T, RND>(a, mode, off, node[q], mq[q], av[q], ep[q]);
      } else {
        T av[NPT][3];
        fine_tile_nodes<T, NPT>(K, cur, sE, PLANE, SHY, P, SEY, SEZ, lx, ly, lz, av);
#pragma unroll
        for (int q = 0; q < NPT; ++q)
          if (node[q] >= 0) epilogue<T, RND>(a, mode, off, node[q], mq[q], av[q]);
        if constexpr (PCG) {
#pragma unroll
          for (int q = 0; q < NPT; ++q) {
            if (node[q] < 0) continue;
            const int sc = ((lx * NPT + q + 1) * SHY + (ly + 1)) * P + (lz + 1);
#pragma unroll
            for (int e = 0; e < 3; ++e)
              if ((mq[q] >> e) & 1u) dot += static_cast<double>(cur[sc + e * PLANE]) * static_cast<double>(av[q][e]);
          }
        }
      }
    }
    if constexpr (PCG) {
      // every lane takes part (non-owners add 0), so the warp's partial is always written
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) dot += __shfl_down_sync(0xffffffffu, dot, o);
      if ((tid & 31) == 0) a.dot_out[((long long)c * gridDim.x + blockIdx.x) * ((NT + 31) / 32) + (tid >> 5)] = dot;
      dot = 0.0;
    }
    if (next >= c_end) break;
    store(other);
    __syncthreads();
    T* t = cur;
    cur = other;
    other = t;
    c = next;
  }
}
template <typename T, int SLOT, bool REFLECT, int TZ, int NPT, int RND, bool PCG>
__global__ void __launch_bounds__(FTXT * TY * TZ, 2) fine_level_kernel(const __grid_constant__ LevelArgs<T> a, int mode, TileMap tm, int cpb) {
  fine_level_body<T, SLOT, REFLECT, TZ, NPT, RND, PCG>(vgrid(), a, mode, tm, cpb);
}

template <typename T, int TZ, int NPT>
constexpr size_t fine_smem_bytes() {
  // two halo buffers (3 component planes each) and the element moduli
  return sizeof(T) * (2 * 3 * (FTXT * NPT + 2) * (TY + 2) * FineTile<T, TZ>::P + (FTXT * NPT + 1) * (TY + 1) * (TZ + 1));
}

// Galerkin levels as assembled 27-point stencils: S[(d * 9 + 3 q + r)][node] is the 3 x 3 coupling of
// the node with its neighbour node + d, summed over the elements holding both.  Per node and column
// that is 243 FMA and 243 / CB coefficient loads, against 576 of each for the element blocks.
//
template <typename T, int CB, int RND>
__device__ __forceinline__ void stencil_level_body(const VGrid vg_, const LevelArgs<T>& a, int mode, TileMap tm) {
  TF_VGRID(vg_);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* su = reinterpret_cast<T*>(smem_raw);   // [CB][HALO][3]
  const int c0 = blockIdx.y * CB;
  if (a.gate && !*a.gate) return;
  const int nc = min(CB, a.ncol - c0);
  bool any = false;
  for (int c = 0; c < nc; ++c) any |= (!a.active || a.active[c0 + c]);
  if (!any) return;
  const Geo& g = a.g;
  const int b = blockIdx.x;
  const int bz = b % tm.tiles_z, r = b / tm.tiles_z, by = r % tm.tiles_y, bx = r / tm.tiles_y;
  const int tz = tm.tz;
  const int x0 = bx * TX, y0 = by * TY, z0 = bz * tz;
  const long long off = (long long)c0 * a.colstride;
  stage_tiles<T, CB>(su, g, a.u + off, a.colstride, nc, a.mask, x0, y0, z0, tz);
  __syncthreads();
  if ((int)threadIdx.x >= TX * TY * tz) return;   // a batched launch sizes its blocks for the tallest tile
  const int lz = threadIdx.x % tz, rr = threadIdx.x / tz, ly = rr % TY, lx = rr / TY;
  const int i = x0 + lx, j = y0 + ly, k = z0 + lz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  const long long n = ((long long)i * g.ny + j) * g.nz + k;
  const long long nst = g.nnode;
  const T* sp = a.E + n;
  // the columns' epilogue inputs are fetched before the stencil arithmetic (their latency overlaps it)
  const unsigned m = a.mask ? a.mask[n] : 7u;
  EpiPre<T> ep[CB];
#pragma unroll
  for (int c = 0; c < CB; ++c)
    if (c < nc && (!a.active || a.active[c0 + c])) epilogue_load(a, mode, off + c * a.colstride, n, ep[c]);
  T out[CB][3];
#pragma unroll
  for (int c = 0; c < CB; ++c) { out[c][0] = T(0); out[c][1] = T(0); out[c][2] = T(0); }
  const int cbase = 3 * (((lx + 1) * HY + (ly + 1)) * HZ + (lz + 1));
#pragma unroll
  for (int di = -1; di <= 1; ++di) {
#pragma unroll
    for (int dj = -1; dj <= 1; ++dj) {
#pragma unroll
      for (int dk = -1; dk <= 1; ++dk) {
        const int d = ((di + 1) * 3 + (dj + 1)) * 3 + (dk + 1);
        const int noff = cbase + 3 * ((di * HY + dj) * HZ + dk);
        T sv[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) sv[q] = sp[(long long)(d * 9 + q) * nst];
#pragma unroll
        for (int c = 0; c < CB; ++c) {
          const T* p = su + c * HALO * 3 + noff;
          const T u0 = p[0], u1 = p[1], u2 = p[2];
#pragma unroll
          for (int q = 0; q < 3; ++q) out[c][q] = fma(sv[3 * q + 2], u2, fma(sv[3 * q + 1], u1, fma(sv[3 * q], u0, out[c][q])));
        }
      }
    }
  }
#pragma unroll
  for (int c = 0; c < CB; ++c) {
    if (c < nc && (!a.active || a.active[c0 + c])) epilogue_pre<T, RND>(a, mode, off + c * a.colstride, n, m, out[c], ep[c]);
  }
}
template <typename T, int CB, int RND>
__global__ void __launch_bounds__(TX * TY * TZMAX) stencil_level_kernel(const __grid_constant__ LevelArgs<T> a, int mode, TileMap tm) {
  stencil_level_body<T, CB, RND>(vgrid(), a, mode, tm);
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
__device__ __forceinline__ void restrict_body(const VGrid vg_,Geo fine, Geo coarse, const T* __restrict__ r, long long fstride, T* __restrict__ out,
                                long long cstride, const uint8_t* __restrict__ cmask, const int* __restrict__ active, int round) {
  TF_VGRID(vg_);
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
    oc[3 * n + 0] = (m & 1u) ? round_store(acc0, round) : T(0);
    oc[3 * n + 1] = (m & 2u) ? round_store(acc1, round) : T(0);
    oc[3 * n + 2] = (m & 4u) ? round_store(acc2, round) : T(0);
  }
}
template <typename T>
__global__ void restrict_kernel(Geo fine, Geo coarse, const T* __restrict__ r, long long fstride, T* __restrict__ out,
                                long long cstride, const uint8_t* __restrict__ cmask, const int* __restrict__ active, int round) {
  restrict_body<T>(vgrid(), fine, coarse, r, fstride, out, cstride, cmask, active, round);
}

// x_fine += mask * P c  (P = transpose of the restriction).  One thread per coarse node I (and
// column) loads the 8 coarse values of the cell I..I+1 once and updates the up to 8 fine nodes
// 2I..2I+1 that take their correction from that cell (each fine node belongs to exactly one cell);
// every fine node sums its coarse contributions in the same order as a per-fine-node loop would.
template <typename T>
__device__ __forceinline__ void prolong_add_body(const VGrid vg_,Geo fine, Geo coarse, const T* __restrict__ c, long long cstride, T* __restrict__ x,
                                   long long fstride, const uint8_t* __restrict__ fmask, const int* __restrict__ active, int round) {
  TF_VGRID(vg_);
  const int col = blockIdx.y;
  if (active && !active[col]) return;
  const T* cc = c + col * cstride;
  T* xc = x + col * fstride;
  for (long long cn = (long long)blockIdx.x * blockDim.x + threadIdx.x; cn < coarse.nnode; cn += (long long)gridDim.x * blockDim.x) {
    int I, J, K;
    node_coords(cn, coarse, I, J, K);
    const bool hx = I + 1 < coarse.nx, hy = J + 1 < coarse.ny, hz = K + 1 < coarse.nz;
    T cv[8][3];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          T* v = cv[(a * 2 + b) * 2 + q];
          v[0] = v[1] = v[2] = T(0);
          if ((!a || hx) && (!b || hy) && (!q || hz)) {
            const T* p = cc + 3 * (((long long)(I + a) * coarse.ny + (J + b)) * coarse.nz + (K + q));
            v[0] = p[0]; v[1] = p[1]; v[2] = p[2];
          }
        }
#pragma unroll
    for (int fi = 0; fi < 2; ++fi) {
      const int i = 2 * I + fi;
      if (i >= fine.nx) continue;
#pragma unroll
      for (int fj = 0; fj < 2; ++fj) {
        const int j = 2 * J + fj;
        if (j >= fine.ny) continue;
#pragma unroll
        for (int fk = 0; fk < 2; ++fk) {
          const int k = 2 * K + fk;
          if (k >= fine.nz) continue;
          // an even fine index takes coarse node I with weight 1, an odd one I (1/2) and I + 1 (1/2, when it exists)
          T acc0 = T(0), acc1 = T(0), acc2 = T(0);
#pragma unroll
          for (int a = 0; a < 2; ++a) {
            if (a && (!fi || !hx)) continue;
            const T wa = fi ? T(0.5) : T(1);
#pragma unroll
            for (int b = 0; b < 2; ++b) {
              if (b && (!fj || !hy)) continue;
              const T wb = fj ? T(0.5) : T(1);
#pragma unroll
              for (int q = 0; q < 2; ++q) {
                if (q && (!fk || !hz)) continue;
                const T wq = fk ? T(0.5) : T(1);
                const T w = wa * wb * wq;
                const T* v = cv[(a * 2 + b) * 2 + q];
                acc0 += w * v[0]; acc1 += w * v[1]; acc2 += w * v[2];
              }
            }
          }
          const long long n = ((long long)i * fine.ny + j) * fine.nz + k;
          const unsigned m = fmask ? fmask[n] : 7u;
          if (m & 1u) xc[3 * n + 0] = round_store(xc[3 * n + 0] + acc0, round);
          if (m & 2u) xc[3 * n + 1] = round_store(xc[3 * n + 1] + acc1, round);
          if (m & 4u) xc[3 * n + 2] = round_store(xc[3 * n + 2] + acc2, round);
        }
      }
    }
  }
}
template <typename T>
__global__ void prolong_add_kernel(Geo fine, Geo coarse, const T* __restrict__ c, long long cstride, T* __restrict__ x,
                                   long long fstride, const uint8_t* __restrict__ fmask, const int* __restrict__ active, int round) {
  prolong_add_body<T>(vgrid(), fine, coarse, c, cstride, x, fstride, fmask, active, round);
}

}  // namespace tfb
