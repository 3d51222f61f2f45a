// Finest-level operator on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// Element form of y = mask * sum_e E_e K0 (mask * u)_e: for every element e of a CTA's tile and one
// column, the row W[e] = E_e * u_e (the element's 24 nodal values, dof order 3 * corner + comp) is
// written to shared memory in the UMMA K-major layout; one thread issues tcgen05.mma kind::tf32
// (M = 128 element rows per instruction, N = 32 = 8 corners x 4, K = 24 in three K = 8 steps) with
// B = K0 (rows 4 * corner + comp, the fourth row of every corner zero) resident in shared memory and
// the FP32 accumulators in TMEM.  tcgen05.ld brings each element's 24 results back to registers; they
// go to a shared corner-major buffer, from which every output node sums its 8 element contributions
// in a fixed corner order (no atomics, bitwise reproducible), and the smoother epilogue of the
// CUDA-core kernel finishes the node.  Operands are rounded to TF32 (10-bit mantissa) by the tensor
// cores and accumulated in FP32, so the apply is accurate to ~1e-3 relative: it serves the V-cycle
// of the FP64-outer PCG, never the FP64 operator.
//
// A CTA covers 8 x 8 x tz output nodes (tz = 8 or 9), i.e. 9 x 9 x (tz + 1) elements and a halo of
// 10 x 10 x (tz + 2) input nodes, and loops over its columns; every wait on the MMA completion
// barrier is bounded and sets *err (the launch then releases its TMEM and returns).
#pragma once
#include "tf_kernels.cuh"

namespace tfb {
namespace tc {

constexpr int NXT = 8, NYT = 8, NZT_MAX = 9;                 // output nodes per tile
constexpr int EXT = NXT + 1, EYT = NYT + 1, EZT_MAX = NZT_MAX + 1;
constexpr int HXT = NXT + 2, HYT = NYT + 2, HZT = NZT_MAX + 2;  // input halo (fixed pitch)
constexpr int NE_MAX = EXT * EYT * EZT_MAX;                  // 810 element rows
constexpr int MMA_M = 128, MMA_N = 32, MMA_K = 24;
constexpr int MMAS_MAX = (NE_MAX + MMA_M - 1) / MMA_M;       // 7
constexpr int ROWS_MAX = MMAS_MAX * MMA_M;                   // 896
constexpr int THREADS = 256;
constexpr int TMEM_COLS = 256;                               // >= MMAS_MAX * MMA_N, power of two
constexpr unsigned SPIN_LIMIT = 1u << 22;                    // bounded barrier wait (tens of ms)

// shared-memory carve-up (bytes)
constexpr size_t W_BYTES = size_t(MMA_K / 4) * ROWS_MAX * 16;           // 6 K-chunks x rows x 16 B
constexpr size_t D_BYTES = size_t(8) * NE_MAX * 3 * sizeof(float);      // [corner][element][3]
constexpr size_t round128(size_t v) { return (v + 127) / 128 * 128; }
constexpr size_t WD_BYTES = round128(W_BYTES > D_BYTES ? W_BYTES : D_BYTES);
constexpr size_t U_BYTES = round128(size_t(HXT) * HYT * HZT * 3 * sizeof(float));   // three component planes
constexpr size_t E_BYTES = round128(size_t(NE_MAX) * sizeof(float));
constexpr size_t B_BYTES = size_t(MMA_K / 4) * MMA_N * 16;
constexpr size_t SMEM_BYTES = WD_BYTES + U_BYTES + E_BYTES + B_BYTES + 64;
static_assert(WD_BYTES % 128 == 0 && U_BYTES % 128 == 0 && E_BYTES % 128 == 0, "UMMA operands need aligned regions");
static_assert(SMEM_BYTES <= 113 * 1024, "two CTAs per SM (TMEM_COLS each) must fit in shared memory");
static_assert(2 * TMEM_COLS <= 512 && MMAS_MAX * MMA_N <= TMEM_COLS, "TMEM columns");

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// UMMA shared-memory descriptor, K-major without swizzle: 8-row core matrices of 16 B rows stored
// contiguously (stride between 8-row groups sbo), K-chunks of 16 B lbo apart.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = static_cast<uint64_t>((addr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
  d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
  d |= static_cast<uint64_t>(1) << 46;   // descriptor version of sm_100
  return d;
}

// Instruction descriptor: D FP32, A and B TF32, both K-major, N = 32, M = 128.
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(MMA_N >> 3) << 17) | (uint32_t(MMA_M >> 4) << 24);

__device__ __forceinline__ bool bar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
               : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool bar_wait_bounded(uint32_t bar, uint32_t parity) {
  for (unsigned it = 0; it < SPIN_LIMIT; ++it)
    if (bar_try_wait(bar, parity)) return true;
  return false;
}

// 16 consecutive FP32 accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_load16(uint32_t addr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
                 "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
               : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

struct TcTiles {
  int tiles_x, tiles_y, tiles_z, tz;
};

constexpr int HALO_PER_THREAD = (HXT * HYT * HZT + THREADS - 1) / THREADS;   // 5
constexpr int NODES_PER_THREAD = (NXT * NYT * NZT_MAX + THREADS - 1) / THREADS;   // 3
constexpr int PLANE = HXT * HYT * HZT;                                         // one component of the halo

// Inputs of the smoother epilogue (ApplyMode) a node needs besides A u, loaded while the MMAs run.
template <int MODE> struct EpiIn { float v[1][3]; };
template <> struct EpiIn<MODE_RESID> { float v[1][3]; };    // b
template <> struct EpiIn<MODE_JACOBI> { float v[3][3]; };   // u, inv, b
template <> struct EpiIn<MODE_CHEB> { float v[4][3]; };     // res, u, inv, x

template <int MODE>
__device__ __forceinline__ void epi_load(const LevelArgs<float>& a, long long d0, long long node, EpiIn<MODE>& in) {
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    if (MODE == MODE_RESID) {
      in.v[0][q] = a.b[d0 + q];
    } else if (MODE == MODE_JACOBI) {
      in.v[0][q] = a.u[d0 + q]; in.v[1][q] = a.inv[3 * node + q]; in.v[2][q] = a.b[d0 + q];
    } else if (MODE == MODE_CHEB) {
      in.v[0][q] = a.res[d0 + q]; in.v[1][q] = a.u[d0 + q]; in.v[2][q] = a.inv[3 * node + q]; in.v[3][q] = a.x[d0 + q];
    }
  }
}

// Same arithmetic as epilogue() of the CUDA-core kernels, from prefetched inputs.
template <int MODE>
__device__ __forceinline__ void epi_store(const LevelArgs<float>& a, long long d0, unsigned m, const float av[3], const EpiIn<MODE>& in) {
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const bool live = (m >> q) & 1u;
    const long long d = d0 + q;
    if (MODE == MODE_APPLY) {
      a.y[d] = live ? av[q] : 0.0f;
    } else if (MODE == MODE_RESID) {
      a.y[d] = live ? (in.v[0][q] - av[q]) : 0.0f;
    } else if (MODE == MODE_JACOBI) {
      a.y[d] = in.v[0][q] + a.s * in.v[1][q] * (in.v[2][q] - (live ? av[q] : 0.0f));
    } else {
      const float r = in.v[0][q] - (live ? av[q] : 0.0f);
      const float dn = a.c1 * in.v[1][q] + a.c2 * in.v[2][q] * r;
      a.res[d] = r;
      a.y[d] = dn;
      a.x[d] = in.v[3][q] + dn;
    }
  }
}

template <int MODE>
__global__ void __launch_bounds__(THREADS, 2) fine_tc_kernel(const __grid_constant__ K0Param<float> K, const LevelArgs<float> a,
                                                             TcTiles tm, int cpb, int* err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float* sWD = reinterpret_cast<float*>(smem_raw);                                // W, then D
  float* su = reinterpret_cast<float*>(smem_raw + WD_BYTES);                     // [3][HXT][HYT][HZT] planar
  float* sE = reinterpret_cast<float*>(smem_raw + WD_BYTES + U_BYTES);           // [EXT][EYT][ez_n]
  float* sB = reinterpret_cast<float*>(smem_raw + WD_BYTES + U_BYTES + E_BYTES); // K0 in UMMA layout
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + WD_BYTES + U_BYTES + E_BYTES + B_BYTES);
  uint32_t* tbase = reinterpret_cast<uint32_t*>(bar + 1);
  int* abort_flag = reinterpret_cast<int*>(bar + 2);
  if (a.gate && !*a.gate) return;
  const Geo& g = a.g;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int b = blockIdx.x;
  const int bz = b % tm.tiles_z, r0 = b / tm.tiles_z, by = r0 % tm.tiles_y, bx = r0 / tm.tiles_y;
  const int tz = tm.tz, ez_n = tz + 1, hz_n = tz + 2;
  const int x0 = bx * NXT, y0 = by * NYT, z0 = bz * tz;
  const int ne = EXT * EYT * ez_n;
  const int nmma = (ne + MMA_M - 1) / MMA_M;
  const int nhalo = HXT * HYT * hz_n, nout = NXT * NYT * tz;
  const int c_begin = blockIdx.y * cpb, c_end = min(a.ncol, c_begin + cpb);

  // K0 as the B operand: row n = 4 corner + comp (comp 3 zero), K-chunk kc at kc * (32 rows * 16 B)
  for (int idx = t; idx < MMA_N * MMA_K; idx += THREADS) {
    const int n = idx / MMA_K, k = idx % MMA_K, corner = n >> 2, comp = n & 3;
    sB[(k >> 2) * (MMA_N * 4) + n * 4 + (k & 3)] = comp < 3 ? K.k[(3 * corner + comp) * 24 + k] : 0.0f;
  }
  // element moduli of the tile (zero outside the grid)
  for (int idx = t; idx < ne; idx += THREADS) {
    const int ez = idx % ez_n, rr = idx / ez_n, ey = rr % EYT, ex = rr / EYT;
    const int gx = x0 - 1 + ex, gy = y0 - 1 + ey, gz = z0 - 1 + ez;
    float e = 0.0f;
    if ((unsigned)gx < (unsigned)g.ex && (unsigned)gy < (unsigned)g.ey && (unsigned)gz < (unsigned)g.ez)
      e = a.E[((long long)gx * g.ey + gy) * g.ez + gz];
    sE[idx] = e;
  }
  // this thread's halo nodes (fixed for the launch) and output nodes
  int hnode[HALO_PER_THREAD];        // node indices fit in 32 bits (checked by the launcher)
  int hslot[HALO_PER_THREAD];
#pragma unroll
  for (int h = 0; h < HALO_PER_THREAD; ++h) {
    const int idx = t + h * THREADS;
    hnode[h] = -1;
    hslot[h] = -1;
    if (idx < nhalo) {
      const int hz = idx % hz_n, rr = idx / hz_n, hy = rr % HYT, hx = rr / HYT;
      const int gx = x0 - 1 + hx, gy = y0 - 1 + hy, gz = z0 - 1 + hz;
      hslot[h] = (hx * HYT + hy) * HZT + hz;
      if ((unsigned)gx < (unsigned)g.nx && (unsigned)gy < (unsigned)g.ny && (unsigned)gz < (unsigned)g.nz)
        hnode[h] = (gx * g.ny + gy) * g.nz + gz;
    }
  }
  unsigned hmask[HALO_PER_THREAD];
#pragma unroll
  for (int h = 0; h < HALO_PER_THREAD; ++h) hmask[h] = (hnode[h] >= 0) ? (a.mask ? a.mask[hnode[h]] : 7u) : 0u;
  int onode[NODES_PER_THREAD];
  int oe[NODES_PER_THREAD];
  unsigned omask[NODES_PER_THREAD];
#pragma unroll
  for (int o = 0; o < NODES_PER_THREAD; ++o) {
    const int idx = t + o * THREADS;
    onode[o] = -1;
    oe[o] = 0;
    omask[o] = 0;
    if (idx < nout) {
      const int lz = idx % tz, rr = idx / tz, ly = rr % NYT, lx = rr / NYT;
      const int i = x0 + lx, j = y0 + ly, k = z0 + lz;
      oe[o] = ((lx + 1) * EYT + (ly + 1)) * ez_n + (lz + 1);   // element whose corner 0 is this node
      if (i < g.nx && j < g.ny && k < g.nz) {
        onode[o] = (i * g.ny + j) * g.nz + k;
        omask[o] = a.mask ? a.mask[onode[o]] : 7u;
      }
    }
  }
  // element offset (in element index units) from a node's corner-0 element to its corner-cn element
  int eoff[8];
#pragma unroll
  for (int cn = 0; cn < 8; ++cn) eoff[cn] = -((corner_x(cn) * EYT + corner_y(cn)) * ez_n + corner_z(cn));

  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_addr(bar)));
    *abort_flag = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(smem_addr(tbase)), "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tbase;
  const uint32_t bar_a = smem_addr(bar);
  uint32_t phase = 0;

  auto next_active = [&](int c) {
    while (c < c_end && a.active && !a.active[c]) ++c;
    return c;
  };
  // halo values of the next column, held in registers while the current one is computed
  float hv[HALO_PER_THREAD][3];
  auto fetch = [&](int c) {
#pragma unroll
    for (int h = 0; h < HALO_PER_THREAD; ++h) {
      hv[h][0] = hv[h][1] = hv[h][2] = 0.0f;
      if (c < c_end && hnode[h] >= 0) {
        const float* p = a.u + (long long)c * a.colstride + 3 * (long long)hnode[h];
        hv[h][0] = p[0]; hv[h][1] = p[1]; hv[h][2] = p[2];
      }
    }
  };
  int c = next_active(c_begin);
  fetch(c);
  while (c < c_end) {
    const long long col_off = (long long)c * a.colstride;
    // 1. masked input halo of this column, component-planar
#pragma unroll
    for (int h = 0; h < HALO_PER_THREAD; ++h) {
      if (hslot[h] < 0) continue;
      su[hslot[h]] = (hmask[h] & 1u) ? hv[h][0] : 0.0f;
      su[PLANE + hslot[h]] = (hmask[h] & 2u) ? hv[h][1] : 0.0f;
      su[2 * PLANE + hslot[h]] = (hmask[h] & 4u) ? hv[h][2] : 0.0f;
    }
    __syncthreads();
    // 2. element rows W[e] = E_e * u_e in the UMMA K-major layout (chunk kc of row r at kc * ROWS_MAX * 16 B + r * 16 B)
    for (int row = t; row < nmma * MMA_M; row += THREADS) {
      const bool live_row = row < ne;
      const int ez = row % ez_n, rr = row / ez_n, ey = rr % EYT, ex = rr / EYT;
      const float e = live_row ? sE[row] : 0.0f;
      const int base = live_row ? (ex * HYT + ey) * HZT + ez : 0;
#pragma unroll
      for (int kc = 0; kc < 6; ++kc) {
        float w4[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int k = 4 * kc + j, cn = k / 3, comp = k % 3;
          w4[j] = e * su[comp * PLANE + base + (corner_x(cn) * HYT + corner_y(cn)) * HZT + corner_z(cn)];
        }
        *reinterpret_cast<float4*>(sWD + (kc * ROWS_MAX + row) * 4) = make_float4(w4[0], w4[1], w4[2], w4[3]);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    // 3. one thread issues the MMAs of all row blocks and commits them to the barrier
    if (t == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t wa = smem_addr(sWD), ba = smem_addr(sB);
      for (int m = 0; m < nmma; ++m) {
#pragma unroll
        for (int ks = 0; ks < 3; ++ks) {
          const uint64_t da = smem_desc(wa + (2 * ks * ROWS_MAX + m * MMA_M) * 16, ROWS_MAX * 16, 128);
          const uint64_t db = smem_desc(ba + 2 * ks * MMA_N * 16, MMA_N * 16, 128);
          const uint32_t acc = ks > 0 ? 1u : 0u;
          asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                       "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                       :: "r"(tmem + m * MMA_N), "l"(da), "l"(db), "r"(IDESC), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(bar_a) : "memory");
    }
    // while the MMAs run: the epilogue inputs of this column and the halo of the next one
    EpiIn<MODE> in[NODES_PER_THREAD];
#pragma unroll
    for (int o = 0; o < NODES_PER_THREAD; ++o)
      if (onode[o] >= 0) epi_load<MODE>(a, col_off + 3 * (long long)onode[o], onode[o], in[o]);
    const int c_next = next_active(c + 1);
    fetch(c_next);
    // 4. bounded wait for the MMAs; a timeout anywhere ends the launch for every thread
    const bool ok = bar_wait_bounded(bar_a, phase);
    if (!ok) *abort_flag = 1;
    phase ^= 1u;
    __syncthreads();
    if (*abort_flag) break;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // 5. accumulators -> corner-major buffer D[corner][element][comp] (overwrites W, which the MMAs have read)
    {
      const int quad = warp & 3;
      for (int m = warp >> 2; m < nmma; m += THREADS / 128) {
        const int row = m * MMA_M + 32 * quad + lane;
#pragma unroll
        for (int half = 0; half < 2; ++half) {     // corners 0-3, then 4-7
          float v[16];
          tmem_load16(tmem + (uint32_t(32 * quad) << 16) + m * MMA_N + 16 * half, v);
          if (row < ne) {
#pragma unroll
            for (int cq = 0; cq < 4; ++cq) {
              float* d = sWD + ((4 * half + cq) * NE_MAX + row) * 3;
              d[0] = v[4 * cq]; d[1] = v[4 * cq + 1]; d[2] = v[4 * cq + 2];
            }
          }
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    // 6. every node sums its 8 element contributions (fixed corner order) and runs the epilogue
#pragma unroll
    for (int o = 0; o < NODES_PER_THREAD; ++o) {
      if (onode[o] < 0) continue;
      float av[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
      for (int cn = 0; cn < 8; ++cn) {
        const float* d = sWD + (cn * NE_MAX + oe[o] + eoff[cn]) * 3;
        av[0] += d[0]; av[1] += d[1]; av[2] += d[2];
      }
      epi_store<MODE>(a, col_off + 3 * (long long)onode[o], omask[o], av, in[o]);
    }
    __syncthreads();
    c = c_next;
  }
  if (*abort_flag) {
    if (t == 0) atomicExch(err, 1);
    // let any MMA still in flight finish before its TMEM is released (bounded)
    bar_wait_bounded(bar_a, phase ^ 1u);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(TMEM_COLS));
}

}  // namespace tc
}  // namespace tfb
