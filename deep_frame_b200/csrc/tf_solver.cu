// Matrix-free hex8 GMG-PCG solver behind the C ABI of include/tf_b200.h.
//
// Mirrors deep_frame/topology_multigrid.py (GeometricMultigrid) of the
// reference: level count and padding (:58-63), finest-level mask (:138-144),
// Jacobi diagonal (:118-124), Galerkin blocks (:145-208), lambda_max power
// iteration (:214-223), Jacobi / Chebyshev smoothing (:284-305), V/W cycle
// (:306-317), residual scaling of the preconditioner (:318-324), batched
// flexible PCG with the true-residual recheck (:407-454) and FP64 retries of
// failed columns (:385-406).  Differences by design: every RHS column runs in
// the same launches (per-column scalars live on the device, converged columns
// are masked out instead of compacted), and the coarsest level is a dense FP64
// factor (tf_dense.cu) instead of cuDSS.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <type_traits>
#include <cmath>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "tf_b200.h"
#include "tf_common.h"
#include "tf_dense.h"
#include "tf_setup.cuh"
#include "tf_tc.cuh"
#include "tf_batch.cuh"

using namespace tfb;

namespace {

thread_local std::string g_last_create_error;

constexpr int CB32 = 6;                  // columns per CTA of the FP32 Galerkin-level operator
constexpr int CB64 = 2;                  // columns per CTA of the FP64 Galerkin-level operator
constexpr long long DENSE_LIMIT = 24000;  // largest dense coarsest factor (4.6 GB in FP64); banded above
constexpr double BAND_LIMIT_BYTES = 32e9;  // largest banded coarsest factor

struct Level {
  Geo g{};
  long long ndof = 0, nelem = 0;
  DevBuf mask;      // uint8 [nnode]
  DevBuf blocks64;  // Galerkin blocks [nelem][576] (levels >= 1), used by the set-up
  DevBuf stencil64; // assembled 27-point stencil, entry-major FP64 [243][nnode], for the operator
  DevBuf stencilw;  // FP32 copy (FP32 work precision only)
  DevBuf inv64;     // inverse diagonal [ndof]
  DevBuf invw;      // FP32 copy (FP32 work precision only)
  double lambda_max = 1.0;
};

struct Hierarchy {
  std::vector<Level> lv;
  int n_live = 0;
  DevBuf live;      // int64 [n_live]: live dofs of the coarsest level
  DevBuf X;         // FP64 [n_live][n_live] inverse Cholesky factor, or the banded factor (band)
  DevBuf A, live_of, bits;  // set-up scratch kept for the next rebuild
  bool band = false;        // coarsest factor banded (n_live above the dense limit)
  int bw = 0;               // its bandwidth in the live-dof numbering
  double setup_s = 0.0;
  bool setup_reported = false;
  bool valid = false;
};

template <typename T>
struct VBufs {
  std::vector<DevBuf> b, x, xa, res, d, da;
  int cap = 0;
};

Geo make_geo(long long ex, long long ey, long long ez) {
  Geo g;
  g.ex = static_cast<int>(ex);
  g.ey = static_cast<int>(ey);
  g.ez = static_cast<int>(ez);
  g.nx = g.ex + 1;
  g.ny = g.ey + 1;
  g.nz = g.ez + 1;
  g.nnode = (long long)g.nx * g.ny * g.nz;
  return g;
}

// Column-batched elementwise launches: blockIdx.y = column, grid-stride loops along x.  The CTAs along
// x are capped so that all columns together make about 32 CTAs per SM: with many columns, fewer and
// longer-running CTAs stream the vectors faster than one short CTA per few hundred elements (measured:
// 16 or up to 1184 per column were slower).
inline dim3 cols_grid(long long n, int ncol, int block = 256, int cap = 1184) {
  const int per_col = std::max(1, std::min(cap, (148 * 32 + std::max(ncol, 1) - 1) / std::max(ncol, 1)));
  return dim3(grid_for(n, block, per_col), ncol);
}

// Optional CUDA-event timing of kernel classes on the launching stream.
enum TimerClass : int {
  TIMER_FINE64 = 0,    // FP64 finest-level operator of the PCG (apply and true residual)
  TIMER_FINE_WORK = 1, // finest-level smoother / residual in the work precision
  TIMER_COARSE = 2,    // Galerkin-level operators
  TIMER_TRANSFER = 3,  // restriction and prolongation
  TIMER_VECTOR = 4,    // PCG reductions and vector updates
  TIMER_COARSEST = 5,  // dense coarsest solve
  TIMER_SETUP = 6,     // hierarchy build (masks, Galerkin blocks, lambda_max, factor)
  TIMER_ENERGY = 7,    // element energies
  TIMER_PCG32 = 8,     // FP32 finest-level operator of the mixed PCG's iterations
  TIMER_CLASSES = 9
};

struct Timers {
  bool enabled = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pool;
  std::vector<int> cls;
  size_t used = 0;
  ~Timers() {
    for (auto& e : pool) {
      cudaEventDestroy(e.first);
      cudaEventDestroy(e.second);
    }
  }
  std::pair<cudaEvent_t, cudaEvent_t>* next(int c) {
    if (used == pool.size()) {
      cudaEvent_t a, b;
      TF_CUDA_CHECK(cudaEventCreate(&a));
      TF_CUDA_CHECK(cudaEventCreate(&b));
      pool.push_back({a, b});
      cls.push_back(c);
    }
    cls[used] = c;
    return &pool[used++];
  }
};

struct TimedRange {
  Timers* t;
  cudaStream_t s;
  std::pair<cudaEvent_t, cudaEvent_t>* ev = nullptr;
  TimedRange(Timers& timers, int c, cudaStream_t stream) : t(&timers), s(stream) {
    if (t->enabled) {
      ev = t->next(c);
      cudaEventRecord(ev->first, s);
    }
  }
  ~TimedRange() {
    if (ev) cudaEventRecord(ev->second, s);
  }
};

}  // namespace

struct tf_handle {
  tf_settings s{};
  long long shape[3]{}, padded[3]{};
  double spacing[3]{};
  int nlev = 0;
  std::vector<Geo> geo;
  Geo un{};
  double ke[576]{};
  K0Param<double> k64{};
  K0Param<float> k32{};
  K0Param<double> m64{};   // consistent element mass M0 (tf_create's me), for tf_mass_apply
  bool have_me = false;
  DevBuf mass64, lumped64;  // padded element masses and lumped nodal masses of the last tf_mass_apply
  DevBuf tc_err;            // int: set by the tensor-core finest-level kernel when an MMA wait timed out
  DevBuf trimul_work;       // split-K partials of the coarsest triangular products
  DevBuf factor_work;       // inverted diagonal blocks of the coarsest factorisation
  DevBuf solve_small;       // per-solve column norms and column lists (grows, never shrinks)
  GalerkinParam W{};
  DevBuf Q, K0dev, k0diag;
  DevBuf moduli_un, moduli64, modulif;
  bool have_moduli = false;
  std::map<uint64_t, std::vector<int64_t>> bcs;
  std::map<uint64_t, Hierarchy> hier;
  // reduction scratch; dotp holds the FP64 operator's per-warp curvature partials
  DevBuf partial, count, scal, dotp;
  // PCG state
  DevBuf pcg_d, pcg_i, hist, colmap;
  int pcg_cap = 0, hist_cap = 0;
  int* host_flags = nullptr;
  // FP64 PCG vectors [cap][ndof0]
  DevBuf vb, vx, vr, vz, vp, vq;
  int vcap = 0;
  DevBuf cb, cy;  // coarsest work [cap][n_live]
  size_t ccap = 0;
  VBufs<float> wf;
  VBufs<double> wd;
  DevBuf tmp_diag;
  bool k0_reflect = false;   // ke has the 8-fold reflection symmetry (72 distinct coefficients)
  int k0_slot = -1;   // constant-memory slot of ke, its device and the slot version it saw
  int k0_device = -1;
  unsigned long long k0_version = 0;
  Timers timers;
  std::string err;
  // the coarsest factorisation runs on `side` while the power iterations run on the caller's stream
  cudaStream_t side = nullptr;
  cudaEvent_t side_fork = nullptr, side_join = nullptr;
  ~tf_handle() {
    if (host_flags) cudaFreeHost(host_flags);
    if (side_fork) cudaEventDestroy(side_fork);
    if (side_join) cudaEventDestroy(side_join);
    if (side) cudaStreamDestroy(side);
  }
};

namespace {

bool work_is_double(const tf_handle* h) { return h->s.precision == TF_PRECISION_FLOAT64; }
// Storage rounding of the V-cycle vectors (round_store): 16-bit storage precisions keep FP32 buffers
// and arithmetic and round every stored value to the 16-bit format.
int store_round(const tf_handle* h) {
  return h->s.precision == TF_PRECISION_BFLOAT16 ? 1 : (h->s.precision == TF_PRECISION_FLOAT16 ? 2 : 0);
}

// ------------------------------------------------------------ buffers -------

void ensure_scratch(tf_handle* h, int ncol) {
  const size_t need = (size_t)std::max(ncol, 1) * PCG_BLOCKS * 4 * sizeof(double);
  if (h->partial.bytes < need) {
    h->partial.alloc(need);
    h->count.alloc(sizeof(unsigned) * std::max(ncol, 1));
    TF_CUDA_CHECK(cudaMemset(h->count.p, 0, h->count.bytes));
  }
  if (!h->scal.p) h->scal.alloc(64 * sizeof(double));
}

template <typename T>
VBufs<T>& vbufs(tf_handle* h);
template <>
VBufs<float>& vbufs<float>(tf_handle* h) { return h->wf; }
template <>
VBufs<double>& vbufs<double>(tf_handle* h) { return h->wd; }

template <typename T>
void ensure_vbufs(tf_handle* h, int ncol) {
  VBufs<T>& v = vbufs<T>(h);
  if (v.cap >= ncol && (int)v.b.size() == h->nlev) return;
  const int cap = std::max(ncol, 1);
  v.b.clear(); v.x.clear(); v.xa.clear(); v.res.clear(); v.d.clear(); v.da.clear();
  for (int l = 0; l < h->nlev; ++l) {
    const size_t bytes = sizeof(T) * 3 * (size_t)h->geo[l].nnode * cap;
    for (auto* vec : {&v.b, &v.x, &v.xa, &v.res, &v.d, &v.da}) {
      vec->emplace_back(bytes);
      TF_CUDA_CHECK(cudaMemset(vec->back().p, 0, bytes));
    }
  }
  v.cap = cap;
}

void ensure_pcg(tf_handle* h, int ncol) {
  ensure_scratch(h, ncol);
  if (h->pcg_cap < ncol) {
    h->pcg_d.alloc(sizeof(double) * 9 * ncol);
    h->pcg_i.alloc(sizeof(int) * (4 * ncol + 8));
    h->colmap.alloc(sizeof(int) * ncol);
    TF_CUDA_CHECK(cudaMemset(h->pcg_d.p, 0, h->pcg_d.bytes));
    TF_CUDA_CHECK(cudaMemset(h->pcg_i.p, 0, h->pcg_i.bytes));
    h->pcg_cap = ncol;
  }
  const int hneed = h->s.max_iterations + 2;
  if (h->hist_cap < hneed) {
    h->hist.alloc(sizeof(unsigned long long) * hneed);
    h->hist_cap = hneed;
  }
  if (!h->host_flags) TF_CUDA_CHECK(cudaMallocHost(&h->host_flags, 64 * sizeof(int)));
  if (h->vcap < ncol) {
    const size_t bytes = sizeof(double) * 3 * (size_t)h->geo[0].nnode * ncol;
    for (DevBuf* b : {&h->vb, &h->vx, &h->vr, &h->vz, &h->vp, &h->vq}) {
      b->alloc(bytes);
      TF_CUDA_CHECK(cudaMemset(b->p, 0, bytes));
    }
    h->vcap = ncol;
  }
}

PcgState pcg_state(tf_handle* h, int ncol) {
  PcgState st;
  double* d = h->pcg_d.as<double>();
  const int c = h->pcg_cap;
  st.bnorm = d + 0 * c;
  st.rho = d + 1 * c;
  st.alpha = d + 2 * c;
  st.rel = d + 3 * c;
  st.scale = d + 4 * c;
  st.rzo = d + 5 * c;
  st.beta = d + 6 * c;
  st.wscale = d + 7 * c;
  st.rtrue = d + 8 * c;
  int* i = h->pcg_i.as<int>();
  st.active = i + 0 * c;
  st.cand = i + 1 * c;
  st.iters = i + 2 * c;
  st.flags = i + 4 * c;
  st.hist = h->hist.as<unsigned long long>();
  st.partial = h->partial.as<double>();
  st.count = h->count.as<unsigned>();
  st.ncol = ncol;
  return st;
}

// --------------------------------------------------------- level apply ------

template <typename T>
const T* level_E(tf_handle* h, Hierarchy& hy, int l, bool precise) {
  const bool dbl = std::is_same<T, double>::value;
  if (l == 0) return static_cast<const T*>(dbl ? h->moduli64.p : h->modulif.p);
  return static_cast<const T*>(dbl ? hy.lv[l].stencil64.p : hy.lv[l].stencilw.p);
}
template <typename T>
const T* level_inv(Hierarchy& hy, int l) {
  const bool dbl = std::is_same<T, double>::value;
  return static_cast<const T*>(dbl ? hy.lv[l].inv64.p : hy.lv[l].invw.p);
}
template <typename T> const K0Param<T>& k0param(tf_handle* h);
template <> const K0Param<double>& k0param<double>(tf_handle* h) { return h->k64; }
template <> const K0Param<float>& k0param<float>(tf_handle* h) { return h->k32; }

// Constant-memory slots of the element stiffness, per device.  A handle whose
// K0 is not resident takes the least recently used slot: the device is drained
// first (no kernel in flight can still read the slot), then the FP64 and FP32
// copies are uploaded.  A per-slot version lets a handle skip the comparison
// while its slot is untouched.
constexpr int MAX_DEVICES = 64;
struct K0Slots {
  double content[K0_SLOTS][576];
  unsigned long long version[K0_SLOTS] = {};
  unsigned long long last_use[K0_SLOTS] = {};
  bool valid[K0_SLOTS] = {};
};
std::mutex g_k0_mutex;
K0Slots g_k0[MAX_DEVICES];
unsigned long long g_k0_clock = 0, g_k0_versions = 0;

int k0_slot(tf_handle* h) {
  int device = 0;
  TF_CUDA_CHECK(cudaGetDevice(&device));
  require(device >= 0 && device < MAX_DEVICES, "device ordinal out of range for the constant-memory slots");
  std::lock_guard<std::mutex> lock(g_k0_mutex);
  K0Slots& t = g_k0[device];
  if (h->k0_slot >= 0 && h->k0_device == device && t.version[h->k0_slot] == h->k0_version) {
    t.last_use[h->k0_slot] = ++g_k0_clock;
    return h->k0_slot;
  }
  int slot = -1;
  for (int s = 0; s < K0_SLOTS; ++s)
    if (t.valid[s] && std::memcmp(t.content[s], h->ke, sizeof(h->ke)) == 0) slot = s;
  if (slot < 0) {
    slot = 0;
    for (int s = 1; s < K0_SLOTS; ++s)
      if (!t.valid[s] || (t.valid[slot] && t.last_use[s] < t.last_use[slot])) slot = s;
    if (t.valid[slot]) TF_CUDA_CHECK(cudaDeviceSynchronize());
    float f[576];
    for (int q = 0; q < 576; ++q) f[q] = static_cast<float>(h->ke[q]);
    TF_CUDA_CHECK(cudaMemcpyToSymbol(c_k0d, h->ke, sizeof(h->ke), sizeof(h->ke) * slot));
    TF_CUDA_CHECK(cudaMemcpyToSymbol(c_k0f, f, sizeof(f), sizeof(f) * slot));
    double kc[72];
    float kcf[72];
    for (int a = 0; a < 3; ++a)
      for (int d = 0; d < 8; ++d)
        for (int b = 0; b < 3; ++b) {
          kc[(a * 8 + d) * 3 + b] = h->ke[a * 24 + 3 * d + b];
          kcf[(a * 8 + d) * 3 + b] = static_cast<float>(kc[(a * 8 + d) * 3 + b]);
        }
    TF_CUDA_CHECK(cudaMemcpyToSymbol(c_kcd, kc, sizeof(kc), sizeof(kc) * slot));
    TF_CUDA_CHECK(cudaMemcpyToSymbol(c_kcf, kcf, sizeof(kcf), sizeof(kcf) * slot));
    std::memcpy(t.content[slot], h->ke, sizeof(h->ke));
    t.valid[slot] = true;
    t.version[slot] = ++g_k0_versions;
  }
  t.last_use[slot] = ++g_k0_clock;
  h->k0_slot = slot;
  h->k0_device = device;
  h->k0_version = t.version[slot];
  return slot;
}

// One finest-level launch: z tiles of 8 or 9 nodes (whichever wastes fewer
// threads on this grid), two x-adjacent nodes per thread in FP32.
// Tiles of a finest-level launch and its columns per CTA: enough CTAs for a few waves on 148 SMs,
// the rest looped inside (at most 64: the kernel keeps its chunk's active columns in a 64-bit mask).
template <int TZ, int NPT>
dim3 fine_shape(const Geo& g, int ncol, TileMap& tm, int& cpb) {
  tm.tz = TZ;
  tm.tiles_x = (g.nx + FTXT * NPT - 1) / (FTXT * NPT);
  tm.tiles_y = (g.ny + TY - 1) / TY;
  tm.tiles_z = (g.nz + TZ - 1) / TZ;
  const int tiles = tm.tiles_x * tm.tiles_y * tm.tiles_z;
  cpb = 1;
  while (cpb < 64 && cpb < ncol && (long long)tiles * ((ncol + 2 * cpb - 1) / (2 * cpb)) >= 4 * 148 * 2) cpb *= 2;
  return dim3((unsigned)tiles, (unsigned)((ncol + cpb - 1) / cpb));
}

template <typename T, int SLOT, bool REFLECT, int TZ, int RND, bool PCG = false>
void launch_fine_rounded(const LevelArgs<T>& a, int mode, cudaStream_t st) {
  constexpr int NPT = (sizeof(T) == 4 && REFLECT) ? 2 : 1;
  constexpr size_t smem = fine_smem_bytes<T, TZ, NPT>();
  static bool configured = false;   // per variant and process; the attribute is per function
  if (!configured) {
    TF_CUDA_CHECK(cudaFuncSetAttribute(fine_level_kernel<T, SLOT, REFLECT, TZ, NPT, RND, PCG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    configured = true;
  }
  TileMap tm;
  int cpb;
  const dim3 grid = fine_shape<TZ, NPT>(a.g, a.ncol, tm, cpb);
  fine_level_kernel<T, SLOT, REFLECT, TZ, NPT, RND, PCG><<<grid, dim3(TZ, TY, FTXT), smem, st>>>(a, mode, tm, cpb);
  TF_LAUNCH_CHECK("fine_level_kernel");
}

// One finest-level launch: z tiles of 8 or 9 nodes (whichever wastes fewer
// threads on this grid), two x-adjacent nodes per thread in FP32.  The storage
// rounding of 16-bit precisions is a separate instantiation (FP32 only).
template <typename T, int SLOT, bool REFLECT, int TZ>
void launch_fine_variant(const LevelArgs<T>& a, int mode, cudaStream_t st) {
  if constexpr (std::is_same<T, float>::value) {
    if (a.round == 1) { launch_fine_rounded<T, SLOT, REFLECT, TZ, 1>(a, mode, st); return; }
    if (a.round == 2) { launch_fine_rounded<T, SLOT, REFLECT, TZ, 2>(a, mode, st); return; }
  } else {
    if (a.dot_out) { launch_fine_rounded<T, SLOT, REFLECT, TZ, 0, true>(a, mode, st); return; }
  }
  launch_fine_rounded<T, SLOT, REFLECT, TZ, 0>(a, mode, st);
}

// Tensor-core finest level (FP32 work precision, settings.tensor_cores): tiles of 8 x 8 x tz nodes
// (tz = 8 or 9, whichever wastes less), columns looped inside the CTA so every CTA's set-up (K0
// operand, element moduli, TMEM allocation) is spread over several columns.
void launch_fine_tc(tf_handle* h, const LevelArgs<float>& a, int mode, cudaStream_t st) {
  static bool configured = false;   // per process; the attribute is per function
  if (!configured) {
    TF_CUDA_CHECK(cudaFuncSetAttribute(tc::fine_tc_kernel<MODE_APPLY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::SMEM_BYTES));
    TF_CUDA_CHECK(cudaFuncSetAttribute(tc::fine_tc_kernel<MODE_RESID>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::SMEM_BYTES));
    TF_CUDA_CHECK(cudaFuncSetAttribute(tc::fine_tc_kernel<MODE_JACOBI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::SMEM_BYTES));
    TF_CUDA_CHECK(cudaFuncSetAttribute(tc::fine_tc_kernel<MODE_CHEB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::SMEM_BYTES));
    configured = true;
  }
  if (!h->tc_err.p) {
    h->tc_err.alloc(sizeof(int));
    TF_CUDA_CHECK(cudaMemsetAsync(h->tc_err.p, 0, sizeof(int), st));
  }
  require(a.g.nnode < (1LL << 31), "grid too large for the tensor-core finest-level apply");
  tc::TcTiles tm;
  const int nz = a.g.nz;
  tm.tz = ((nz + 8) / 9) * 9 < ((nz + 7) / 8) * 8 ? 9 : 8;
  tm.tiles_x = (a.g.nx + tc::NXT - 1) / tc::NXT;
  tm.tiles_y = (a.g.ny + tc::NYT - 1) / tc::NYT;
  tm.tiles_z = (nz + tm.tz - 1) / tm.tz;
  const long long tiles = (long long)tm.tiles_x * tm.tiles_y * tm.tiles_z;
  int cpb = 1;
  while (cpb < a.ncol && tiles * ((a.ncol + 2 * cpb - 1) / (2 * cpb)) >= 4 * 148 * 2) cpb *= 2;
  dim3 grid((unsigned)tiles, (unsigned)((a.ncol + cpb - 1) / cpb));
  int* err = h->tc_err.as<int>();
  switch (mode) {
    case MODE_APPLY: tc::fine_tc_kernel<MODE_APPLY><<<grid, tc::THREADS, tc::SMEM_BYTES, st>>>(h->k32, a, tm, cpb, err); break;
    case MODE_RESID: tc::fine_tc_kernel<MODE_RESID><<<grid, tc::THREADS, tc::SMEM_BYTES, st>>>(h->k32, a, tm, cpb, err); break;
    case MODE_JACOBI: tc::fine_tc_kernel<MODE_JACOBI><<<grid, tc::THREADS, tc::SMEM_BYTES, st>>>(h->k32, a, tm, cpb, err); break;
    default: tc::fine_tc_kernel<MODE_CHEB><<<grid, tc::THREADS, tc::SMEM_BYTES, st>>>(h->k32, a, tm, cpb, err); break;
  }
  TF_LAUNCH_CHECK("fine_tc_kernel");
}

// 8-high node tiles unless 9-high ones pad at least 15 % fewer threads along z: the 9-high
// variants spill registers at two CTAs per SM.  Measured: on the 352 x 352 x 48 plate (49 node
// planes: 56 padded with 8, 54 with 9) the 8-high FP32 apply is 17 % faster; on the 96 x 96 x 16
// plate (17 planes: 24 against 18) the 9-high one is 10 % faster.  The FP32 operator also takes
// 7-high tiles where they pad at least 10 % fewer threads than 8-high ones (352 x 352 x 48: 49
// planes exactly, 731 against 755 ms per evaluation); the FP64 operator does not (784 against
// 672 ms there: its 7-high tiles are slower despite the padding).  settings.fine_tz forces one.
int fine_tile_height(const tf_handle* h, int nz, bool fp64) {
  if (!h->k0_reflect) return 8;
  if (h->s.fine_tz == 7 || h->s.fine_tz == 8 || h->s.fine_tz == 9) return h->s.fine_tz;
  const int pad8 = ((nz + 7) / 8) * 8, pad9 = ((nz + 8) / 9) * 9, pad7 = ((nz + 6) / 7) * 7;
  if (100 * pad9 < 85 * pad8) return 9;
  if (!fp64 && 10 * pad7 <= 9 * pad8) return 7;
  return 8;
}

// Per-column count of the FP64 finest-level operator's curvature partials: its tiles (one node per
// thread along x, tz nodes high) times the warps of a tile.
long long fine_dot_stride(const tf_handle* h, int tz) {
  const Geo& g = h->geo[0];
  const long long tiles = (long long)((g.nx + FTXT - 1) / FTXT) * ((g.ny + TY - 1) / TY) * ((g.nz + tz - 1) / tz);
  return tiles * ((FTXT * TY * tz + 31) / 32);
}

template <typename T>
void launch_fine(tf_handle* h, const LevelArgs<T>& a, int mode, cudaStream_t st) {
  if constexpr (std::is_same<T, float>::value) {
    if (h->s.tensor_cores) {
      launch_fine_tc(h, a, mode, st);
      return;
    }
  }
  const int slot = k0_slot(h);
  const int tz = fine_tile_height(h, a.g.nz, std::is_same<T, double>::value);
  if (h->k0_reflect) {
    if (tz == 9) {
      if (slot == 0) launch_fine_variant<T, 0, true, 9>(a, mode, st);
      else launch_fine_variant<T, 1, true, 9>(a, mode, st);
    } else if (tz == 7) {
      if (slot == 0) launch_fine_variant<T, 0, true, 7>(a, mode, st);
      else launch_fine_variant<T, 1, true, 7>(a, mode, st);
    } else {
      if (slot == 0) launch_fine_variant<T, 0, true, 8>(a, mode, st);
      else launch_fine_variant<T, 1, true, 8>(a, mode, st);
    }
  } else {
    if (slot == 0) launch_fine_variant<T, 0, false, 8>(a, mode, st);
    else launch_fine_variant<T, 1, false, 8>(a, mode, st);
  }
}

template <typename T>
void launch_level(tf_handle* h, int l, LevelArgs<T> a, int mode, cudaStream_t st, int timer = -1) {
  TimedRange tr(h->timers, timer >= 0 ? timer : (l == 0 ? TIMER_FINE_WORK : TIMER_COARSE), st);
  if (l == 0) {
    launch_fine<T>(h, a, mode, st);
  } else {
    const TileMap tm = tile_map(a.g);
    const int threads = TX * TY * tm.tz;
    const unsigned tiles = (unsigned)(tm.tiles_x * tm.tiles_y * tm.tiles_z);
    constexpr int cb = sizeof(T) == 4 ? CB32 : CB64;
    constexpr size_t smem = stencil_smem_bytes<T, cb>();
    auto launch = [&](auto rnd) {
      constexpr int RND = decltype(rnd)::value;
      static bool configured = false;   // per instantiation and process; the attribute is per function
      if (!configured) {
        TF_CUDA_CHECK(cudaFuncSetAttribute(stencil_level_kernel<T, cb, RND>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured = true;
      }
      stencil_level_kernel<T, cb, RND><<<dim3(tiles, (a.ncol + cb - 1) / cb), threads, smem, st>>>(a, mode, tm);
    };
    if (std::is_same<T, float>::value && a.round == 1) launch(std::integral_constant<int, 1>{});
    else if (std::is_same<T, float>::value && a.round == 2) launch(std::integral_constant<int, 2>{});
    else launch(std::integral_constant<int, 0>{});
    TF_LAUNCH_CHECK("stencil_level_kernel");
  }
}

template <typename T>
LevelArgs<T> level_args(tf_handle* h, Hierarchy& hy, int l, int ncol, const int* active) {
  LevelArgs<T> a{};
  a.g = h->geo[l];
  a.E = level_E<T>(h, hy, l, false);
  a.mask = hy.lv[l].mask.as<uint8_t>();
  a.inv = level_inv<T>(hy, l);
  a.colstride = 3 * a.g.nnode;
  a.ncol = ncol;
  a.active = active;
  a.gate = nullptr;
  a.round = std::is_same<T, float>::value ? store_round(h) : 0;
  return a;
}

// ------------------------------------------------------------- V-cycle ------

template <typename T>
void coarsest_solve(tf_handle* h, Hierarchy& hy, VBufs<T>& vb, int ncol, const int* active, cudaStream_t st) {
  TimedRange tr(h->timers, TIMER_COARSEST, st);
  const int l = h->nlev - 1;
  const long long nd = 3 * h->geo[l].nnode;
  const int n = hy.n_live;
  const T* b = vb.b[l].template as<T>();
  T* x = vb.x[l].template as<T>();
  dim3 g0 = cols_grid(nd, ncol);
  zero_cols_kernel<T><<<g0, 256, 0, st>>>(x, nd, active);
  TF_LAUNCH_CHECK("zero_cols_kernel");
  if (n == 0) return;
  dim3 g1 = cols_grid(n, ncol);
  coarsest_gather_kernel<T><<<g1, 256, 0, st>>>(b, nd, hy.live.as<long long>(), n, h->cb.as<double>(), active);
  TF_LAUNCH_CHECK("coarsest_gather_kernel");
  const double* solved = h->cb.as<double>();
  if (hy.band) {
    // forward and backward substitution with the banded factor, one CTA per column
    band_solve(hy.X.as<double>(), n, hy.bw, h->cb.as<double>(), h->cy.as<double>(), ncol, st);
    solved = h->cy.as<double>();
  } else {
    const size_t need = dense_trimul_work(n, ncol);
    if (h->trimul_work.bytes < need) h->trimul_work.alloc(need);
    dense_trimul(hy.X.as<double>(), h->cb.as<double>(), h->cy.as<double>(), n, ncol, 0, active, h->trimul_work.as<double>(), st);
    dense_trimul(hy.X.as<double>(), h->cy.as<double>(), h->cb.as<double>(), n, ncol, 1, active, h->trimul_work.as<double>(), st);
  }
  coarsest_scatter_kernel<T><<<g1, 256, 0, st>>>(solved, hy.live.as<long long>(), n, x, nd, active, store_round(h));
  TF_LAUNCH_CHECK("coarsest_scatter_kernel");
}

template <typename T>
void smooth(tf_handle* h, Hierarchy& hy, VBufs<T>& vb, int l, bool first, int ncol, const int* active, cudaStream_t st) {
  const tf_settings& s = h->s;
  const long long nd = 3 * h->geo[l].nnode;
  const double lam = hy.lv[l].lambda_max;
  const bool jacobi = s.smoother == TF_SMOOTHER_JACOBI;
  const int base = jacobi ? s.sweeps : s.chebyshev_degree;
  const int count = std::max(1, (int)std::lround(base * std::pow(s.growth, l)));
  LevelArgs<T> a = level_args<T>(h, hy, l, ncol, active);
  dim3 ge = cols_grid(nd, ncol);
  if (jacobi) {
    const T step = static_cast<T>(s.damping / lam);
    int start = 0;
    if (first) {
      jacobi_first_kernel<T><<<ge, 256, 0, st>>>(nd, a.inv, vb.b[l].template as<T>(), vb.x[l].template as<T>(), step, active,
                                                  store_round(h));
      TF_LAUNCH_CHECK("jacobi_first_kernel");
      start = 1;
    }
    for (int k = start; k < count; ++k) {
      a.u = vb.x[l].template as<T>();
      a.b = vb.b[l].template as<T>();
      a.y = vb.xa[l].template as<T>();
      a.s = step;
      launch_level<T>(h, l, a, MODE_JACOBI, st);
      std::swap(vb.x[l], vb.xa[l]);
    }
    return;
  }
  const double upper = 1.1 * lam, lower = upper / s.chebyshev_ratio;
  const double theta = 0.5 * (upper + lower), delta = 0.5 * (upper - lower);
  const double sigma = theta / delta;
  double rho = 1.0 / sigma;
  if (!first) {
    a.u = vb.x[l].template as<T>();
    a.b = vb.b[l].template as<T>();
    a.y = vb.res[l].template as<T>();
    launch_level<T>(h, l, a, MODE_RESID, st);
  }
  // with one sweep nothing reads res or d afterwards (the V-cycle's next residual apply rewrites res)
  cheb_first_kernel<T><<<ge, 256, 0, st>>>(nd, a.inv, vb.b[l].template as<T>(), vb.res[l].template as<T>(),
                                           vb.d[l].template as<T>(), vb.x[l].template as<T>(), static_cast<T>(1.0 / theta),
                                           first ? 0 : 1, count > 1 ? 1 : 0, active, store_round(h));
  TF_LAUNCH_CHECK("cheb_first_kernel");
  for (int k = 1; k < count; ++k) {
    const double rn = 1.0 / (2.0 * sigma - rho);
    a.u = vb.d[l].template as<T>();
    a.res = vb.res[l].template as<T>();
    a.x = vb.x[l].template as<T>();
    a.y = vb.da[l].template as<T>();
    a.c1 = static_cast<T>(rn * rho);
    a.c2 = static_cast<T>(2.0 * rn / delta);
    launch_level<T>(h, l, a, MODE_CHEB, st);
    std::swap(vb.d[l], vb.da[l]);
    rho = rn;
  }
}

template <typename T>
void vcycle(tf_handle* h, Hierarchy& hy, VBufs<T>& vb, int l, int ncol, const int* active, cudaStream_t st) {
  if (l == h->nlev - 1) {
    coarsest_solve<T>(h, hy, vb, ncol, active, st);
    return;
  }
  smooth<T>(h, hy, vb, l, true, ncol, active, st);
  const int reps = (h->s.cycle == TF_CYCLE_W && l + 2 < h->nlev) ? 2 : 1;
  const Geo& fg = h->geo[l];
  const Geo& cg = h->geo[l + 1];
  for (int rep = 0; rep < reps; ++rep) {
    LevelArgs<T> a = level_args<T>(h, hy, l, ncol, active);
    a.u = vb.x[l].template as<T>();
    a.b = vb.b[l].template as<T>();
    a.y = vb.res[l].template as<T>();
    launch_level<T>(h, l, a, MODE_RESID, st);
    {
    TimedRange tr(h->timers, TIMER_TRANSFER, st);
    restrict_kernel<T><<<cols_grid(cg.nnode, ncol), 256, 0, st>>>(fg, cg, vb.res[l].template as<T>(), 3 * fg.nnode,
                                                                  vb.b[l + 1].template as<T>(), 3 * cg.nnode,
                                                                  hy.lv[l + 1].mask.as<uint8_t>(), active, store_round(h));
    TF_LAUNCH_CHECK("restrict_kernel");
    }
    vcycle<T>(h, hy, vb, l + 1, ncol, active, st);
    TimedRange tr(h->timers, TIMER_TRANSFER, st);
    prolong_add_kernel<T><<<cols_grid(cg.nnode, ncol), 256, 0, st>>>(fg, cg, vb.x[l + 1].template as<T>(), 3 * cg.nnode,
                                                                     vb.x[l].template as<T>(), 3 * fg.nnode,
                                                                     hy.lv[l].mask.as<uint8_t>(), active, store_round(h));
    TF_LAUNCH_CHECK("prolong_add_kernel");
  }
  smooth<T>(h, hy, vb, l, false, ncol, active, st);
}

// ----------------------------------------------------------- hierarchy ------

template <typename T>
double power_lambda(tf_handle* h, Hierarchy& hy, int l, cudaStream_t st) {
  VBufs<T>& vb = vbufs<T>(h);
  const Geo& g = h->geo[l];
  const long long nd = 3 * g.nnode;
  T* v = vb.x[l].template as<T>();
  T* y = vb.res[l].template as<T>();
  power_init_kernel<T><<<grid_for(g.nnode, 256), 256, 0, st>>>(g.nnode, hy.lv[l].mask.as<uint8_t>(), v);
  TF_LAUNCH_CHECK("power_init_kernel");
  double* est = h->scal.as<double>();
  for (int it = 0; it < h->s.power_iterations; ++it) {
    LevelArgs<T> a = level_args<T>(h, hy, l, 1, nullptr);
    a.u = v;
    a.y = y;
    launch_level<T>(h, l, a, MODE_APPLY, st);
    power_scale_kernel<T><<<grid_for(nd, 256, PCG_BLOCKS), 256, 0, st>>>(nd, level_inv<T>(hy, l), y, h->partial.as<double>(),
                                                                          h->count.as<unsigned>(), est);
    TF_LAUNCH_CHECK("power_scale_kernel");
    power_norm_kernel<T><<<grid_for(nd, 256), 256, 0, st>>>(nd, y, est, v);
    TF_LAUNCH_CHECK("power_norm_kernel");
  }
  double host = 1.0;
  if (h->s.power_iterations > 0) {
    TF_CUDA_CHECK(cudaMemcpyAsync(&host, est, sizeof(double), cudaMemcpyDeviceToHost, st));
    TF_CUDA_CHECK(cudaStreamSynchronize(st));
  }
  if (!std::isfinite(host) || host <= 0.0) throw Error(TF_NUMERIC, "lambda_max power iteration broke down on level " + std::to_string(l));
  return host;
}

void build_hierarchy(tf_handle* h, uint64_t key, Hierarchy& hy, cudaStream_t st) {
  auto t0 = std::chrono::steady_clock::now();
  const bool timing = h->timers.enabled;
  h->timers.enabled = false;   // the set-up is timed as one range below
  struct Restore { Timers& t; bool v; ~Restore() { t.enabled = v; } } restore{h->timers, timing};
  std::pair<cudaEvent_t, cudaEvent_t>* range = timing ? h->timers.next(TIMER_SETUP) : nullptr;
  if (range) cudaEventRecord(range->first, st);
  const bool dbl = work_is_double(h);
  ensure_scratch(h, 1);
  if ((int)hy.lv.size() != h->nlev) {
    hy.lv.clear();
    hy.lv.resize(h->nlev);
  }
  const std::vector<int64_t>& fixed = h->bcs.at(key);
  // level 0
  Level& f = hy.lv[0];
  f.g = h->geo[0];
  f.ndof = 3 * f.g.nnode;
  f.nelem = (long long)f.g.ex * f.g.ey * f.g.ez;
  {
    std::vector<uint8_t> bits(f.g.nnode, 0);
    const Geo& un = h->un;
    const long long nd_un = 3 * un.nnode;
    for (int64_t dof : fixed) {
      if (dof < 0 || dof >= nd_un) throw Error(TF_INVALID, "fixed dof index out of range");
      const long long node = dof / 3;
      const int comp = static_cast<int>(dof % 3);
      const long long k = node % un.nz, r = node / un.nz, j = r % un.ny, i = r / un.ny;
      const long long pn = (i * f.g.ny + j) * f.g.nz + k;
      bits[pn] |= static_cast<uint8_t>(1u << comp);
    }
    DevBuf& dbits = hy.bits;
    dbits.ensure(bits.size());
    TF_CUDA_CHECK(cudaMemcpyAsync(dbits.p, bits.data(), bits.size(), cudaMemcpyHostToDevice, st));
    f.mask.ensure(f.g.nnode);
    fine_mask_kernel<<<grid_for(f.g.nnode, 256), 256, 0, st>>>(f.g, h->moduli64.as<double>(), dbits.as<uint8_t>(), f.mask.as<uint8_t>());
    TF_LAUNCH_CHECK("fine_mask_kernel");
    DevBuf& diag = h->tmp_diag;
    diag.ensure(sizeof(double) * f.ndof);
    fine_diag_kernel<<<grid_for(f.g.nnode, 256), 256, 0, st>>>(f.g, h->moduli64.as<double>(), f.mask.as<uint8_t>(),
                                                               h->k0diag.as<double>(), diag.as<double>());
    TF_LAUNCH_CHECK("fine_diag_kernel");
    f.inv64.ensure(sizeof(double) * f.ndof);
    if (!dbl) f.invw.ensure(sizeof(float) * f.ndof);
    fine_inv_kernel<float><<<grid_for(f.g.nnode, 256), 256, 0, st>>>(f.g.nnode, diag.as<double>(), f.mask.as<uint8_t>(),
                                                                     f.inv64.as<double>(), dbl ? nullptr : f.invw.as<float>());
    TF_LAUNCH_CHECK("fine_inv_kernel");
  }
  for (int l = 1; l < h->nlev; ++l) {
    Level& c = hy.lv[l];
    Level& p = hy.lv[l - 1];
    c.g = h->geo[l];
    c.ndof = 3 * c.g.nnode;
    c.nelem = (long long)c.g.ex * c.g.ey * c.g.ez;
    c.blocks64.ensure(sizeof(double) * 576 * c.nelem);
    galerkin_kernel<<<grid_for(c.nelem, 1, 148 * 16), 128, 0, st>>>(h->W, c.g, p.g, l == 1 ? 1 : 0, h->moduli64.as<double>(),
                                                                     hy.lv[0].mask.as<uint8_t>(), h->K0dev.as<double>(),
                                                                     h->Q.as<double>(), l == 1 ? nullptr : p.blocks64.as<double>(),
                                                                     c.blocks64.as<double>());
    TF_LAUNCH_CHECK("galerkin_kernel");
    DevBuf& diag = h->tmp_diag;
    block_diag_kernel<<<grid_for(c.g.nnode, 256), 256, 0, st>>>(c.g, c.blocks64.as<double>(), diag.as<double>());
    TF_LAUNCH_CHECK("block_diag_kernel");
    double* dmax = h->scal.as<double>() + 1;
    amax_kernel<<<grid_for(c.ndof, 256, PCG_BLOCKS), 256, 0, st>>>(diag.as<double>(), c.ndof, h->partial.as<double>(),
                                                                   h->count.as<unsigned>(), dmax);
    TF_LAUNCH_CHECK("amax_kernel");
    c.mask.ensure(c.g.nnode);
    c.inv64.ensure(sizeof(double) * c.ndof);
    if (!dbl) c.invw.ensure(sizeof(float) * c.ndof);
    coarse_mask_inv_kernel<float><<<grid_for(c.g.nnode, 256), 256, 0, st>>>(c.g.nnode, diag.as<double>(), dmax, h->s.dead_ratio,
                                                                            c.mask.as<uint8_t>(), c.inv64.as<double>(),
                                                                            dbl ? nullptr : c.invw.as<float>());
    TF_LAUNCH_CHECK("coarse_mask_inv_kernel");
    c.stencil64.ensure(sizeof(double) * 243 * c.g.nnode);
    if (!dbl) c.stencilw.ensure(sizeof(float) * 243 * c.g.nnode);
    stencil_assemble_kernel<<<grid_for(27 * c.g.nnode, 256), 256, 0, st>>>(c.g, c.blocks64.as<double>(), c.stencil64.as<double>(),
                                                                           dbl ? nullptr : c.stencilw.as<float>());
    TF_LAUNCH_CHECK("stencil_assemble_kernel");
  }
  // Dense coarsest factor of the live dofs.  It depends on nothing the power iterations below
  // produce, so it runs on the handle's side stream while they run on `st`.
  if (dbl) ensure_vbufs<double>(h, 1); else ensure_vbufs<float>(h, 1);
  Level& cl = hy.lv[h->nlev - 1];
  std::vector<uint8_t> cmask(cl.g.nnode);
  TF_CUDA_CHECK(cudaMemcpyAsync(cmask.data(), cl.mask.p, cmask.size(), cudaMemcpyDeviceToHost, st));
  TF_CUDA_CHECK(cudaStreamSynchronize(st));
  std::vector<long long> live;
  std::vector<int> live_of(cl.ndof, -1);
  for (long long n = 0; n < cl.g.nnode; ++n)
    for (int a = 0; a < 3; ++a)
      if ((cmask[n] >> a) & 1u) {
        live_of[3 * n + a] = static_cast<int>(live.size());
        live.push_back(3 * n + a);
      }
  const long long nl = static_cast<long long>(live.size());
  // above the dense limit the coarsest factor is banded: its bandwidth is the largest live-index
  // distance between two coupled dofs (nodes within one step of each other)
  hy.band = nl > DENSE_LIMIT;
  hy.bw = 0;
  if (hy.band) {
    long long bw = 0;
    for (long long t = 0; t < nl; ++t) {
      const long long node = live[t] / 3;
      int i, j, k;
      {
        const long long r = node / cl.g.nz;
        k = static_cast<int>(node - r * cl.g.nz);
        j = static_cast<int>(r % cl.g.ny);
        i = static_cast<int>(r / cl.g.ny);
      }
      for (int di = -1; di <= 1; ++di)
        for (int dj = -1; dj <= 1; ++dj)
          for (int dk = -1; dk <= 1; ++dk) {
            const int ni = i + di, nj = j + dj, nk = k + dk;
            if (ni < 0 || nj < 0 || nk < 0 || ni >= cl.g.nx || nj >= cl.g.ny || nk >= cl.g.nz) continue;
            const long long m = ((long long)ni * cl.g.ny + nj) * cl.g.nz + nk;
            for (int q = 0; q < 3; ++q) {
              const int col = live_of[3 * m + q];
              if (col >= 0) bw = std::max(bw, std::abs(t - col));
            }
          }
    }
    require(8.0 * (double)nl * (double)(bw + 1) <= BAND_LIMIT_BYTES,
            "coarsest grid has " + std::to_string(nl) + " live dofs with bandwidth " + std::to_string(bw) +
                ": its banded factor exceeds 32 GB (raise max_levels or lower coarsest_dofs)");
    hy.bw = static_cast<int>(bw);
  }
  hy.n_live = static_cast<int>(nl);
  int* info = reinterpret_cast<int*>(h->scal.as<double>() + 8);
  if (nl > 0) {
    hy.live.ensure(sizeof(long long) * nl);
    TF_CUDA_CHECK(cudaMemcpyAsync(hy.live.p, live.data(), sizeof(long long) * nl, cudaMemcpyHostToDevice, st));
    DevBuf& dlive_of = hy.live_of;
    dlive_of.ensure(sizeof(int) * cl.ndof);
    TF_CUDA_CHECK(cudaMemcpyAsync(dlive_of.p, live_of.data(), sizeof(int) * cl.ndof, cudaMemcpyHostToDevice, st));
    DevBuf& A = hy.A;
    if (hy.band) {
      hy.X.ensure(sizeof(double) * nl * (size_t)(hy.bw + 1));
      TF_CUDA_CHECK(cudaMemsetAsync(hy.X.p, 0, hy.X.bytes, st));
      coarsest_assemble_band_kernel<<<grid_for(nl, 128), 128, 0, st>>>(cl.g, cl.blocks64.as<double>(), dlive_of.as<int>(),
                                                                       hy.live.as<long long>(), static_cast<int>(nl), hy.bw,
                                                                       hy.X.as<double>());
      TF_LAUNCH_CHECK("coarsest_assemble_band_kernel");
    } else {
      A.ensure(sizeof(double) * nl * nl);
      TF_CUDA_CHECK(cudaMemsetAsync(A.p, 0, A.bytes, st));
      coarsest_assemble_kernel<<<grid_for(nl, 128), 128, 0, st>>>(cl.g, cl.blocks64.as<double>(), dlive_of.as<int>(),
                                                                  hy.live.as<long long>(), static_cast<int>(nl), A.as<double>());
      TF_LAUNCH_CHECK("coarsest_assemble_kernel");
      dense_symmetrize(A.as<double>(), static_cast<int>(nl), st);
      TF_CUDA_CHECK(cudaMemsetAsync(info, 0, sizeof(int), st));
      hy.X.ensure(sizeof(double) * nl * nl);
      const size_t fwork = dense_factor_work(static_cast<int>(nl));
      if (h->factor_work.bytes < fwork) h->factor_work.alloc(fwork);
    }
    if (!h->side) {
      TF_CUDA_CHECK(cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking));
      TF_CUDA_CHECK(cudaEventCreateWithFlags(&h->side_fork, cudaEventDisableTiming));
      TF_CUDA_CHECK(cudaEventCreateWithFlags(&h->side_join, cudaEventDisableTiming));
    }
    TF_CUDA_CHECK(cudaEventRecord(h->side_fork, st));
    TF_CUDA_CHECK(cudaStreamWaitEvent(h->side, h->side_fork, 0));
    if (hy.band) band_cholesky(hy.X.as<double>(), static_cast<int>(nl), hy.bw, info, h->side);
    else dense_cholesky_inverse(A.as<double>(), hy.X.as<double>(), static_cast<int>(nl), info, h->factor_work.as<double>(), h->side);
    TF_CUDA_CHECK(cudaEventRecord(h->side_join, h->side));
  }
  // lambda_max(D^-1 A) of every smoothed level, in the work precision
  for (int l = 0; l + 1 < h->nlev; ++l)
    hy.lv[l].lambda_max = dbl ? power_lambda<double>(h, hy, l, st) : power_lambda<float>(h, hy, l, st);
  if (nl > 0) {
    TF_CUDA_CHECK(cudaStreamWaitEvent(st, h->side_join, 0));
    int hinfo = 0;
    TF_CUDA_CHECK(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, st));
    TF_CUDA_CHECK(cudaStreamSynchronize(st));
    if (hinfo != 0)
      throw Error(TF_NUMERIC, "coarsest Galerkin matrix is not positive definite (pivot " + std::to_string(hinfo) +
                                  "); the supports do not remove every rigid-body mode");
  }
  if (range) cudaEventRecord(range->second, st);
  hy.setup_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  hy.setup_reported = false;
}

Hierarchy& get_hierarchy(tf_handle* h, uint64_t key, cudaStream_t st) {
  require(h->have_moduli, "update(moduli) must be called before solving");
  require(h->bcs.count(key) > 0, "no boundary conditions registered for this key (tf_set_bc)");
  Hierarchy& hy = h->hier[key];
  if (hy.valid) return hy;
  try {
    build_hierarchy(h, key, hy, st);
  } catch (...) {
    h->hier.erase(key);
    throw;
  }
  hy.valid = true;
  return hy;
}

void ensure_coarse_work(tf_handle* h, Hierarchy& hy, int ncol) {
  const size_t need = sizeof(double) * (size_t)std::max(hy.n_live, 1) * ncol;
  if (h->ccap < need) {
    h->cb.alloc(need);
    h->cy.alloc(need);
    h->ccap = need;
  }
}

// ----------------------------------------------------------------- PCG ------

// z = M r for the active columns: r scaled by its column max into the work precision, one cycle,
// and the new search direction p.  With `prep` the scale is formed here; otherwise pcg_take_kernel /
// pcg_update_kernel / pcg_retire_kernel have formed it.  z is stored only with store_z.  R is the
// type of the PCG vectors r and p (double, or float in the mixed PCG).
template <typename T, typename R>
void precondition(tf_handle* h, Hierarchy& hy, int ncol, const PcgState& st, int initial, bool store_z, cudaStream_t s,
                  bool prep = false) {
  const long long n = 3 * h->geo[0].nnode;
  VBufs<T>& vb = vbufs<T>(h);
  R* r = static_cast<R*>(h->vr.p);
  dim3 gr(grid_for(n, RED_THREADS, PCG_BLOCKS), ncol);
  {
  TimedRange tr_(h->timers, TIMER_VECTOR, s);
  if (prep) {
    pcg_prep_kernel<R><<<gr, RED_THREADS, 0, s>>>(r, n, st);
    TF_LAUNCH_CHECK("pcg_prep_kernel");
  }
  pcg_to_work_kernel<T, R><<<cols_grid(n, ncol), 256, 0, s>>>(r, n, st, vb.b[0].template as<T>(), store_round(h));
  TF_LAUNCH_CHECK("pcg_to_work_kernel");
  }
  vcycle<T>(h, hy, vb, 0, ncol, st.active, s);
  {
  TimedRange tr_(h->timers, TIMER_VECTOR, s);
  pcg_from_work_kernel<T, R><<<gr, RED_THREADS, 0, s>>>(vb.x[0].template as<T>(), r, store_z ? h->vz.as<double>() : nullptr, n, st,
                                                        initial);
  TF_LAUNCH_CHECK("pcg_from_work_kernel");
  pcg_direction_kernel<T, R><<<cols_grid(n, ncol), 256, 0, s>>>(vb.x[0].template as<T>(), static_cast<R*>(h->vp.p), n, st, initial);
  TF_LAUNCH_CHECK("pcg_direction_kernel");
  }
}

// FP64 fine operator with mask (the PCG operator, topology_multigrid.py:411)
void fine_apply64(tf_handle* h, Hierarchy& hy, const double* u, const double* b, double* y, int mode, int ncol,
                  const int* active, const int* gate, cudaStream_t s) {
  LevelArgs<double> a{};
  a.g = h->geo[0];
  a.E = h->moduli64.as<double>();
  a.mask = hy.lv[0].mask.as<uint8_t>();
  a.u = u;
  a.b = b;
  a.y = y;
  a.colstride = 3 * a.g.nnode;
  a.ncol = ncol;
  a.active = active;
  a.gate = gate;
  launch_level<double>(h, 0, a, mode, s, TIMER_FINE64);
}

// FP64 PCG operator q = K p that also leaves the partial sums of p . q for the step length
// (topology_multigrid.py:424) in h->dotp, one per warp of each tile and column: the separate
// curvature pass over p and q is not needed.
void fine_apply64_curvature(tf_handle* h, Hierarchy& hy, const double* p, double* q, int ncol, const int* active, cudaStream_t s) {
  LevelArgs<double> a{};
  a.g = h->geo[0];
  a.E = h->moduli64.as<double>();
  a.mask = hy.lv[0].mask.as<uint8_t>();
  a.u = p;
  a.y = q;
  a.colstride = 3 * a.g.nnode;
  a.ncol = ncol;
  a.active = active;
  const size_t need = sizeof(double) * (size_t)fine_dot_stride(h, fine_tile_height(h, a.g.nz, true)) * ncol;
  if (h->dotp.bytes < need) h->dotp.alloc(need);
  a.dot_out = h->dotp.as<double>();
  launch_level<double>(h, 0, a, MODE_APPLY, s, TIMER_FINE64);
}

// FP32 fine operator with mask: the operator of the mixed PCG's FP32 iterations, on the CUDA-core
// stencil whatever the smoother uses (its accuracy bounds how far an FP32 stretch can reduce the
// residual between two FP64 recomputations).
void fine_apply32(tf_handle* h, Hierarchy& hy, const float* u, float* y, int ncol, const int* active, cudaStream_t s) {
  LevelArgs<float> a{};
  a.g = h->geo[0];
  a.E = h->modulif.as<float>();
  a.mask = hy.lv[0].mask.as<uint8_t>();
  a.u = u;
  a.y = y;
  a.colstride = 3 * a.g.nnode;
  a.ncol = ncol;
  a.active = active;
  TimedRange tr(h->timers, TIMER_PCG32, s);
  const int tc = h->s.tensor_cores;
  h->s.tensor_cores = 0;
  struct Restore { tf_handle* h; int v; ~Restore() { h->s.tensor_cores = v; } } restore{h, tc};
  launch_fine<float>(h, a, MODE_APPLY, s);
}

struct PcgResult {
  std::vector<int> iters;
  std::vector<double> rel;
  std::vector<double> history;
  int steps = 0;
};

PcgResult pcg_finish(tf_handle* h, Hierarchy& hy, const PcgState& st, int ncol, const std::vector<int>& run, int step, bool running,
                     cudaStream_t s);

// Batched flexible PCG over `ncol` columns held in h->vb (rhs) / h->vx (solution).
// `run` selects the columns; with `warm` the current h->vx is the start vector.
//
// R = double: the reference's FP64 PCG (FP64 operator, FP64 vectors).  R = float: the mixed PCG.
// Its iterations run in FP32 (r, p, q and the operator), while x accumulates in FP64 and the
// residual is recomputed in FP64 (b - K x, the FP64 operator) whenever a column's iterated
// residual fell by the factor settings.reliable since its last recomputation, or below the
// tolerance; the recomputed residual replaces the FP32 one (a reliable update) and decides
// convergence, so every column still converges on its FP64 true residual like the reference.
template <typename T, typename R>
PcgResult pcg(tf_handle* h, Hierarchy& hy, int ncol, const std::vector<int>& run, bool warm, cudaStream_t s) {
  constexpr bool mixed = std::is_same<R, float>::value;
  const long long n = 3 * h->geo[0].nnode;
  ensure_vbufs<T>(h, ncol);
  ensure_coarse_work(h, hy, ncol);
  PcgState st = pcg_state(h, ncol);
  const double tol = h->s.tolerance;
  const double reliable = mixed ? h->s.reliable : 0.0;
  const int limit = h->s.max_iterations;
  R* r = static_cast<R*>(h->vr.p);
  R* p = static_cast<R*>(h->vp.p);
  R* q = mixed ? static_cast<R*>(h->vz.p) : static_cast<R*>(h->vq.p);
  // the FP64 operator also forms the curvature p . q (fine_apply64_curvature)
  constexpr bool fused = !mixed;
  double* t = h->vq.as<double>();   // b - K x in FP64 (shares vq with q in the FP64 PCG: q is consumed first)
  std::vector<int> zeros(ncol, 0);
  TF_CUDA_CHECK(cudaMemcpyAsync(st.active, run.data(), sizeof(int) * ncol, cudaMemcpyHostToDevice, s));
  TF_CUDA_CHECK(cudaMemcpyAsync(st.cand, zeros.data(), sizeof(int) * ncol, cudaMemcpyHostToDevice, s));
  TF_CUDA_CHECK(cudaMemcpyAsync(st.iters, zeros.data(), sizeof(int) * ncol, cudaMemcpyHostToDevice, s));
  TF_CUDA_CHECK(cudaMemsetAsync(st.flags, 0, sizeof(int) * 8, s));
  TF_CUDA_CHECK(cudaMemsetAsync(st.hist, 0, sizeof(unsigned long long) * h->hist_cap, s));
  dim3 gr(grid_for(n, RED_THREADS, PCG_BLOCKS), ncol);
  dim3 ge = cols_grid(n, ncol);
  pcg_norm_kernel<<<gr, RED_THREADS, 0, s>>>(h->vb.as<double>(), n, st, st.bnorm, 1);
  TF_LAUNCH_CHECK("pcg_norm_kernel");
  const double* start = h->vb.as<double>();
  if (warm) {
    fine_apply64(h, hy, h->vx.as<double>(), h->vb.as<double>(), t, MODE_RESID, ncol, st.active, nullptr, s);
    start = t;
  } else {
    zero_cols_kernel<double><<<ge, 256, 0, s>>>(h->vx.as<double>(), n, st.active);
    TF_LAUNCH_CHECK("zero_cols_kernel");
  }
  {
    TimedRange tr_(h->timers, TIMER_VECTOR, s);
    pcg_take_kernel<R><<<gr, RED_THREADS, 0, s>>>(start, r, n, st);
    TF_LAUNCH_CHECK("pcg_take_kernel");
  }
  precondition<T, R>(h, hy, ncol, st, 1, false, s);
  int step = 0;
  int n_active = 0;
  for (int c = 0; c < ncol; ++c) n_active += run[c];
  while (n_active > 0 && step < limit) {
    if constexpr (mixed) fine_apply32(h, hy, p, q, ncol, st.active, s);
    else fine_apply64_curvature(h, hy, p, q, ncol, st.active, s);
    {
  TimedRange tr_(h->timers, TIMER_VECTOR, s);
  if constexpr (fused) {
    pcg_alpha_sum_kernel<<<ncol, RED_THREADS, 0, s>>>(h->dotp.as<double>(), fine_dot_stride(h, fine_tile_height(h, h->geo[0].nz, true)), st);
    TF_LAUNCH_CHECK("pcg_alpha_sum_kernel");
  } else {
    pcg_alpha_kernel<R><<<gr, RED_THREADS, 0, s>>>(p, q, n, st);
    TF_LAUNCH_CHECK("pcg_alpha_kernel");
  }
    ++step;
    pcg_update_kernel<T, R><<<gr, RED_THREADS, 0, s>>>(h->vx.as<double>(), r, p, q, vbufs<T>(h).x[0].template as<T>(), n, st, tol,
                                                       step, reliable);
    TF_LAUNCH_CHECK("pcg_update_kernel");
  }
    fine_apply64(h, hy, h->vx.as<double>(), h->vb.as<double>(), t, MODE_RESID, ncol, st.active, st.flags, s);
    {
  TimedRange tr_(h->timers, TIMER_VECTOR, s);
  pcg_truecheck_kernel<<<gr, RED_THREADS, 0, s>>>(t, n, st, tol, step);
    TF_LAUNCH_CHECK("pcg_truecheck_kernel");
    pcg_retire_kernel<T, R><<<gr, RED_THREADS, 0, s>>>(t, r, vbufs<T>(h).x[0].template as<T>(), n, st);
    TF_LAUNCH_CHECK("pcg_retire_kernel");
    pcg_flags_kernel<<<1, 256, 0, s>>>(st, step);
    TF_LAUNCH_CHECK("pcg_flags_kernel");
  }
    TF_CUDA_CHECK(cudaMemcpyAsync(h->host_flags, st.flags + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    TF_CUDA_CHECK(cudaStreamSynchronize(s));
    n_active = h->host_flags[0];
    if (n_active == 0) break;
    precondition<T, R>(h, hy, ncol, st, 0, false, s);
  }
  return pcg_finish(h, hy, st, ncol, run, step, n_active > 0, s);
}

// The per-column outcome of a PCG run that took `step` steps: with `running` (the iteration limit
// stopped it) the columns still active get their final true residual (topology_multigrid.py:450-453).
PcgResult pcg_finish(tf_handle* h, Hierarchy& hy, const PcgState& st, int ncol, const std::vector<int>& run, int step, bool running,
                     cudaStream_t s) {
  const long long n = 3 * h->geo[0].nnode;
  PcgResult res;
  res.steps = step;
  if (running) {
    double* t = h->vq.as<double>();
    fine_apply64(h, hy, h->vx.as<double>(), h->vb.as<double>(), t, MODE_RESID, ncol, st.active, nullptr, s);
    pcg_norm_kernel<<<dim3(grid_for(n, RED_THREADS, PCG_BLOCKS), ncol), RED_THREADS, 0, s>>>(t, n, st, st.rzo, 1);
    TF_LAUNCH_CHECK("pcg_norm_kernel");
  }
  std::vector<int> act(ncol), it(ncol);
  std::vector<double> rel(ncol), bn(ncol), fin(ncol);
  std::vector<unsigned long long> hb(std::max(step, 1));
  TF_CUDA_CHECK(cudaMemcpyAsync(act.data(), st.active, sizeof(int) * ncol, cudaMemcpyDeviceToHost, s));
  TF_CUDA_CHECK(cudaMemcpyAsync(it.data(), st.iters, sizeof(int) * ncol, cudaMemcpyDeviceToHost, s));
  TF_CUDA_CHECK(cudaMemcpyAsync(rel.data(), st.rel, sizeof(double) * ncol, cudaMemcpyDeviceToHost, s));
  TF_CUDA_CHECK(cudaMemcpyAsync(bn.data(), st.bnorm, sizeof(double) * ncol, cudaMemcpyDeviceToHost, s));
  TF_CUDA_CHECK(cudaMemcpyAsync(fin.data(), st.rzo, sizeof(double) * ncol, cudaMemcpyDeviceToHost, s));
  if (step > 0)
    TF_CUDA_CHECK(cudaMemcpyAsync(hb.data(), st.hist, sizeof(unsigned long long) * step, cudaMemcpyDeviceToHost, s));
  TF_CUDA_CHECK(cudaStreamSynchronize(s));
  res.iters.assign(ncol, 0);
  res.rel.assign(ncol, 1.0);
  for (int c = 0; c < ncol; ++c) {
    if (!run[c]) continue;
    if (act[c]) {
      res.iters[c] = step;
      res.rel[c] = fin[c] / bn[c];
    } else {
      res.iters[c] = it[c];
      res.rel[c] = rel[c];
    }
  }
  for (int q = 0; q < step; ++q) {
    double v;
    std::memcpy(&v, &hb[q], sizeof(double));
    res.history.push_back(v);
  }
  return res;
}

// Precise FP64 re-run of the columns that missed the tolerance (topology_multigrid.py:376-406).
PcgResult pcg_precise(tf_handle* h, Hierarchy& hy, int ncol, const std::vector<int>& run, cudaStream_t s) {
  return pcg<double, double>(h, hy, ncol, run, true, s);
}

template <typename F>
int guard(tf_handle* h, F&& f) {
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

void validate_settings(const tf_settings& s) {
  require(s.precision >= TF_PRECISION_FLOAT64 && s.precision <= TF_PRECISION_FLOAT16, "invalid precision");
  require(s.precision <= TF_PRECISION_FLOAT32 || !s.tensor_cores,
          "bfloat16/float16 storage runs on the CUDA-core operators (tensor_cores must be off)");
  require(s.smoother == TF_SMOOTHER_JACOBI || s.smoother == TF_SMOOTHER_CHEBYSHEV, "invalid smoother");
  require(s.cycle == TF_CYCLE_V || s.cycle == TF_CYCLE_W, "invalid cycle");
  require(s.coarse == TF_COARSE_GALERKIN, "only Galerkin coarse operators are available in this library");
  require(s.sweeps >= 1 && s.chebyshev_degree >= 1, "sweeps and chebyshev_degree must be positive");
  require(s.max_levels >= 2 && s.max_levels <= 16, "max_levels must be in [2, 16]");
  require(s.power_iterations >= 1, "power_iterations must be positive");
  require(s.max_iterations >= 1, "max_iterations must be positive");
  require(s.retries >= 0 && s.batch >= 0, "retries and batch must be non-negative");
  require(s.coarsest_dofs >= 1, "coarsest_dofs must be positive");
  require(std::isfinite(s.damping) && s.damping > 0, "damping must be positive");
  require(std::isfinite(s.chebyshev_ratio) && s.chebyshev_ratio > 1, "chebyshev_ratio must exceed 1");
  require(std::isfinite(s.growth) && s.growth > 0, "growth must be positive");
  require(std::isfinite(s.tolerance) && s.tolerance > 0, "tolerance must be positive");
  require(std::isfinite(s.dead_ratio) && s.dead_ratio >= 0, "dead_ratio must be non-negative");
  require(std::isfinite(s.zero_rhs) && s.zero_rhs >= 0, "zero_rhs must be non-negative");
  require(s.pcg_precision == TF_PRECISION_FLOAT64 || s.pcg_precision == TF_PRECISION_FLOAT32,
          "pcg_precision must be float64 or float32");
  require(s.pcg_precision == TF_PRECISION_FLOAT64 || s.precision != TF_PRECISION_FLOAT64,
          "float32 PCG iterations need the float32 work precision");
  require(std::isfinite(s.reliable) && s.reliable > 0 && s.reliable < 1, "reliable must be in (0, 1)");
  require(s.fine_tz == 0 || s.fine_tz == 7 || s.fine_tz == 8 || s.fine_tz == 9, "fine_tz must be 0, 7, 8 or 9");
}

}  // namespace

// =============================================================== C ABI ======

namespace tfb {
// Message for tf_last_error(NULL) from entry points that take no handle.
void record_unhandled_error(const std::string& message) { g_last_create_error = message; }
const char* unhandled_error() { return g_last_create_error.c_str(); }
}  // namespace tfb

extern "C" int tf_default_settings(tf_settings* s) {
  if (!s) return TF_INVALID;
  *s = tf_settings{};
  s->precision = TF_PRECISION_FLOAT32;
  s->smoother = TF_SMOOTHER_CHEBYSHEV;
  s->cycle = TF_CYCLE_V;
  s->coarse = TF_COARSE_GALERKIN;
  s->sweeps = 2;
  s->chebyshev_degree = 3;
  s->max_levels = 8;
  s->power_iterations = 20;
  s->max_iterations = 2000;
  s->retries = 2;
  s->batch = 0;
  s->coarsest_dofs = 8000;
  s->damping = 1.0;
  s->chebyshev_ratio = 20.0;
  s->growth = 2.0;
  s->tolerance = 1e-8;
  s->dead_ratio = 1e-12;
  s->zero_rhs = 1e-12;
  s->reliable = 0.01;
  s->pcg_precision = TF_PRECISION_FLOAT64;
  return TF_OK;
}

extern "C" int tf_create(const tf_grid* grid, const double* ke, const double* me, const tf_settings* settings, tf_handle** out) {
  g_last_create_error.clear();
  if (!out) { g_last_create_error = "out must not be NULL"; return TF_INVALID; }
  *out = nullptr;
  tf_handle* h = new tf_handle();
  int rc = guard(h, [&] {
    require(grid && ke, "grid and ke must not be NULL");
    if (settings) h->s = *settings; else tf_default_settings(&h->s);
    validate_settings(h->s);
    for (int d = 0; d < 3; ++d) {
      require(grid->shape[d] >= 1 && grid->shape[d] < (1 << 20), "grid shape must be positive");
      require(std::isfinite(grid->spacing[d]) && grid->spacing[d] > 0, "grid spacing must be finite and positive");
      h->shape[d] = grid->shape[d];
      h->spacing[d] = grid->spacing[d];
    }
    for (int t = 0; t < 576; ++t) {
      require(std::isfinite(ke[t]), "ke must be finite");
      h->ke[t] = ke[t];
      h->k64.k[t] = ke[t];
      h->k32.k[t] = static_cast<float>(ke[t]);
    }
    if (me) {
      for (int t = 0; t < 576; ++t) {
        require(std::isfinite(me[t]), "me must be finite");
        h->m64.k[t] = me[t];
      }
      h->have_me = true;
    }
    {
      // reflection symmetry of ke (box element, axis-aligned orthotropic material)
      double kmax = 0.0, err = 0.0;
      for (int t = 0; t < 576; ++t) kmax = std::max(kmax, std::fabs(ke[t]));
      for (int c = 0; c < 8; ++c)
        for (int a = 0; a < 3; ++a)
          for (int d = 0; d < 8; ++d)
            for (int b = 0; b < 3; ++b) {
              const int rx = corner_x(c), ry = corner_y(c), rz = corner_z(c);
              const int rd = corner_id(corner_x(d) ^ rx, corner_y(d) ^ ry, corner_z(d) ^ rz);
              const int ra = a == 0 ? rx : (a == 1 ? ry : rz), rb = b == 0 ? rx : (b == 1 ? ry : rz);
              const double v = ((ra ^ rb) ? -1.0 : 1.0) * ke[a * 24 + 3 * rd + b];
              err = std::max(err, std::fabs(ke[(3 * c + a) * 24 + 3 * d + b] - v));
            }
      h->k0_reflect = err <= 1e-13 * kmax;
    }
    // level count and padding (topology_multigrid.py:58-63)
    int count = 2;
    auto coarse_dofs = [&](int c) {
      double p = 3.0;
      for (int d = 0; d < 3; ++d) p *= std::ceil(double(h->shape[d]) / std::pow(2.0, c - 1)) + 1.0;
      return p;
    };
    while (count < h->s.max_levels && coarse_dofs(count) > double(h->s.coarsest_dofs)) ++count;
    const long long factor = 1LL << (count - 1);
    for (int d = 0; d < 3; ++d) h->padded[d] = ((h->shape[d] + factor - 1) / factor) * factor;
    h->nlev = count;
    for (int l = 0; l < count; ++l)
      h->geo.push_back(make_geo(h->padded[0] >> l, h->padded[1] >> l, h->padded[2] >> l));
    h->un = make_geo(h->shape[0], h->shape[1], h->shape[2]);
    require(h->geo[0].nnode < (1LL << 31), "grid too large: the padded grid must have fewer than 2^31 nodes");
    // trilinear interpolation weights W[child][fine corner][coarse corner] (topology_multigrid.py:19-27)
    static const int C[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    for (int c = 0; c < 8; ++c) {
      const int off[3] = {c >> 2, (c >> 1) & 1, c & 1};
      for (int r = 0; r < 8; ++r)
        for (int s2 = 0; s2 < 8; ++s2) {
          double w = 1.0;
          for (int d = 0; d < 3; ++d) {
            const double pos = 0.5 * (off[d] + C[r][d]);
            w *= C[s2][d] == 1 ? pos : 1.0 - pos;
          }
          h->W.W[c][r][s2] = w;
        }
    }
    // Q_c = P_c^T K0 P_c for children whose 24 dofs are all live
    std::vector<double> Q(8 * 576, 0.0);
    for (int c = 0; c < 8; ++c)
      for (int s1 = 0; s1 < 8; ++s1)
        for (int x = 0; x < 3; ++x)
          for (int t = 0; t < 8; ++t)
            for (int y = 0; y < 3; ++y) {
              double v = 0.0;
              for (int r = 0; r < 8; ++r)
                for (int q = 0; q < 8; ++q) v += h->W.W[c][r][s1] * ke[(3 * r + x) * 24 + 3 * q + y] * h->W.W[c][q][t];
              Q[c * 576 + (3 * s1 + x) * 24 + 3 * t + y] = v;
            }
    h->Q.alloc(sizeof(double) * Q.size());
    TF_CUDA_CHECK(cudaMemcpy(h->Q.p, Q.data(), sizeof(double) * Q.size(), cudaMemcpyHostToDevice));
    h->K0dev.alloc(sizeof(double) * 576);
    TF_CUDA_CHECK(cudaMemcpy(h->K0dev.p, ke, sizeof(double) * 576, cudaMemcpyHostToDevice));
    double kd[24];
    for (int t = 0; t < 24; ++t) kd[t] = ke[t * 25];
    h->k0diag.alloc(sizeof(kd));
    TF_CUDA_CHECK(cudaMemcpy(h->k0diag.p, kd, sizeof(kd), cudaMemcpyHostToDevice));
    const long long ne = h->un.ex * (long long)h->un.ey * h->un.ez;
    const long long np = (long long)h->geo[0].ex * h->geo[0].ey * h->geo[0].ez;
    h->moduli_un.alloc(sizeof(double) * ne);
    h->moduli64.alloc(sizeof(double) * np);
    TF_CUDA_CHECK(cudaMemset(h->moduli64.p, 0, h->moduli64.bytes));
    if (!work_is_double(h)) {
      h->modulif.alloc(sizeof(float) * np);
      TF_CUDA_CHECK(cudaMemset(h->modulif.p, 0, h->modulif.bytes));
    }
    ensure_scratch(h, 1);
  });
  if (rc != TF_OK) {
    g_last_create_error = h->err;
    delete h;
    return rc;
  }
  *out = h;
  return TF_OK;
}

extern "C" int tf_levels(const tf_handle* h, int32_t* levels, int64_t padded[3]) {
  if (!h) return TF_INVALID;
  if (levels) *levels = h->nlev;
  if (padded)
    for (int d = 0; d < 3; ++d) padded[d] = h->padded[d];
  return TF_OK;
}

namespace {
__global__ void pad_moduli_kernel(Geo un, Geo pd, const double* __restrict__ src, double* __restrict__ dst64, float* __restrict__ dstf) {
  const long long total = (long long)pd.ex * pd.ey * pd.ez;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int k = static_cast<int>(e % pd.ez);
    const long long r = e / pd.ez;
    const int j = static_cast<int>(r % pd.ey), i = static_cast<int>(r / pd.ey);
    const double v = (i < un.ex && j < un.ey && k < un.ez) ? src[((long long)i * un.ey + j) * un.ez + k] : 0.0;
    dst64[e] = v;
    if (dstf) dstf[e] = static_cast<float>(v);
  }
}
}  // namespace

extern "C" int tf_update(tf_handle* h, const double* moduli_dev, void* stream) {
  if (!h) return TF_INVALID;
  return guard(h, [&] {
    require(moduli_dev != nullptr, "moduli must not be NULL");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long ne = (long long)h->un.ex * h->un.ey * h->un.ez;
    TF_CUDA_CHECK(cudaMemcpyAsync(h->moduli_un.p, moduli_dev, sizeof(double) * ne, cudaMemcpyDeviceToDevice, s));
    const Geo& pd = h->geo[0];
    pad_moduli_kernel<<<grid_for((long long)pd.ex * pd.ey * pd.ez, 256), 256, 0, s>>>(
        h->un, pd, h->moduli_un.as<double>(), h->moduli64.as<double>(), work_is_double(h) ? nullptr : h->modulif.as<float>());
    TF_LAUNCH_CHECK("pad_moduli_kernel");
    for (auto& kv : h->hier) kv.second.valid = false;   // rebuilt lazily, reusing their buffers
    h->have_moduli = true;
  });
}

extern "C" int tf_set_bc(tf_handle* h, uint64_t key, const int64_t* fixed, int64_t count) {
  if (!h) return TF_INVALID;
  return guard(h, [&] {
    require(count >= 0 && (count == 0 || fixed), "fixed must not be NULL");
    const long long nd = 3 * h->un.nnode;
    std::vector<int64_t> v(fixed, fixed + count);
    for (int64_t d : v) require(d >= 0 && d < nd, "fixed dof index out of range");
    auto it = h->bcs.find(key);
    if (it != h->bcs.end() && it->second != v) {
      auto hit = h->hier.find(key);
      if (hit != h->hier.end()) hit->second.valid = false;
    }
    h->bcs[key] = std::move(v);
  });
}

namespace {
// A tensor-core finest-level launch whose MMA wait ran out sets tc_err and skips the rest of its
// columns; surface that as an error of the call instead of returning a wrong answer.
void check_tensor_core_error(tf_handle* h, cudaStream_t s) {
  if (!h->tc_err.p) return;
  int v = 0;
  TF_CUDA_CHECK(cudaMemcpyAsync(&v, h->tc_err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  TF_CUDA_CHECK(cudaStreamSynchronize(s));
  if (v) {
    TF_CUDA_CHECK(cudaMemsetAsync(h->tc_err.p, 0, sizeof(int), s));
    throw Error(TF_INTERNAL, "tensor-core finest-level apply: an MMA completion wait timed out");
  }
}

// Shared body of tf_solve (start from zero) and tf_solve_guess (start from u_dev, the reference's
// _pcg(..., initial), topology_multigrid.py:407-417).
// The columns of f_dev whose norm is not negligible against the largest (topology_multigrid.py:350-351)
// go to `live`; the others to `dead`, and their solutions are zeroed in u_dev.
void split_columns(tf_handle* h, const double* f_dev, int32_t nrhs, double* u_dev, cudaStream_t s, std::vector<int>& live,
                   std::vector<int>& dead) {
  const long long nun = 3 * h->un.nnode;
  std::vector<double> norms(nrhs, 0.0);
  if (nrhs > 0) {
    ensure_scratch(h, nrhs);
    if (h->solve_small.bytes < sizeof(double) * nrhs) h->solve_small.alloc(sizeof(double) * nrhs);
    colnorm_kernel<<<dim3(grid_for(nun, RED_THREADS, PCG_BLOCKS), nrhs), RED_THREADS, 0, s>>>(
        f_dev, nun, h->solve_small.as<double>(), h->partial.as<double>(), h->count.as<unsigned>());
    TF_LAUNCH_CHECK("colnorm_kernel");
    TF_CUDA_CHECK(cudaMemcpyAsync(norms.data(), h->solve_small.p, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, s));
    TF_CUDA_CHECK(cudaStreamSynchronize(s));
  }
  double mx = 0.0;
  for (double v : norms) {
    if (!std::isfinite(v)) throw Error(TF_INVALID, "forces must be finite");
    mx = std::max(mx, v);
  }
  live.clear();
  dead.clear();
  for (int c = 0; c < nrhs; ++c) (norms[c] > h->s.zero_rhs * std::max(mx, 1e-300) ? live : dead).push_back(c);
  if (!dead.empty()) {
    // solve_small is reused in stream order: the norms above were read back before this copy
    if (h->solve_small.bytes < sizeof(int) * dead.size()) h->solve_small.alloc(sizeof(int) * dead.size());
    TF_CUDA_CHECK(cudaMemcpyAsync(h->solve_small.p, dead.data(), sizeof(int) * dead.size(), cudaMemcpyHostToDevice, s));
    zero_flat_cols_kernel<<<dim3(grid_for(nun, 256), (unsigned)dead.size()), 256, 0, s>>>(u_dev, nun, h->solve_small.as<int>());
    TF_LAUNCH_CHECK("zero_flat_cols_kernel");
    TF_CUDA_CHECK(cudaStreamSynchronize(s));
  }
}

// Columns `cols` of f_dev (and with `warm` of u_dev) into the padded PCG layout h->vb (h->vx).
void load_columns(tf_handle* h, Hierarchy& hy, const double* f_dev, double* u_dev, const std::vector<int>& cols, bool warm,
                  cudaStream_t s) {
  const long long nun = 3 * h->un.nnode;
  const int nc = static_cast<int>(cols.size());
  ensure_pcg(h, nc);
  TF_CUDA_CHECK(cudaMemcpyAsync(h->colmap.p, cols.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, s));
  pad_kernel<<<cols_grid(h->geo[0].nnode, nc), 256, 0, s>>>(f_dev, nun, h->un, h->geo[0], hy.lv[0].mask.as<uint8_t>(),
                                                            h->vb.as<double>(), h->colmap.as<int>());
  TF_LAUNCH_CHECK("pad_kernel");
  if (warm) {
    // the caller's guess, masked like the forces; pcg then starts from r = b - A x
    pad_kernel<<<cols_grid(h->geo[0].nnode, nc), 256, 0, s>>>(u_dev, nun, h->un, h->geo[0], hy.lv[0].mask.as<uint8_t>(),
                                                              h->vx.as<double>(), h->colmap.as<int>());
    TF_LAUNCH_CHECK("pad_kernel");
  }
}

// The precise FP64 re-runs of the columns that missed the tolerance (topology_multigrid.py:376-406),
// restarting from the previous iterate where it improved on zero (:393).
void retry_columns(tf_handle* h, Hierarchy& hy, int nc, PcgResult& r, std::vector<double>& history, int& steps, int& retried,
                   cudaStream_t s) {
  const long long n = 3 * h->geo[0].nnode;
  for (int attempt = 0; attempt < h->s.retries; ++attempt) {
    std::vector<int> failed(nc, 0);
    int nfail = 0;
    for (int c = 0; c < nc; ++c)
      if (!(r.rel[c] < h->s.tolerance)) { failed[c] = 1; ++nfail; }
    if (!nfail) break;
    std::vector<int> reset(nc, 0);
    for (int c = 0; c < nc; ++c) reset[c] = failed[c] && !(r.rel[c] < 1.0);
    // solve_small is reused in stream order (every user of it runs on stream s)
    if (h->solve_small.bytes < sizeof(int) * nc) h->solve_small.alloc(sizeof(int) * nc);
    TF_CUDA_CHECK(cudaMemcpyAsync(h->solve_small.p, reset.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, s));
    zero_cols_kernel<double><<<cols_grid(n, nc), 256, 0, s>>>(h->vx.as<double>(), n, h->solve_small.as<int>());
    TF_LAUNCH_CHECK("zero_cols_kernel");
    PcgResult again = pcg_precise(h, hy, nc, failed, s);
    for (int c = 0; c < nc; ++c)
      if (failed[c]) {
        r.iters[c] += again.iters[c];
        r.rel[c] = again.rel[c];
      }
    history.insert(history.end(), again.history.begin(), again.history.end());
    steps += again.steps;
    retried += nfail;
  }
}

// Solutions of the block `cols` back to u_dev, and the block's per-column outcome.
void store_columns(tf_handle* h, double* u_dev, const std::vector<int>& cols, const PcgResult& r, std::vector<int>& iters,
                   std::vector<double>& rel, cudaStream_t s) {
  const long long nun = 3 * h->un.nnode;
  const int nc = static_cast<int>(cols.size());
  unpad_kernel<<<cols_grid(h->un.nnode, nc), 256, 0, s>>>(h->vx.as<double>(), h->un, h->geo[0], u_dev, nun, h->colmap.as<int>());
  TF_LAUNCH_CHECK("unpad_kernel");
  for (int c = 0; c < nc; ++c) {
    iters[cols[c]] = r.iters[c];
    rel[cols[c]] = r.rel[c];
  }
}

struct SolveTally {
  std::vector<int> live, dead, iters;
  std::vector<double> rel, history;
  int batches = 0, retried = 0, steps = 0;
};

void fill_solve_report(tf_handle* h, Hierarchy& hy, tf_report* report, int32_t nrhs, const SolveTally& t,
                       std::chrono::steady_clock::time_point t0) {
  bool converged = true;
  for (int c : t.live) converged &= t.rel[c] < h->s.tolerance;
  if (report) {
    if (report->iterations)
      for (int c = 0; c < nrhs; ++c) report->iterations[c] = t.iters[c];
    if (report->relative_residual)
      for (int c = 0; c < nrhs; ++c) report->relative_residual[c] = t.rel[c];
    report->history_len = 0;
    if (report->history)
      for (double v : t.history) {
        if (report->history_len >= report->history_capacity) break;
        report->history[report->history_len++] = v;
      }
    report->converged = converged ? 1 : 0;
    report->batches = t.batches;
    report->retried_columns = t.retried;
    report->zero_rhs_columns = static_cast<int>(t.dead.size());
    report->steps = t.steps;
    report->levels = h->nlev;
    report->coarsest_dofs = hy.n_live;
    report->setup_s = hy.setup_reported ? 0.0 : hy.setup_s;
    for (int l = 0; l < 16; ++l) report->lambda_max[l] = (l + 1 < h->nlev) ? hy.lv[l].lambda_max : 0.0;
    report->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  hy.setup_reported = true;
}

int solve_impl(tf_handle* h, uint64_t key, const double* f_dev, int32_t nrhs, double* u_dev, tf_report* report, void* stream,
               bool warm) {
  return guard(h, [&] {
    auto t0 = std::chrono::steady_clock::now();
    require(nrhs >= 0, "nrhs must be non-negative");
    require(nrhs == 0 || (f_dev && u_dev), "forces and solution must not be NULL");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Hierarchy& hy = get_hierarchy(h, key, s);
    SolveTally t;
    split_columns(h, f_dev, nrhs, u_dev, s, t.live, t.dead);
    t.iters.assign(nrhs, 0);
    t.rel.assign(nrhs, 0.0);
    const int chunk = h->s.batch > 0 ? h->s.batch : std::max<int>(1, static_cast<int>(t.live.size()));
    for (size_t start = 0; start < t.live.size(); start += chunk) {
      const int nc = static_cast<int>(std::min<size_t>(chunk, t.live.size() - start));
      std::vector<int> cols(t.live.begin() + start, t.live.begin() + start + nc);
      load_columns(h, hy, f_dev, u_dev, cols, warm, s);
      std::vector<int> run(nc, 1);
      PcgResult r = work_is_double(h) ? pcg<double, double>(h, hy, nc, run, warm, s)
                    : (h->s.pcg_precision == TF_PRECISION_FLOAT32 ? pcg<float, float>(h, hy, nc, run, warm, s)
                                                                  : pcg<float, double>(h, hy, nc, run, warm, s));
      t.history.insert(t.history.end(), r.history.begin(), r.history.end());
      t.steps += r.steps;
      retry_columns(h, hy, nc, r, t.history, t.steps, t.retried, s);
      store_columns(h, u_dev, cols, r, t.iters, t.rel, s);
      ++t.batches;
    }
    TF_CUDA_CHECK(cudaStreamSynchronize(s));
    check_tensor_core_error(h, s);
    fill_solve_report(h, hy, report, nrhs, t, t0);
  });
}

#include "tf_solve_batch.cuh"

// tf_solve_batch: the instances' set-up (hierarchies, zero columns, the padded right-hand sides) one
// by one, their PCG runs in lockstep (pcg_batch), then each instance's retries and results as in
// tf_solve.
template <typename T>
void solve_batch_run(tf_handle* const* hs, const uint64_t* keys, int count, const double* const* f_dev, const int32_t* nrhs,
                     double* const* u_dev, tf_report* reports, cudaStream_t s) {
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<BatchSolve> inst(count);
  std::vector<SolveTally> tally(count);
  Group all;
  for (int i = 0; i < count; ++i) {
    tf_handle* h = hs[i];
    BatchSolve& b = inst[i];
    b.h = h;
    b.hy = &get_hierarchy(h, keys[i], s);
    SolveTally& t = tally[i];
    split_columns(h, f_dev[i], nrhs[i], u_dev[i], s, t.live, t.dead);
    t.iters.assign(nrhs[i], 0);
    t.rel.assign(nrhs[i], 0.0);
    b.ncol = static_cast<int>(t.live.size());
    if (b.ncol == 0) continue;
    require(h->s.batch <= 0 || h->s.batch >= b.ncol, "tf_solve_batch runs each instance's live columns as one block: "
                                                      "settings.batch must be 0 or at least the live column count");
    load_columns(h, *b.hy, f_dev[i], u_dev[i], t.live, false, s);
    b.run.assign(b.ncol, 1);
    all.push_back(&b);
  }
  if (!all.empty()) pcg_batch<T>(all, s);
  for (int i = 0; i < count; ++i) {
    BatchSolve& b = inst[i];
    SolveTally& t = tally[i];
    if (b.ncol > 0) {
      PcgResult& r = b.res;
      t.history.insert(t.history.end(), r.history.begin(), r.history.end());
      t.steps += r.steps;
      retry_columns(b.h, *b.hy, b.ncol, r, t.history, t.steps, t.retried, s);
      store_columns(b.h, u_dev[i], t.live, r, t.iters, t.rel, s);
      t.batches = 1;
    }
  }
  TF_CUDA_CHECK(cudaStreamSynchronize(s));
  for (int i = 0; i < count; ++i)
    fill_solve_report(inst[i].h, *inst[i].hy, reports ? &reports[i] : nullptr, nrhs[i], tally[i], t0);
}

int solve_batch_impl(tf_handle* const* hs, const uint64_t* keys, int32_t count, const double* const* f_dev, const int32_t* nrhs,
                     double* const* u_dev, tf_report* reports, void* stream) {
  std::string where = "tf_solve_batch: ";
  try {
    require(count >= 1, "count must be positive");
    require(hs && keys && f_dev && nrhs && u_dev, "handles, keys, forces, column counts and solutions must not be NULL");
    for (int i = 0; i < count; ++i) require(hs[i] != nullptr, "handle " + std::to_string(i) + " is NULL");
    const tf_settings& s0 = hs[0]->s;
    for (int i = 0; i < count; ++i) {
      for (int j = 0; j < i; ++j) require(hs[j] != hs[i], "each instance needs its own handle (handles " + std::to_string(j) + " and " +
                                                            std::to_string(i) + " are the same)");
      require(nrhs[i] >= 0, "nrhs must be non-negative");
      require(nrhs[i] == 0 || (f_dev[i] && u_dev[i]), "forces and solution must not be NULL");
      const tf_settings& si = hs[i]->s;
      require(si.pcg_precision == TF_PRECISION_FLOAT64, "tf_solve_batch runs the FP64 PCG (settings.pcg_precision float64)");
      require(!si.tensor_cores, "tf_solve_batch runs the CUDA-core finest-level operator (settings.tensor_cores 0)");
      require(si.cycle == TF_CYCLE_V, "tf_solve_batch runs V-cycles");
      require(si.precision == s0.precision && si.smoother == s0.smoother && si.sweeps == s0.sweeps &&
                  si.chebyshev_degree == s0.chebyshev_degree && si.growth == s0.growth && si.chebyshev_ratio == s0.chebyshev_ratio &&
                  si.damping == s0.damping,
              "the instances of a batch share the V-cycle settings (precision, smoother, sweeps, degree, growth, ratio, damping)");
      require(hs[i]->k0_reflect == hs[0]->k0_reflect && std::memcmp(hs[i]->ke, hs[0]->ke, sizeof(hs[0]->ke)) == 0,
              "the instances of a batch share the element stiffness ke");
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (work_is_double(hs[0])) solve_batch_run<double>(hs, keys, count, f_dev, nrhs, u_dev, reports, s);
    else solve_batch_run<float>(hs, keys, count, f_dev, nrhs, u_dev, reports, s);
    return TF_OK;
  } catch (const Error& e) {
    const std::string msg = where + e.what();
    record_unhandled_error(msg);
    for (int i = 0; hs && i < count; ++i)
      if (hs[i]) hs[i]->err = msg;
    return e.code;
  } catch (const std::exception& e) {
    const std::string msg = where + e.what();
    record_unhandled_error(msg);
    for (int i = 0; hs && i < count; ++i)
      if (hs[i]) hs[i]->err = msg;
    return TF_INTERNAL;
  }
}
}  // namespace

extern "C" int tf_solve(tf_handle* h, uint64_t key, const double* f_dev, int32_t nrhs, double* u_dev, tf_report* report,
                        void* stream) {
  if (!h) return TF_INVALID;
  return solve_impl(h, key, f_dev, nrhs, u_dev, report, stream, false);
}

extern "C" int tf_solve_batch(tf_handle* const* handles, const uint64_t* keys, int32_t count, const double* const* f_dev,
                              const int32_t* nrhs, double* const* u_dev, tf_report* reports, void* stream) {
  return solve_batch_impl(handles, keys, count, f_dev, nrhs, u_dev, reports, stream);
}

extern "C" int tf_solve_guess(tf_handle* h, uint64_t key, const double* f_dev, int32_t nrhs, double* u_dev, tf_report* report,
                              void* stream) {
  if (!h) return TF_INVALID;
  return solve_impl(h, key, f_dev, nrhs, u_dev, report, stream, true);
}

namespace {
void fill_level_report(tf_handle* h, Hierarchy& hy, tf_report* report) {
  if (!report) return;
  report->levels = h->nlev;
  report->coarsest_dofs = hy.n_live;
  report->setup_s = hy.setup_reported ? 0.0 : hy.setup_s;
  for (int l = 0; l < 16; ++l) report->lambda_max[l] = (l + 1 < h->nlev) ? hy.lv[l].lambda_max : 0.0;
}
}  // namespace

extern "C" int tf_prepare(tf_handle* h, uint64_t key, tf_report* report, void* stream) {
  if (!h) return TF_INVALID;
  return guard(h, [&] {
    Hierarchy& hy = get_hierarchy(h, key, static_cast<cudaStream_t>(stream));
    fill_level_report(h, hy, report);
    hy.setup_reported = true;
  });
}

extern "C" int tf_precondition(tf_handle* h, uint64_t key, const double* r_dev, int32_t nrhs, double* z_dev, void* stream) {
  if (!h) return TF_INVALID;
  return guard(h, [&] {
    require(nrhs >= 0 && (nrhs == 0 || (r_dev && z_dev)), "invalid preconditioner arguments");
    if (nrhs == 0) return;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Hierarchy& hy = get_hierarchy(h, key, s);
    const long long nun = 3 * h->un.nnode;
    ensure_pcg(h, nrhs);
    ensure_coarse_work(h, hy, nrhs);
    PcgState st = pcg_state(h, nrhs);
    std::vector<int> ones(nrhs, 1);
    TF_CUDA_CHECK(cudaMemcpyAsync(st.active, ones.data(), sizeof(int) * nrhs, cudaMemcpyHostToDevice, s));
    pad_kernel<<<cols_grid(h->geo[0].nnode, nrhs), 256, 0, s>>>(r_dev, nun, h->un, h->geo[0], nullptr, h->vr.as<double>(), nullptr);
    TF_LAUNCH_CHECK("pad_kernel");
    if (work_is_double(h)) {
      ensure_vbufs<double>(h, nrhs);
      precondition<double, double>(h, hy, nrhs, st, 1, true, s, true);
    } else {
      ensure_vbufs<float>(h, nrhs);
      precondition<float, double>(h, hy, nrhs, st, 1, true, s, true);
    }
    unpad_kernel<<<cols_grid(h->un.nnode, nrhs), 256, 0, s>>>(h->vz.as<double>(), h->un, h->geo[0], z_dev, nun, nullptr);
    TF_LAUNCH_CHECK("unpad_kernel");
    TF_CUDA_CHECK(cudaStreamSynchronize(s));
    check_tensor_core_error(h, s);
  });
}

extern "C" int tf_apply(tf_handle* h, uint64_t key, int32_t use_mask, const double* u_dev, int32_t nrhs, double* y_dev, void* stream) {
  if (!h) return TF_INVALID;
  return guard(h, [&] {
    require(h->have_moduli, "update(moduli) must be called before applying the operator");
    require(nrhs >= 0 && (nrhs == 0 || (u_dev && y_dev)), "invalid operator arguments");
    if (nrhs == 0) return;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!use_mask) {
      LevelArgs<double> a{};
      a.g = h->un;
      a.E = h->moduli_un.as<double>();
      a.mask = nullptr;
      a.u = u_dev;
      a.y = y_dev;
      a.colstride = 3 * h->un.nnode;
      a.ncol = nrhs;
      launch_level<double>(h, 0, a, MODE_APPLY, s);
      return;
    }
    Hierarchy& hy = get_hierarchy(h, key, s);
    const long long nun = 3 * h->un.nnode;
    ensure_pcg(h, nrhs);
    pad_kernel<<<cols_grid(h->geo[0].nnode, nrhs), 256, 0, s>>>(u_dev, nun, h->un, h->geo[0], hy.lv[0].mask.as<uint8_t>(),
                                                                h->vb.as<double>(), nullptr);
    TF_LAUNCH_CHECK("pad_kernel");
    fine_apply64(h, hy, h->vb.as<double>(), nullptr, h->vq.as<double>(), MODE_APPLY, nrhs, nullptr, nullptr, s);
    unpad_kernel<<<cols_grid(h->un.nnode, nrhs), 256, 0, s>>>(h->vq.as<double>(), h->un, h->geo[0], y_dev, nun, nullptr);
    TF_LAUNCH_CHECK("unpad_kernel");
  });
}

extern "C" int tf_apply_level(tf_handle* h, uint64_t key, int32_t level, const double* u_dev, int32_t nrhs, double* y_dev,
                              void* stream) {
  if (!h) return TF_INVALID;
  return guard(h, [&] {
    require(nrhs >= 0 && (nrhs == 0 || (u_dev && y_dev)), "invalid operator arguments");
    require(level >= 0 && level < h->nlev, "level out of range");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Hierarchy& hy = get_hierarchy(h, key, s);
    if (nrhs == 0) return;
    LevelArgs<double> a = level_args<double>(h, hy, level, nrhs, nullptr);
    a.E = level_E<double>(h, hy, level, true);
    a.u = u_dev;
    a.y = y_dev;
    launch_level<double>(h, level, a, MODE_APPLY, s);
  });
}

namespace {
// y = mask * (sum_e mass_e M0 u_e + lumped * u) on the padded finest grid, u already masked; one thread
// per (node, column), 8 elements x 8 corners x 9 FMA per node in a fixed order (deterministic).
__global__ void mass_node_kernel(const __grid_constant__ K0Param<double> M, Geo g, const double* __restrict__ mass,
                                 const double* __restrict__ lumped, const uint8_t* __restrict__ mask,
                                 const double* __restrict__ u, long long colstride, double* __restrict__ y) {
  const int col = blockIdx.y;
  const double* uc = u + (long long)col * colstride;
  double* yc = y + (long long)col * colstride;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < g.nnode; n += (long long)gridDim.x * blockDim.x) {
    const int k = static_cast<int>(n % g.nz);
    const long long r = n / g.nz;
    const int j = static_cast<int>(r % g.ny), i = static_cast<int>(r / g.ny);
    double acc[3] = {0.0, 0.0, 0.0};
    for (int e = 0; e < 8; ++e) {
      const int ox = e >> 2, oy = (e >> 1) & 1, oz = e & 1;
      const int ei = i - 1 + ox, ej = j - 1 + oy, ek = k - 1 + oz;
      if (!((unsigned)ei < (unsigned)g.ex && (unsigned)ej < (unsigned)g.ey && (unsigned)ek < (unsigned)g.ez)) continue;
      const double me = mass[((long long)ei * g.ey + ej) * g.ez + ek];
      if (me == 0.0) continue;
      const int cn = corner_id(1 - ox, 1 - oy, 1 - oz);
      for (int cm = 0; cm < 8; ++cm) {
        const long long nm = ((long long)(ei + corner_x(cm)) * g.ny + (ej + corner_y(cm))) * g.nz + (ek + corner_z(cm));
        const double u0 = uc[3 * nm], u1 = uc[3 * nm + 1], u2 = uc[3 * nm + 2];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const double* row = M.k + (3 * cn + q) * 24 + 3 * cm;
          acc[q] = fma(me, fma(row[2], u2, fma(row[1], u1, row[0] * u0)), acc[q]);
        }
      }
    }
    const unsigned m = mask ? mask[n] : 7u;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const double l = lumped ? lumped[3 * n + q] * uc[3 * n + q] : 0.0;
      yc[3 * n + q] = ((m >> q) & 1u) ? acc[q] + l : 0.0;
    }
  }
}
}  // namespace

extern "C" int tf_mass_apply(tf_handle* h, uint64_t key, const double* mass_dev, const double* lumped_dev, const double* u_dev,
                             int32_t nrhs, double* y_dev, void* stream) {
  if (!h) return TF_INVALID;
  return guard(h, [&] {
    require(h->have_me, "the handle was created without an element mass matrix");
    require(mass_dev != nullptr, "element masses must not be NULL");
    require(nrhs >= 0 && (nrhs == 0 || (u_dev && y_dev)), "invalid mass operator arguments");
    require(h->have_moduli, "update(moduli) must be called before the mass operator (it uses the hierarchy mask)");
    if (nrhs == 0) return;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Hierarchy& hy = get_hierarchy(h, key, s);
    const Geo& pd = h->geo[0];
    const long long nun = 3 * h->un.nnode;
    h->mass64.ensure(sizeof(double) * (size_t)pd.ex * pd.ey * pd.ez);
    pad_moduli_kernel<<<grid_for((long long)pd.ex * pd.ey * pd.ez, 256), 256, 0, s>>>(h->un, pd, mass_dev, h->mass64.as<double>(), nullptr);
    TF_LAUNCH_CHECK("pad_moduli_kernel");
    if (lumped_dev) {
      h->lumped64.ensure(sizeof(double) * 3 * pd.nnode);
      pad_kernel<<<cols_grid(pd.nnode, 1), 256, 0, s>>>(lumped_dev, nun, h->un, pd, nullptr, h->lumped64.as<double>(), nullptr);
      TF_LAUNCH_CHECK("pad_kernel");
    }
    ensure_pcg(h, nrhs);
    pad_kernel<<<cols_grid(pd.nnode, nrhs), 256, 0, s>>>(u_dev, nun, h->un, pd, hy.lv[0].mask.as<uint8_t>(), h->vb.as<double>(), nullptr);
    TF_LAUNCH_CHECK("pad_kernel");
    mass_node_kernel<<<cols_grid(pd.nnode, nrhs), 256, 0, s>>>(h->m64, pd, h->mass64.as<double>(), lumped_dev ? h->lumped64.as<double>() : nullptr,
                                                               hy.lv[0].mask.as<uint8_t>(), h->vb.as<double>(), 3 * pd.nnode, h->vq.as<double>());
    TF_LAUNCH_CHECK("mass_node_kernel");
    unpad_kernel<<<cols_grid(h->un.nnode, nrhs), 256, 0, s>>>(h->vq.as<double>(), h->un, pd, y_dev, nun, nullptr);
    TF_LAUNCH_CHECK("unpad_kernel");
  });
}

extern "C" int tf_element_energy(tf_handle* h, const double* u_dev, int32_t nrhs, const double* comb_dev, int32_t ncomb,
                                 const double* coef_dev, const double* scale_dev, double* out_dev, int32_t accumulate,
                                 int32_t per_column, void* stream) {
  if (!h) return TF_INVALID;
  return guard(h, [&] {
    require(nrhs >= 0 && (nrhs == 0 || (u_dev && out_dev)), "invalid energy arguments");
    require(!comb_dev || ncomb >= 1, "ncomb must be positive with a combination matrix");
    require(!(per_column && comb_dev), "per_column energies take no combination matrix");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long ne = (long long)h->un.ex * h->un.ey * h->un.ez;
    {
  TimedRange tr_(h->timers, TIMER_ENERGY, s);
  energy_kernel<double><<<grid_for(ne, 128, 148 * 16), 128, 0, s>>>(h->k64, h->un, u_dev, 3 * h->un.nnode, nrhs, comb_dev,
                                                                        comb_dev ? ncomb : nrhs, coef_dev, scale_dev, out_dev,
                                                                        accumulate, per_column);
    TF_LAUNCH_CHECK("energy_kernel");
  }
  });
}

extern "C" int tf_timers(tf_handle* h, int32_t enable, double* ms, int64_t* counts, int32_t nclasses) {
  if (!h) return TF_INVALID;
  return guard(h, [&] {
    require(nclasses >= 0 && (nclasses == 0 || (ms && counts)), "invalid timer buffers");
    if (nclasses > 0) {
      for (int c = 0; c < nclasses; ++c) { ms[c] = 0.0; counts[c] = 0; }
      for (size_t q = 0; q < h->timers.used; ++q) {
        auto& e = h->timers.pool[q];
        TF_CUDA_CHECK(cudaEventSynchronize(e.second));
        float t = 0.f;
        TF_CUDA_CHECK(cudaEventElapsedTime(&t, e.first, e.second));
        const int c = h->timers.cls[q];
        if (c < nclasses) { ms[c] += t; counts[c] += 1; }
      }
    }
    h->timers.used = 0;
    h->timers.enabled = enable != 0;
  });
}

extern "C" int tf_destroy(tf_handle* h) {
  if (!h) return TF_OK;
  // an error the device reports here (from earlier work) is returned, and the handle is freed regardless
  const cudaError_t e = cudaDeviceSynchronize();
  delete h;
  if (e != cudaSuccess) {
    g_last_create_error = std::string("tf_destroy: ") + cudaGetErrorString(e);
    return TF_CUDA;
  }
  return TF_OK;
}

extern "C" const char* tf_last_error(const tf_handle* h) {
  if (!h) return g_last_create_error.c_str();
  return h->err.c_str();
}
