// tf_solve_batch: tf_solve over several independent instances (their own grids, hierarchies and
// load columns) with every PCG and V-cycle stage one launch for all of them.
//
// Each instance keeps its handle's buffers, hierarchy and PCG state; a stage builds one record per
// instance (the arguments its own launch would get) and runs the shared kernel body over the
// concatenated grids (tf_batch.cuh).  Instances whose hierarchies are shallower skip the deeper
// levels' stages; each coarsest solve runs in the one coarsest stage after the down-sweep.  The
// columns of every instance converge on their own true residuals exactly as in tf_solve
// (topology_multigrid.py:407-454); an instance leaves the batched loop when its last column has.
//
// Included by tf_solver.cu inside its anonymous namespace: it uses the handle internals.

// ------------------------------------------------------------ records ------

template <typename T>
struct LevelRec {
  LevelArgs<T> a;
  int mode;
  TileMap tm;
  int cpb;
};

template <typename T, int SLOT, bool REFLECT, int TZ, int NPT, int RND, bool PCG>
__global__ void __launch_bounds__(FTXT * TY * TZ, 2) fine_level_batch(const __grid_constant__ Batch<LevelRec<T>> b) {
  VGrid vg;
  const LevelRec<T>& r = b.rec[batch_locate(b, vg)];
  fine_level_body<T, SLOT, REFLECT, TZ, NPT, RND, PCG>(vg, r.a, r.mode, r.tm, r.cpb);
}

template <typename T, int CB, int RND>
__global__ void __launch_bounds__(TX * TY * TZMAX) stencil_level_batch(const __grid_constant__ Batch<LevelRec<T>> b) {
  VGrid vg;
  const LevelRec<T>& r = b.rec[batch_locate(b, vg)];
  stencil_level_body<T, CB, RND>(vg, r.a, r.mode, r.tm);
}

template <typename T>
struct ColsRec {
  T* v;
  long long stride;
  const int* active;
};
template <typename T>
__global__ void zero_cols_batch(const __grid_constant__ Batch<ColsRec<T>> b) {
  VGrid vg;
  const ColsRec<T>& r = b.rec[batch_locate(b, vg)];
  zero_cols_body<T>(vg, r.v, r.stride, r.active);
}

template <typename T>
struct JacobiFirstRec {
  long long ndof;
  const T* inv;
  const T* b;
  T* x;
  T s;
  const int* active;
  int round;
};
template <typename T>
__global__ void jacobi_first_batch(const __grid_constant__ Batch<JacobiFirstRec<T>> b) {
  VGrid vg;
  const JacobiFirstRec<T>& r = b.rec[batch_locate(b, vg)];
  jacobi_first_body<T>(vg, r.ndof, r.inv, r.b, r.x, r.s, r.active, r.round);
}

template <typename T>
struct ChebFirstRec {
  long long ndof;
  const T* inv;
  const T* b;
  T* res;
  T* d;
  T* x;
  T inv_theta;
  int has_x, write_rd;
  const int* active;
  int round;
};
template <typename T>
__global__ void cheb_first_batch(const __grid_constant__ Batch<ChebFirstRec<T>> b) {
  VGrid vg;
  const ChebFirstRec<T>& r = b.rec[batch_locate(b, vg)];
  cheb_first_body<T>(vg, r.ndof, r.inv, r.b, r.res, r.d, r.x, r.inv_theta, r.has_x, r.write_rd, r.active, r.round);
}

// restriction (src = fine residual, dst = coarse right-hand side, mask = coarse) and
// prolongation (src = coarse correction, dst = fine iterate, mask = fine)
template <typename T>
struct TransferRec {
  Geo fine, coarse;
  const T* src;
  long long sstride;
  T* dst;
  long long dstride;
  const uint8_t* mask;
  const int* active;
  int round;
};
template <typename T>
__global__ void restrict_batch(const __grid_constant__ Batch<TransferRec<T>> b) {
  VGrid vg;
  const TransferRec<T>& r = b.rec[batch_locate(b, vg)];
  restrict_body<T>(vg, r.fine, r.coarse, r.src, r.sstride, r.dst, r.dstride, r.mask, r.active, r.round);
}
template <typename T>
__global__ void prolong_add_batch(const __grid_constant__ Batch<TransferRec<T>> b) {
  VGrid vg;
  const TransferRec<T>& r = b.rec[batch_locate(b, vg)];
  prolong_add_body<T>(vg, r.fine, r.coarse, r.src, r.sstride, r.dst, r.dstride, r.mask, r.active, r.round);
}

template <typename T>
struct GatherRec {
  const T* src;
  long long stride;
  const long long* live;
  int n;
  double* dst;
  const int* active;
};
template <typename T>
__global__ void coarsest_gather_batch(const __grid_constant__ Batch<GatherRec<T>> b) {
  VGrid vg;
  const GatherRec<T>& r = b.rec[batch_locate(b, vg)];
  coarsest_gather_body<T>(vg, r.src, r.stride, r.live, r.n, r.dst, r.active);
}

template <typename T>
struct ScatterRec {
  const double* src;
  const long long* live;
  int n;
  T* dst;
  long long stride;
  const int* active;
  int round;
};
template <typename T>
__global__ void coarsest_scatter_batch(const __grid_constant__ Batch<ScatterRec<T>> b) {
  VGrid vg;
  const ScatterRec<T>& r = b.rec[batch_locate(b, vg)];
  coarsest_scatter_body<T>(vg, r.src, r.live, r.n, r.dst, r.stride, r.active, r.round);
}

struct NormRec {
  const double* b;
  long long n;
  PcgState st;
  double* out;
  int take_sqrt;
};
__global__ void pcg_norm_batch(const __grid_constant__ Batch<NormRec> b) {
  VGrid vg;
  const NormRec& r = b.rec[batch_locate(b, vg)];
  pcg_norm_body(vg, r.b, r.n, r.st, r.out, r.take_sqrt);
}

struct TakeRec {
  const double* t;
  double* r;
  long long n;
  PcgState st;
};
__global__ void pcg_take_batch(const __grid_constant__ Batch<TakeRec> b) {
  VGrid vg;
  const TakeRec& r = b.rec[batch_locate(b, vg)];
  pcg_take_body<double>(vg, r.t, r.r, r.n, r.st);
}

template <typename T>
struct ToWorkRec {
  const double* r;
  long long n;
  PcgState st;
  T* w;
  int round;
};
template <typename T>
__global__ void pcg_to_work_batch(const __grid_constant__ Batch<ToWorkRec<T>> b) {
  VGrid vg;
  const ToWorkRec<T>& r = b.rec[batch_locate(b, vg)];
  pcg_to_work_body<T, double>(vg, r.r, r.n, r.st, r.w, r.round);
}

template <typename T>
struct FromWorkRec {
  const T* w;
  const double* r;
  long long n;
  PcgState st;
  int initial;
};
template <typename T>
__global__ void pcg_from_work_batch(const __grid_constant__ Batch<FromWorkRec<T>> b) {
  VGrid vg;
  const FromWorkRec<T>& r = b.rec[batch_locate(b, vg)];
  pcg_from_work_body<T, double>(vg, r.w, r.r, nullptr, r.n, r.st, r.initial);
}

template <typename T>
struct DirectionRec {
  const T* w;
  double* p;
  long long n;
  PcgState st;
  int initial;
};
template <typename T>
__global__ void pcg_direction_batch(const __grid_constant__ Batch<DirectionRec<T>> b) {
  VGrid vg;
  const DirectionRec<T>& r = b.rec[batch_locate(b, vg)];
  pcg_direction_body<T, double>(vg, r.w, r.p, r.n, r.st, r.initial);
}

struct AlphaSumRec {
  const double* part;
  long long per_col;
  PcgState st;
};
__global__ void pcg_alpha_sum_batch(const __grid_constant__ Batch<AlphaSumRec> b) {
  VGrid vg;
  const AlphaSumRec& r = b.rec[batch_locate(b, vg)];
  pcg_alpha_sum_body(vg, r.part, r.per_col, r.st);
}

template <typename T>
struct UpdateRec {
  double* x;
  double* r;
  const double* p;
  const double* q;
  const T* w;
  long long n;
  PcgState st;
  double tol;
  int step;
};
template <typename T>
__global__ void pcg_update_batch(const __grid_constant__ Batch<UpdateRec<T>> b) {
  VGrid vg;
  const UpdateRec<T>& r = b.rec[batch_locate(b, vg)];
  pcg_update_body<T, double>(vg, r.x, r.r, r.p, r.q, r.w, r.n, r.st, r.tol, r.step, 0.0);
}

struct TruecheckRec {
  const double* t;
  long long n;
  PcgState st;
  double tol;
  int step;
};
__global__ void pcg_truecheck_batch(const __grid_constant__ Batch<TruecheckRec> b) {
  VGrid vg;
  const TruecheckRec& r = b.rec[batch_locate(b, vg)];
  pcg_truecheck_body(vg, r.t, r.n, r.st, r.tol, r.step);
}

template <typename T>
struct RetireRec {
  const double* t;
  double* r;
  const T* w;
  long long n;
  PcgState st;
};
template <typename T>
__global__ void pcg_retire_batch(const __grid_constant__ Batch<RetireRec<T>> b) {
  VGrid vg;
  const RetireRec<T>& r = b.rec[batch_locate(b, vg)];
  pcg_retire_body<T, double>(vg, r.t, r.r, r.w, r.n, r.st);
}

struct FlagsRec {
  PcgState st;
  int step;
};
__global__ void pcg_flags_batch(const __grid_constant__ Batch<FlagsRec> b) {
  VGrid vg;
  const FlagsRec& r = b.rec[batch_locate(b, vg)];
  pcg_flags_body(vg, r.st, r.step);
}

// ------------------------------------------------------------ instances ----

struct BatchSolve {
  tf_handle* h = nullptr;
  Hierarchy* hy = nullptr;
  int ncol = 0;             // live columns, solved as one block
  std::vector<int> run;     // all ones
  PcgState st{};
  int steps = 0;
  bool running = false;     // still iterating when the batched loop stopped
  double rho = 0.0;         // Chebyshev recurrence of the current smoothing pass
  int tz = 8;               // node-tile height of the batch's finest-level launches (batch_tz)
  PcgResult res;
  long long n() const { return 3 * h->geo[0].nnode; }
};
using Group = std::vector<BatchSolve*>;

template <class Rec, class F>
std::vector<std::pair<dim3, Rec>> records(const Group& in, F&& make) {
  std::vector<std::pair<dim3, Rec>> items;
  items.reserve(in.size());
  for (BatchSolve* b : in) items.push_back(make(*b));
  return items;
}

dim3 red_grid(const BatchSolve& b) { return dim3(grid_for(b.n(), RED_THREADS, PCG_BLOCKS), b.ncol); }

// ------------------------------------------------------- level applies -----

// One tile height for every instance of a batched finest-level launch: 9-high tiles when they pad
// at least 15 % fewer threads along z over the whole batch (weighted by nodes and columns), as
// launch_fine decides for one grid.
int batch_tz(const Group& in) {
  if (in.empty() || !in[0]->h->k0_reflect) return 8;
  double pad8 = 0.0, pad9 = 0.0;
  for (const BatchSolve* b : in) {
    const Geo& g = b->h->geo[0];
    const double plane = (double)g.nx * g.ny * b->ncol;
    pad8 += plane * (((g.nz + 7) / 8) * 8);
    pad9 += plane * (((g.nz + 8) / 9) * 9);
  }
  return 100.0 * pad9 < 85.0 * pad8 ? 9 : 8;
}

template <typename T, int SLOT, bool REFLECT, int TZ, int RND, bool PCG>
void fine_batch_variant(const std::vector<LevelArgs<T>>& as, int mode, cudaStream_t st) {
  constexpr int NPT = (sizeof(T) == 4 && REFLECT) ? 2 : 1;
  constexpr size_t smem = fine_smem_bytes<T, TZ, NPT>();
  static bool configured = false;   // per variant and process; the attribute is per function
  if (!configured) {
    TF_CUDA_CHECK(cudaFuncSetAttribute(fine_level_batch<T, SLOT, REFLECT, TZ, NPT, RND, PCG>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured = true;
  }
  std::vector<std::pair<dim3, LevelRec<T>>> items;
  for (const LevelArgs<T>& a : as) {
    LevelRec<T> r{a, mode, TileMap{}, 1};
    const dim3 grid = fine_shape<TZ, NPT>(a.g, a.ncol, r.tm, r.cpb);
    items.push_back({grid, r});
  }
  launch_batched<LevelRec<T>>(fine_level_batch<T, SLOT, REFLECT, TZ, NPT, RND, PCG>, items, dim3(TZ, TY, FTXT), smem, st,
                              "fine_level_batch");
}

// The instances of a batch share the element matrix (one constant-memory slot), its symmetry and
// the storage rounding: checked when the batch starts.
template <typename T, bool PCG>
void fine_batch(tf_handle* h0, int tz, const std::vector<LevelArgs<T>>& as, int mode, cudaStream_t st) {
  if (as.empty()) return;
  const int slot = k0_slot(h0);
  const int rnd = std::is_same<T, float>::value ? as[0].round : 0;
  auto go = [&](auto slot_c, auto reflect_c, auto tz_c) {
    constexpr int S = decltype(slot_c)::value;
    constexpr bool RF = decltype(reflect_c)::value;
    constexpr int TZ = decltype(tz_c)::value;
    if constexpr (std::is_same<T, float>::value && !PCG) {
      if (rnd == 1) { fine_batch_variant<T, S, RF, TZ, 1, PCG>(as, mode, st); return; }
      if (rnd == 2) { fine_batch_variant<T, S, RF, TZ, 2, PCG>(as, mode, st); return; }
    }
    fine_batch_variant<T, S, RF, TZ, 0, PCG>(as, mode, st);
  };
  using I0 = std::integral_constant<int, 0>;
  using I1 = std::integral_constant<int, 1>;
  using Z8 = std::integral_constant<int, 8>;
  using Z9 = std::integral_constant<int, 9>;
  using BT = std::integral_constant<bool, true>;
  using BF = std::integral_constant<bool, false>;
  if (h0->k0_reflect) {
    if (tz == 9) {
      if (slot == 0) go(I0{}, BT{}, Z9{});
      else go(I1{}, BT{}, Z9{});
    } else {
      if (slot == 0) go(I0{}, BT{}, Z8{});
      else go(I1{}, BT{}, Z8{});
    }
  } else {
    if (slot == 0) go(I0{}, BF{}, Z8{});
    else go(I1{}, BF{}, Z8{});
  }
}

template <typename T>
void stencil_batch(const std::vector<LevelArgs<T>>& as, int mode, cudaStream_t st) {
  if (as.empty()) return;
  constexpr int cb = sizeof(T) == 4 ? CB32 : CB64;
  constexpr size_t smem = stencil_smem_bytes<T, cb>();
  auto launch = [&](auto rnd) {
    constexpr int RND = decltype(rnd)::value;
    static bool configured = false;
    if (!configured) {
      TF_CUDA_CHECK(cudaFuncSetAttribute(stencil_level_batch<T, cb, RND>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      configured = true;
    }
    std::vector<std::pair<dim3, LevelRec<T>>> items;
    for (const LevelArgs<T>& a : as) {
      const TileMap tm = tile_map(a.g);
      const unsigned tiles = (unsigned)(tm.tiles_x * tm.tiles_y * tm.tiles_z);
      items.push_back({dim3(tiles, (a.ncol + cb - 1) / cb), LevelRec<T>{a, mode, tm, 0}});
    }
    // blocks sized for the tallest tile; shorter tiles leave their extra threads idle
    launch_batched<LevelRec<T>>(stencil_level_batch<T, cb, RND>, items, dim3(TX * TY * TZMAX), smem, st, "stencil_level_batch");
  };
  const int rnd = std::is_same<T, float>::value ? as[0].round : 0;
  if (rnd == 1) launch(std::integral_constant<int, 1>{});
  else if (rnd == 2) launch(std::integral_constant<int, 2>{});
  else launch(std::integral_constant<int, 0>{});
}

// One level apply for every instance of `in` on level l (the finest-level operator or the
// Galerkin stencils); `set` fills the mode's vectors and scalars.
template <typename T, class F>
void level_batch(const Group& in, int l, int mode, cudaStream_t s, F&& set) {
  if (in.empty()) return;
  std::vector<LevelArgs<T>> as;
  for (BatchSolve* b : in) {
    LevelArgs<T> a = level_args<T>(b->h, *b->hy, l, b->ncol, b->st.active);
    set(*b, a);
    as.push_back(a);
  }
  if (l == 0) fine_batch<T, false>(in[0]->h, in[0]->tz, as, mode, s);
  else stencil_batch<T>(as, mode, s);
}

// ------------------------------------------------------------ V-cycle ------

template <typename T>
void smooth_batch(const Group& in, int l, bool first, cudaStream_t s) {
  if (in.empty()) return;
  const tf_settings& set = in[0]->h->s;
  const bool jacobi = set.smoother == TF_SMOOTHER_JACOBI;
  const int base = jacobi ? set.sweeps : set.chebyshev_degree;
  const int count = std::max(1, (int)std::lround(base * std::pow(set.growth, l)));
  auto vb = [](BatchSolve& b) -> VBufs<T>& { return vbufs<T>(b.h); };
  auto nd = [l](BatchSolve& b) { return 3 * b.h->geo[l].nnode; };
  if (jacobi) {
    auto step = [l, &set](BatchSolve& b) { return static_cast<T>(set.damping / b.hy->lv[l].lambda_max); };
    int start = 0;
    if (first) {
      launch_batched<JacobiFirstRec<T>>(jacobi_first_batch<T>, records<JacobiFirstRec<T>>(in, [&](BatchSolve& b) {
        return std::make_pair(cols_grid(nd(b), b.ncol), JacobiFirstRec<T>{nd(b), level_inv<T>(*b.hy, l), vb(b).b[l].template as<T>(),
                                                                           vb(b).x[l].template as<T>(), step(b), b.st.active,
                                                                           store_round(b.h)});
      }), dim3(256), 0, s, "jacobi_first_batch");
      start = 1;
    }
    for (int k = start; k < count; ++k) {
      level_batch<T>(in, l, MODE_JACOBI, s, [&](BatchSolve& b, LevelArgs<T>& a) {
        a.u = vb(b).x[l].template as<T>();
        a.b = vb(b).b[l].template as<T>();
        a.y = vb(b).xa[l].template as<T>();
        a.s = step(b);
      });
      for (BatchSolve* b : in) std::swap(vb(*b).x[l], vb(*b).xa[l]);
    }
    return;
  }
  struct Cheb {
    double theta, delta, sigma;
  };
  auto cheb = [l, &set](BatchSolve& b) {
    const double upper = 1.1 * b.hy->lv[l].lambda_max, lower = upper / set.chebyshev_ratio;
    Cheb c;
    c.theta = 0.5 * (upper + lower);
    c.delta = 0.5 * (upper - lower);
    c.sigma = c.theta / c.delta;
    return c;
  };
  if (!first) {
    level_batch<T>(in, l, MODE_RESID, s, [&](BatchSolve& b, LevelArgs<T>& a) {
      a.u = vb(b).x[l].template as<T>();
      a.b = vb(b).b[l].template as<T>();
      a.y = vb(b).res[l].template as<T>();
    });
  }
  launch_batched<ChebFirstRec<T>>(cheb_first_batch<T>, records<ChebFirstRec<T>>(in, [&](BatchSolve& b) {
    b.rho = 1.0 / cheb(b).sigma;
    return std::make_pair(cols_grid(nd(b), b.ncol),
                          ChebFirstRec<T>{nd(b), level_inv<T>(*b.hy, l), vb(b).b[l].template as<T>(), vb(b).res[l].template as<T>(),
                                          vb(b).d[l].template as<T>(), vb(b).x[l].template as<T>(), static_cast<T>(1.0 / cheb(b).theta),
                                          first ? 0 : 1, count > 1 ? 1 : 0, b.st.active, store_round(b.h)});
  }), dim3(256), 0, s, "cheb_first_batch");
  for (int k = 1; k < count; ++k) {
    level_batch<T>(in, l, MODE_CHEB, s, [&](BatchSolve& b, LevelArgs<T>& a) {
      const Cheb c = cheb(b);
      const double rn = 1.0 / (2.0 * c.sigma - b.rho);
      a.u = vb(b).d[l].template as<T>();
      a.res = vb(b).res[l].template as<T>();
      a.x = vb(b).x[l].template as<T>();
      a.y = vb(b).da[l].template as<T>();
      a.c1 = static_cast<T>(rn * b.rho);
      a.c2 = static_cast<T>(2.0 * rn / c.delta);
      b.rho = rn;
    });
    for (BatchSolve* b : in) std::swap(vb(*b).d[l], vb(*b).da[l]);
  }
}

template <typename T>
void coarsest_batch(const Group& in, cudaStream_t s) {
  auto last = [](BatchSolve& b) { return b.h->nlev - 1; };
  auto nd = [&](BatchSolve& b) { return 3 * b.h->geo[last(b)].nnode; };
  launch_batched<ColsRec<T>>(zero_cols_batch<T>, records<ColsRec<T>>(in, [&](BatchSolve& b) {
    return std::make_pair(cols_grid(nd(b), b.ncol), ColsRec<T>{vbufs<T>(b.h).x[last(b)].template as<T>(), nd(b), b.st.active});
  }), dim3(256), 0, s, "zero_cols_batch");
  Group live;
  for (BatchSolve* b : in)
    if (b->hy->n_live > 0) live.push_back(b);
  if (live.empty()) return;
  launch_batched<GatherRec<T>>(coarsest_gather_batch<T>, records<GatherRec<T>>(live, [&](BatchSolve& b) {
    return std::make_pair(cols_grid(b.hy->n_live, b.ncol), GatherRec<T>{vbufs<T>(b.h).b[last(b)].template as<T>(), nd(b),
                                                                        b.hy->live.as<long long>(), b.hy->n_live, b.h->cb.as<double>(),
                                                                        b.st.active});
  }), dim3(256), 0, s, "coarsest_gather_batch");
  std::vector<TrimulJob> jobs;
  Group dense;
  for (BatchSolve* b : live) {
    if (b->hy->band) {   // banded coarsest factors: one substitution launch per instance
      band_solve(b->hy->X.as<double>(), b->hy->n_live, b->hy->bw, b->h->cb.as<double>(), b->h->cy.as<double>(), b->ncol, s);
      continue;
    }
    const size_t need = dense_trimul_work(b->hy->n_live, b->ncol);
    if (b->h->trimul_work.bytes < need) b->h->trimul_work.alloc(need);
    jobs.push_back(TrimulJob{b->hy->X.as<double>(), b->h->cb.as<double>(), b->h->cy.as<double>(), b->h->trimul_work.as<double>(),
                             b->hy->n_live, b->ncol, b->st.active});
    dense.push_back(b);
  }
  // x = X^T (X b) with X = L^-1: cb -> cy, then cy -> cb
  dense_trimul_batch(jobs.data(), (int)jobs.size(), 0, s);
  for (size_t i = 0; i < jobs.size(); ++i) {
    jobs[i].B = dense[i]->h->cy.as<double>();
    jobs[i].C = dense[i]->h->cb.as<double>();
  }
  dense_trimul_batch(jobs.data(), (int)jobs.size(), 1, s);
  launch_batched<ScatterRec<T>>(coarsest_scatter_batch<T>, records<ScatterRec<T>>(live, [&](BatchSolve& b) {
    const double* solved = b.hy->band ? b.h->cy.as<double>() : b.h->cb.as<double>();
    return std::make_pair(cols_grid(b.hy->n_live, b.ncol), ScatterRec<T>{solved, b.hy->live.as<long long>(), b.hy->n_live,
                                                                         vbufs<T>(b.h).x[last(b)].template as<T>(), nd(b), b.st.active,
                                                                         store_round(b.h)});
  }), dim3(256), 0, s, "coarsest_scatter_batch");
}

template <typename T>
void vcycle_batch(const Group& in, cudaStream_t s) {
  int lmax = 0;
  for (BatchSolve* b : in) lmax = std::max(lmax, b->h->nlev);
  auto above = [&](int l) {   // instances for which level l is not the coarsest
    Group g;
    for (BatchSolve* b : in)
      if (l < b->h->nlev - 1) g.push_back(b);
    return g;
  };
  auto transfer = [](BatchSolve& b, int l, bool down) {
    VBufs<T>& v = vbufs<T>(b.h);
    const Geo& fg = b.h->geo[l];
    const Geo& cg = b.h->geo[l + 1];
    if (down)
      return std::make_pair(cols_grid(cg.nnode, b.ncol),
                            TransferRec<T>{fg, cg, v.res[l].template as<T>(), 3 * fg.nnode, v.b[l + 1].template as<T>(), 3 * cg.nnode,
                                           b.hy->lv[l + 1].mask.as<uint8_t>(), b.st.active, store_round(b.h)});
    return std::make_pair(cols_grid(cg.nnode, b.ncol),
                          TransferRec<T>{fg, cg, v.x[l + 1].template as<T>(), 3 * cg.nnode, v.x[l].template as<T>(), 3 * fg.nnode,
                                         b.hy->lv[l].mask.as<uint8_t>(), b.st.active, store_round(b.h)});
  };
  for (int l = 0; l + 1 < lmax; ++l) {
    const Group g = above(l);
    if (g.empty()) continue;
    smooth_batch<T>(g, l, true, s);
    level_batch<T>(g, l, MODE_RESID, s, [&](BatchSolve& b, LevelArgs<T>& a) {
      a.u = vbufs<T>(b.h).x[l].template as<T>();
      a.b = vbufs<T>(b.h).b[l].template as<T>();
      a.y = vbufs<T>(b.h).res[l].template as<T>();
    });
    launch_batched<TransferRec<T>>(restrict_batch<T>, records<TransferRec<T>>(g, [&](BatchSolve& b) { return transfer(b, l, true); }),
                                   dim3(256), 0, s, "restrict_batch");
  }
  coarsest_batch<T>(in, s);
  for (int l = lmax - 2; l >= 0; --l) {
    const Group g = above(l);
    if (g.empty()) continue;
    launch_batched<TransferRec<T>>(prolong_add_batch<T>, records<TransferRec<T>>(g, [&](BatchSolve& b) { return transfer(b, l, false); }),
                                   dim3(256), 0, s, "prolong_add_batch");
    smooth_batch<T>(g, l, false, s);
  }
}

template <typename T>
void precondition_batch(const Group& in, int initial, cudaStream_t s) {
  launch_batched<ToWorkRec<T>>(pcg_to_work_batch<T>, records<ToWorkRec<T>>(in, [&](BatchSolve& b) {
    return std::make_pair(cols_grid(b.n(), b.ncol),
                          ToWorkRec<T>{b.h->vr.as<double>(), b.n(), b.st, vbufs<T>(b.h).b[0].template as<T>(), store_round(b.h)});
  }), dim3(256), 0, s, "pcg_to_work_batch");
  vcycle_batch<T>(in, s);
  launch_batched<FromWorkRec<T>>(pcg_from_work_batch<T>, records<FromWorkRec<T>>(in, [&](BatchSolve& b) {
    return std::make_pair(red_grid(b), FromWorkRec<T>{vbufs<T>(b.h).x[0].template as<T>(), b.h->vr.as<double>(), b.n(), b.st, initial});
  }), dim3(RED_THREADS), 0, s, "pcg_from_work_batch");
  launch_batched<DirectionRec<T>>(pcg_direction_batch<T>, records<DirectionRec<T>>(in, [&](BatchSolve& b) {
    return std::make_pair(cols_grid(b.n(), b.ncol),
                          DirectionRec<T>{vbufs<T>(b.h).x[0].template as<T>(), b.h->vp.as<double>(), b.n(), b.st, initial});
  }), dim3(256), 0, s, "pcg_direction_batch");
}

// ---------------------------------------------------------------- PCG ------

// pcg<T, double> over every instance of `in` in lockstep (cold start, all columns live).
template <typename T>
void pcg_batch(const Group& in, cudaStream_t s) {
  const int TZ = batch_tz(in);   // the tile height of every batched finest-level launch
  for (BatchSolve* b : in) {
    b->tz = TZ;
    tf_handle* h = b->h;
    ensure_vbufs<T>(h, b->ncol);
    ensure_coarse_work(h, *b->hy, b->ncol);
    b->st = pcg_state(h, b->ncol);
    std::vector<int> zeros(b->ncol, 0);
    TF_CUDA_CHECK(cudaMemcpyAsync(b->st.active, b->run.data(), sizeof(int) * b->ncol, cudaMemcpyHostToDevice, s));
    TF_CUDA_CHECK(cudaMemcpyAsync(b->st.cand, zeros.data(), sizeof(int) * b->ncol, cudaMemcpyHostToDevice, s));
    TF_CUDA_CHECK(cudaMemcpyAsync(b->st.iters, zeros.data(), sizeof(int) * b->ncol, cudaMemcpyHostToDevice, s));
    TF_CUDA_CHECK(cudaMemsetAsync(b->st.flags, 0, sizeof(int) * 8, s));
    TF_CUDA_CHECK(cudaMemsetAsync(b->st.hist, 0, sizeof(unsigned long long) * h->hist_cap, s));
    const size_t need = sizeof(double) * (size_t)fine_dot_stride(h, TZ) * b->ncol;
    if (h->dotp.bytes < need) h->dotp.alloc(need);
    // the copies above read host vectors that die with this scope
    TF_CUDA_CHECK(cudaStreamSynchronize(s));
  }
  launch_batched<NormRec>(pcg_norm_batch, records<NormRec>(in, [&](BatchSolve& b) {
    return std::make_pair(red_grid(b), NormRec{b.h->vb.as<double>(), b.n(), b.st, b.st.bnorm, 1});
  }), dim3(RED_THREADS), 0, s, "pcg_norm_batch");
  launch_batched<ColsRec<double>>(zero_cols_batch<double>, records<ColsRec<double>>(in, [&](BatchSolve& b) {
    return std::make_pair(cols_grid(b.n(), b.ncol), ColsRec<double>{b.h->vx.as<double>(), b.n(), b.st.active});
  }), dim3(256), 0, s, "zero_cols_batch");
  launch_batched<TakeRec>(pcg_take_batch, records<TakeRec>(in, [&](BatchSolve& b) {
    return std::make_pair(red_grid(b), TakeRec{b.h->vb.as<double>(), b.h->vr.as<double>(), b.n(), b.st});
  }), dim3(RED_THREADS), 0, s, "pcg_take_batch");
  precondition_batch<T>(in, 1, s);
  Group act = in;
  for (BatchSolve* b : act) b->running = true;
  int step = 0;
  while (!act.empty()) {
    // q = K p with the curvature partials, then alpha = rho / (p . q)
    std::vector<LevelArgs<double>> as;
    for (BatchSolve* b : act) {
      LevelArgs<double> a{};
      a.g = b->h->geo[0];
      a.E = b->h->moduli64.as<double>();
      a.mask = b->hy->lv[0].mask.as<uint8_t>();
      a.u = b->h->vp.as<double>();
      a.y = b->h->vq.as<double>();
      a.colstride = 3 * a.g.nnode;
      a.ncol = b->ncol;
      a.active = b->st.active;
      a.dot_out = b->h->dotp.as<double>();
      as.push_back(a);
    }
    fine_batch<double, true>(act[0]->h, TZ, as, MODE_APPLY, s);
    launch_batched<AlphaSumRec>(pcg_alpha_sum_batch, records<AlphaSumRec>(act, [&](BatchSolve& b) {
      return std::make_pair(dim3(b.ncol), AlphaSumRec{b.h->dotp.as<double>(), fine_dot_stride(b.h, TZ), b.st});
    }), dim3(RED_THREADS), 0, s, "pcg_alpha_sum_batch");
    ++step;
    launch_batched<UpdateRec<T>>(pcg_update_batch<T>, records<UpdateRec<T>>(act, [&](BatchSolve& b) {
      return std::make_pair(red_grid(b), UpdateRec<T>{b.h->vx.as<double>(), b.h->vr.as<double>(), b.h->vp.as<double>(),
                                                      b.h->vq.as<double>(), vbufs<T>(b.h).x[0].template as<T>(), b.n(), b.st,
                                                      b.h->s.tolerance, step});
    }), dim3(RED_THREADS), 0, s, "pcg_update_batch");
    // true residual t = b - K x where a column is a candidate (gated per instance), into vq
    as.clear();
    for (BatchSolve* b : act) {
      LevelArgs<double> a{};
      a.g = b->h->geo[0];
      a.E = b->h->moduli64.as<double>();
      a.mask = b->hy->lv[0].mask.as<uint8_t>();
      a.u = b->h->vx.as<double>();
      a.b = b->h->vb.as<double>();
      a.y = b->h->vq.as<double>();
      a.colstride = 3 * a.g.nnode;
      a.ncol = b->ncol;
      a.active = b->st.active;
      a.gate = b->st.flags;
      as.push_back(a);
    }
    fine_batch<double, false>(act[0]->h, TZ, as, MODE_RESID, s);
    launch_batched<TruecheckRec>(pcg_truecheck_batch, records<TruecheckRec>(act, [&](BatchSolve& b) {
      return std::make_pair(red_grid(b), TruecheckRec{b.h->vq.as<double>(), b.n(), b.st, b.h->s.tolerance, step});
    }), dim3(RED_THREADS), 0, s, "pcg_truecheck_batch");
    launch_batched<RetireRec<T>>(pcg_retire_batch<T>, records<RetireRec<T>>(act, [&](BatchSolve& b) {
      return std::make_pair(red_grid(b), RetireRec<T>{b.h->vq.as<double>(), b.h->vr.as<double>(),
                                                      vbufs<T>(b.h).x[0].template as<T>(), b.n(), b.st});
    }), dim3(RED_THREADS), 0, s, "pcg_retire_batch");
    launch_batched<FlagsRec>(pcg_flags_batch, records<FlagsRec>(act, [&](BatchSolve& b) {
      return std::make_pair(dim3(1), FlagsRec{b.st, step});
    }), dim3(256), 0, s, "pcg_flags_batch");
    for (BatchSolve* b : act)
      TF_CUDA_CHECK(cudaMemcpyAsync(b->h->host_flags, b->st.flags + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    TF_CUDA_CHECK(cudaStreamSynchronize(s));
    Group next;
    for (BatchSolve* b : act) {
      b->steps = step;
      if (b->h->host_flags[0] == 0) b->running = false;
      else if (step < b->h->s.max_iterations) next.push_back(b);
    }
    act.swap(next);
    if (act.empty()) break;
    precondition_batch<T>(act, 0, s);
  }
  for (BatchSolve* b : in) b->res = pcg_finish(b->h, *b->hy, b->st, b->ncol, b->run, b->steps, b->running, s);
}
