// Batched fluid advance: many independent grids of uneven sizes advanced together.
//
// Each phase of the step (dt reduce, dt finalize, the three ghost-fill passes, the x3, x1
// and x2 sweeps, the ghost epilogue, the null-edge velocity fix and the diffusion) is ONE
// persistent launch over a work list of (instance, block) items, ordered largest instance
// first; the block bodies are the plain kernels' bodies (gem_kernels.cuh, b_*), so every
// instance computes exactly what gem_dt_calc_dev + gem_fluid_adv_dev compute for it.  The
// eleven launches of a step are captured once into a CUDA graph and replayed.
//
// Included by gem_fluid.cu (one translation unit with the plain path).

namespace gemk {

// Everything a batched block needs about its instance (device copy, one per instance).
struct InstDev {
  SweepArgs sw;  // fused-sweep arguments (grid, blocks, vs1i, dt)
  DiffArgs df;   // fused-diffusion arguments
  unsigned long long* acc;
  double tcfl;
};

// work item: instance, block x, block y, the instance's own grid x extent
using Item = int4;

template <bool UNIT>
__global__ void __launch_bounds__(32 * LSP, 4) kb_dt_reduce(const InstDev* __restrict__ inst, const Item* __restrict__ it, int n) {
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const Item q = it[w];
    const InstDev& I = inst[q.x];
    b_dt_reduce<UNIT, 0>(I.sw.G, I.sw.B, I.acc, nullptr, VB{q.y, q.z, q.w});
  }
}

__global__ void kb_zero_acc(const InstDev* inst, int ninst) {
  const int i = blockIdx.x;
  if (i < ninst && threadIdx.x < 3 * LSP) inst[i].acc[threadIdx.x] = 0ull;
}

// fixed time steps (differentiable path): instance i takes dt_in[i]
__global__ void kb_set_dt(const InstDev* inst, const double* dt_in, int ninst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ninst) *inst[i].sw.dtp_w = dt_in[i];
}

// k_dt_finalize per instance
__global__ void kb_dt_finalize(const InstDev* inst, int ninst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ninst) return;
  const InstDev& I = inst[i];
  double m = 0.0;
  for (int q = 0; q < 3 * LSP; ++q) {
    const double gr = fmax_f(__longlong_as_double((long long)I.acc[q]), 1e-10);
    const double inv = 1.0 / gr;
    if (q == 0 || inv < m) m = inv;
  }
  *I.sw.dtp_w = fmax_f(I.tcfl * m, 1e-6);
}

__global__ void __launch_bounds__(128) kb_ghost_x1(const InstDev* __restrict__ inst, const Item* __restrict__ it, int n) {
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const Item q = it[w];
    const InstDev& I = inst[q.x];
    b_ghost_x1<true>(I.sw.G, I.sw.B, I.sw.vs1i, LSP, VB{q.y, q.z, q.w});
  }
}

__global__ void __launch_bounds__(128) kb_ghost_x2(const InstDev* __restrict__ inst, const Item* __restrict__ it, int n) {
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const Item q = it[w];
    const InstDev& I = inst[q.x];
    b_ghost_x2<true>(I.sw.G, I.sw.B, LSP, VB{q.y, q.z, q.w});
  }
}

__global__ void __launch_bounds__(128) kb_ghost_x3(const InstDev* __restrict__ inst, const Item* __restrict__ it, int n) {
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const Item q = it[w];
    const InstDev& I = inst[q.x];
    if (I.sw.G.flagper)
      b_ghost_x3<true, true>(I.sw.G, I.sw.B, LSP, VB{q.y, q.z, q.w});
    else
      b_ghost_x3<true, false>(I.sw.G, I.sw.B, LSP, VB{q.y, q.z, q.w});
  }
}

template <int DIM, bool UNIT>
__global__ void __launch_bounds__(224, 2) kb_sweep_march(const InstDev* __restrict__ inst, const Item* __restrict__ it, int n) {
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const Item q = it[w];
    const InstDev& I = inst[q.x];
    b_sweep_march<DIM, UNIT, true>(I.sw, VB{q.y, q.z, q.w});
    if (DIM == 2) __syncthreads();  // the epilogue's shared buffers are reused by the next item
  }
}

template <bool UNIT>
__global__ void __launch_bounds__(224) kb_sweep_x1(const InstDev* __restrict__ inst, const Item* __restrict__ it, int n) {
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const Item q = it[w];
    const InstDev& I = inst[q.x];
    b_sweep_x1<UNIT, true>(I.sw, VB{q.y, q.z, q.w});
  }
}

__global__ void __launch_bounds__(256) kb_ghost_epilogue(const InstDev* __restrict__ inst, const Item* __restrict__ it, int n) {
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const Item q = it[w];
    const InstDev& I = inst[q.x];
    b_ghost_epilogue(I.sw.G, I.sw.B, VB{q.y, q.z, q.w});
  }
}

__global__ void __launch_bounds__(128) kb_clean_vel_edges(const InstDev* __restrict__ inst, const Item* __restrict__ it, int n) {
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const Item q = it[w];
    const InstDev& I = inst[q.x];
    b_clean_vel_edges(I.sw.G, I.sw.B.vs1(0), VB{q.y, q.z, q.w});
  }
}

// The band-solve diffusion (k_diffusion_lu) over the batch: an item is one block's worth
// (LU_WPB warp tasks) of an instance; the grid never exceeds the scratch slots, and each
// resident warp keeps the slot of its (block, warp) for every item it runs.
template <bool UNIT>
__global__ void __launch_bounds__(32 * LU_WPB, GEM_LU_MINB) kb_diffusion_lu(const InstDev* __restrict__ inst,
                                                              const Item* __restrict__ it, int n, double* lu,
                                                              long long lu_slot) {
  const int warp = threadIdx.x >> 5;
  double* slot = lu + (long long)(blockIdx.x * LU_WPB + warp) * lu_slot;
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const Item q = it[w];
    const DiffArgs& P = inst[q.x].df;
    const int ncol = P.G.d.lx2 * P.G.d.lx3;
    const int ntask = ((ncol + 31) / 32) * LSP;
    const int t = q.y * LU_WPB + warp;
    if (t < ntask) b_diffusion_lu<UNIT>(P, t, slot);
  }
}

}  // namespace gemk

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
namespace {

// One launch of the batched step: a phase, its metric variant and the work items of the
// instances it covers.
enum BatchKernel { BK_DT = 0, BK_GX1, BK_GX2, BK_GX3, BK_SW3, BK_SW1, BK_SW2, BK_EPI, BK_CVE, BK_DIFF, BK_N };

struct BatchLaunch {
  int kernel = 0;
  int unit = 0;
  int grid = 0;
  std::vector<Item> items;
  Item* d_items = nullptr;
};

}  // namespace

struct gem_batch {
  int n = 0;
  std::vector<const gem_grid*> grids;
  std::vector<gem_work*> works;
  InstDev* d_inst = nullptr;
  std::vector<BatchLaunch> launches;  // in step order
  int diff_blocks = LU_MINB_DEFAULT;  // diffusion blocks per SM (each LU_WPB warps)
  int per_sm_scale = 100;  // percent of the occupancy-limited persistent grid
  cudaStream_t cap_stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph_fixed = nullptr;  // the step with prescribed time steps
  cudaGraphExec_t exec_fixed = nullptr;
  double* d_dt_in = nullptr;  // per-instance prescribed dt (device)
  double* d_lu = nullptr;     // band-solve scratch shared by the instances' diffusion items
  long long lu_slot = 0;      // doubles per scratch slot (the longest column's)
  int use_graph = 1;
};

namespace {

void add_items(BatchLaunch& L, int idx, long long nbx, int nby = 1) {
  for (int by = 0; by < nby; ++by)
    for (long long bx = 0; bx < nbx; ++bx) L.items.push_back(make_int4(idx, (int)bx, by, (int)nbx));
}

template <class K>
int occupancy_grid(K kernel, int threads, size_t smem, size_t nitems, int scale_pct, int* out) {
  if (scale_pct == 0) {  // one block per work item: the hardware scheduler balances
    *out = (int)std::max<size_t>(1, nitems);
    return GEM_OK;
  }
  int per_sm = 0;
  GEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
  if (per_sm < 1) per_sm = 1;
  long long g = (long long)num_sms() * per_sm * scale_pct / 100;
  g = std::max<long long>(1, std::min<long long>(g, (long long)nitems));
  *out = (int)g;
  return GEM_OK;
}

int launch_grid(gem_batch* b, BatchLaunch& L) {
  const size_t n = L.items.size();
  const int sc = b->per_sm_scale;
  const bool u = L.unit != 0;
  switch (L.kernel) {
    case BK_DT: return u ? occupancy_grid(kb_dt_reduce<true>, 32 * LSP, 0, n, sc, &L.grid)
                         : occupancy_grid(kb_dt_reduce<false>, 32 * LSP, 0, n, sc, &L.grid);
    case BK_GX1: return occupancy_grid(kb_ghost_x1, 128, 0, n, sc, &L.grid);
    case BK_GX2: return occupancy_grid(kb_ghost_x2, 128, 0, n, sc, &L.grid);
    case BK_GX3: return occupancy_grid(kb_ghost_x3, 128, 0, n, sc, &L.grid);
    case BK_SW3: return u ? occupancy_grid(kb_sweep_march<3, true>, 32 * LSP, 0, n, sc, &L.grid)
                          : occupancy_grid(kb_sweep_march<3, false>, 32 * LSP, 0, n, sc, &L.grid);
    case BK_SW1: return u ? occupancy_grid(kb_sweep_x1<true>, 32 * LSP, 0, n, sc, &L.grid)
                          : occupancy_grid(kb_sweep_x1<false>, 32 * LSP, 0, n, sc, &L.grid);
    case BK_SW2: return u ? occupancy_grid(kb_sweep_march<2, true>, 32 * LSP, 0, n, sc, &L.grid)
                          : occupancy_grid(kb_sweep_march<2, false>, 32 * LSP, 0, n, sc, &L.grid);
    case BK_EPI: return occupancy_grid(kb_ghost_epilogue, 256, 0, n, sc, &L.grid);
    case BK_CVE: return occupancy_grid(kb_clean_vel_edges, 128, 0, n, sc, &L.grid);
    case BK_DIFF: {  // persistent, never more blocks than the scratch has slots for
      const long long cap = std::min<long long>((long long)num_sms() * b->diff_blocks, lu_slots() / LU_WPB);
      L.grid = (int)std::max<long long>(1, std::min<long long>((long long)n, cap));
      return GEM_OK;
    }
  }
  return set_err(GEM_EINVAL, "unknown batched kernel %d", L.kernel);
}

int batch_build_lists(gem_batch* b) {
  for (auto& L : b->launches)
    if (L.d_items) cudaFree(L.d_items);
  b->launches.clear();
  // largest instances first, so the long items start early
  std::vector<int> order(b->n);
  for (int i = 0; i < b->n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return b->grids[x]->dev.d.ng > b->grids[y]->dev.d.ng; });
  auto launch_for = [&](int kernel, int unit) -> BatchLaunch& {
    for (auto& L : b->launches)
      if (L.kernel == kernel && L.unit == unit) return L;
    BatchLaunch L;
    L.kernel = kernel;
    L.unit = unit;
    b->launches.push_back(L);
    return b->launches.back();
  };
  // create the launches in step order (variants of one phase next to each other)
  for (int k = 0; k < BK_N; ++k) {
    for (int u = 1; u >= 0; --u) {
      for (int i : order) {
        const gem_grid* g = b->grids[i];
        const Dims& d = g->dev.d;
        const bool unit = g->dev.unit != 0;
        const bool variant = (k == BK_DT || k == BK_SW3 || k == BK_SW1 || k == BK_SW2 || k == BK_DIFF);
        if (variant && unit != (u == 1)) continue;
        if (!variant && u == 0) continue;  // unsplit phases: once
        const int gx13 = (d.lx1 + 31) / 32;
        switch (k) {
          case BK_DT:
            add_items(launch_for(k, u), i, std::min<long long>((long long)d.lx2 * d.lx3, (long long)num_sms() * 8));
            break;
          case BK_GX1: add_items(launch_for(k, 0), i, grid_for((long long)(d.lx2 + 4) * (d.lx3 + 4) * LSP, 128)); break;
          case BK_GX2: add_items(launch_for(k, 0), i, grid_for((long long)(d.lx1 + 4) * (d.lx3 + 4) * LSP, 128)); break;
          case BK_GX3: add_items(launch_for(k, 0), i, grid_for((long long)(d.lx1 + 4) * (d.lx2 + 4) * LSP, 128)); break;
          case BK_SW3: add_items(launch_for(k, u), i, gx13, d.lx2); break;
          case BK_SW1: add_items(launch_for(k, u), i, d.lx2, d.lx3); break;
          case BK_SW2: add_items(launch_for(k, u), i, gx13, d.lx3); break;
          case BK_EPI: add_items(launch_for(k, 0), i, grid_for(ghost_cells(d), 256)); break;
          case BK_CVE:
            if (g->dev.has_null && (g->dev.gridflag == 0 || g->dev.gridflag == 1))
              add_items(launch_for(k, 0), i, grid_for((long long)d.lx2 * d.lx3 * LSP, 128));
            break;
          case BK_DIFF: {
            const long long ntask = (((long long)d.lx2 * d.lx3 + 31) / 32) * LSP;
            add_items(launch_for(k, u), i, (ntask + LU_WPB - 1) / LU_WPB);
            break;
          }
        }
      }
    }
  }
  for (auto& L : b->launches) {
    if (cudaMalloc(&L.d_items, L.items.size() * sizeof(Item)) != cudaSuccess)
      return set_err(GEM_ENOMEM, "cudaMalloc of a batch work list failed");
    GEM_CUDA(cudaMemcpy(L.d_items, L.items.data(), L.items.size() * sizeof(Item), cudaMemcpyHostToDevice));
    const int rc = launch_grid(b, L);
    if (rc) return rc;
  }
  return GEM_OK;
}

void batch_drop_graph(gem_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->exec_fixed) cudaGraphExecDestroy(b->exec_fixed);
  if (b->graph_fixed) cudaGraphDestroy(b->graph_fixed);
  b->exec = nullptr;
  b->graph = nullptr;
  b->exec_fixed = nullptr;
  b->graph_fixed = nullptr;
}

// fixed_dt: the instances' dt slots are loaded from d_dt_in instead of dt_calc
int batch_enqueue(gem_batch* b, cudaStream_t st, bool fixed_dt = false) {
  const InstDev* I = b->d_inst;
  if (fixed_dt)
    kb_set_dt<<<(b->n + 63) / 64, 64, 0, st>>>(I, b->d_dt_in, b->n);
  else
    kb_zero_acc<<<b->n, 32, 0, st>>>(I, b->n);
  bool finalized = fixed_dt;
  for (const auto& L : b->launches) {
    const int n = (int)L.items.size();
    const bool u = L.unit != 0;
    if (fixed_dt && L.kernel == BK_DT) continue;
    if (L.kernel != BK_DT && !finalized) {
      kb_dt_finalize<<<(b->n + 63) / 64, 64, 0, st>>>(I, b->n);
      finalized = true;
    }
    switch (L.kernel) {
      case BK_DT:
        if (u) kb_dt_reduce<true><<<L.grid, dim3(32, LSP), 0, st>>>(I, L.d_items, n);
        else kb_dt_reduce<false><<<L.grid, dim3(32, LSP), 0, st>>>(I, L.d_items, n);
        break;
      case BK_GX1: kb_ghost_x1<<<L.grid, 128, 0, st>>>(I, L.d_items, n); break;
      case BK_GX2: kb_ghost_x2<<<L.grid, 128, 0, st>>>(I, L.d_items, n); break;
      case BK_GX3: kb_ghost_x3<<<L.grid, 128, 0, st>>>(I, L.d_items, n); break;
      case BK_SW3:
        if (u) kb_sweep_march<3, true><<<L.grid, dim3(32, LSP), 0, st>>>(I, L.d_items, n);
        else kb_sweep_march<3, false><<<L.grid, dim3(32, LSP), 0, st>>>(I, L.d_items, n);
        break;
      case BK_SW1:
        if (u) kb_sweep_x1<true><<<L.grid, dim3(32, LSP), 0, st>>>(I, L.d_items, n);
        else kb_sweep_x1<false><<<L.grid, dim3(32, LSP), 0, st>>>(I, L.d_items, n);
        break;
      case BK_SW2:
        if (u) kb_sweep_march<2, true><<<L.grid, dim3(32, LSP), 0, st>>>(I, L.d_items, n);
        else kb_sweep_march<2, false><<<L.grid, dim3(32, LSP), 0, st>>>(I, L.d_items, n);
        break;
      case BK_EPI: kb_ghost_epilogue<<<L.grid, 256, 0, st>>>(I, L.d_items, n); break;
      case BK_CVE: kb_clean_vel_edges<<<L.grid, 128, 0, st>>>(I, L.d_items, n); break;
      case BK_DIFF:
        if (u) kb_diffusion_lu<true><<<L.grid, 32 * LU_WPB, 0, st>>>(I, L.d_items, n, b->d_lu, b->lu_slot);
        else kb_diffusion_lu<false><<<L.grid, 32 * LU_WPB, 0, st>>>(I, L.d_items, n, b->d_lu, b->lu_slot);
        break;
    }
  }
  GEM_LAUNCHED("batched step");
  return GEM_OK;
}

}  // namespace

extern "C" {

int gem_batch_create(int n, const gem_grid* const* grids, gem_work* const* works, double* const* fluidvars,
                     double* const* fluidauxvars, const double* const* electrovars, const gem_cfg* cfgs,
                     gem_batch** out) {
  if (!out || n < 1 || !grids || !works || !fluidvars || !fluidauxvars || !electrovars || !cfgs)
    return set_err(GEM_EINVAL, "gem_batch_create: null argument or n < 1");
  *out = nullptr;
  std::vector<InstDev> h(n);
  gem_batch* b = new gem_batch();
  b->n = n;
  int lx1_max = 0;
  for (int i = 0; i < n; ++i)
    if (grids[i]) lx1_max = std::max(lx1_max, grids[i]->dev.d.lx1);
  b->lu_slot = lu_slot_doubles(lx1_max);
  if (cudaMalloc(&b->d_lu, sizeof(double) * lu_slots() * b->lu_slot) != cudaSuccess) {
    delete b;
    return set_err(GEM_ENOMEM, "cudaMalloc of the batch's band-solve scratch failed");
  }
  for (int i = 0; i < n; ++i) {
    const gem_grid* g = grids[i];
    gem_work* w = works[i];
    if (!g || !w || !fluidvars[i] || !fluidauxvars[i] || !electrovars[i]) {
      gem_batch_destroy(b);
      return set_err(GEM_EINVAL, "gem_batch_create: instance %d has a null argument", i);
    }
    int rc = check_step(g);
    if (rc) {
      gem_batch_destroy(b);
      return set_err(rc, "gem_batch_create: instance %d: %s", i, g_err.c_str());
    }
    if (cfgs[i].diffsolvetype != 1 && cfgs[i].diffsolvetype != 2) {
      gem_batch_destroy(b);
      return set_err(GEM_EINVAL, "gem_batch_create: instance %d: diffsolvetype %d (1 or 2)", i,
                     cfgs[i].diffsolvetype);
    }
    if (w->lx1 != g->dev.d.lx1 || w->lx2 != g->dev.d.lx2 || w->lx3 != g->dev.d.lx3) {
      gem_batch_destroy(b);
      return set_err(GEM_EINVAL, "gem_batch_create: instance %d: work and grid sizes differ", i);
    }
    InstDev& I = h[i];
    std::memset(&I, 0, sizeof(I));
    I.sw.G = g->dev;
    I.sw.B = blocks(g, fluidvars[i], fluidauxvars[i]);
    I.sw.vsi = nullptr;
    I.sw.vs1i = w->vs1i;
    I.sw.dtp = w->dt;
    I.sw.dtp_w = w->dt;
    I.sw.which = 0;
    I.df.G = g->dev;
    I.df.B = I.sw.B;
    I.df.J1 = electrovars[i] + 3 * g->dev.d.ng;
    I.df.nn = w->nn;
    I.df.Tn = w->Tn;
    I.df.dtp = w->dt;
    I.df.Teinf = cfgs[i].Teinf;
    I.df.Ttop = w->Ttop;
    I.df.lu = b->d_lu;
    I.df.lu_slot = b->lu_slot;
    I.df.x3fast = (!g->dev.unit && g->dev.c3 == 0) ? 1 : 0;
    I.df.solver = cfgs[i].diffsolvetype;
    I.df.fused = 1;
    I.acc = w->acc;
    I.tcfl = cfgs[i].tcfl;
    b->grids.push_back(g);
    b->works.push_back(w);
  }
  int rc = GEM_OK;
  if (cudaMalloc(&b->d_inst, sizeof(InstDev) * n) != cudaSuccess) {
    gem_batch_destroy(b);
    return set_err(GEM_ENOMEM, "cudaMalloc of the batch instance table failed");
  }
  if (cudaMemcpy(b->d_inst, h.data(), sizeof(InstDev) * n, cudaMemcpyHostToDevice) != cudaSuccess)
    rc = set_err(GEM_ECUDA, "copy of the batch instance table failed");
  if (rc == GEM_OK) rc = batch_build_lists(b);
  if (rc == GEM_OK && cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking) != cudaSuccess)
    rc = set_err(GEM_ECUDA, "cudaStreamCreate failed");
  if (rc != GEM_OK) {
    gem_batch_destroy(b);
    return rc;
  }
  *out = b;
  return GEM_OK;
}

int gem_batch_destroy(gem_batch* b) {
  if (!b) return GEM_OK;
  batch_drop_graph(b);
  for (auto& L : b->launches)
    if (L.d_items) cudaFree(L.d_items);
  if (b->d_inst) cudaFree(b->d_inst);
  if (b->d_dt_in) cudaFree(b->d_dt_in);
  if (b->d_lu) cudaFree(b->d_lu);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  delete b;
  return GEM_OK;
}

int gem_batch_size(const gem_batch* b) { return b ? b->n : 0; }

int gem_batch_set_param(gem_batch* b, int param, int value) {
  if (!b) return set_err(GEM_EINVAL, "null batch");
  if (param == GEM_BATCH_USE_GRAPH) {
    b->use_graph = value ? 1 : 0;
    return GEM_OK;
  }
  if (param == GEM_BATCH_DIFF_BLOCKS) {
    if (value < 1 || value > LU_MINB_DEFAULT)
      return set_err(GEM_EINVAL, "diffusion blocks per SM %d: 1..%d", value, LU_MINB_DEFAULT);
    b->diff_blocks = value;
  } else if (param == GEM_BATCH_GRID_PCT) {
    if (value != 0 && (value < 10 || value > 400))
      return set_err(GEM_EINVAL, "persistent grid percentage %d: 0 (one block per item) or 10..400", value);
    b->per_sm_scale = value;
  } else {
    return set_err(GEM_EINVAL, "unknown batch parameter %d", param);
  }
  batch_drop_graph(b);
  return batch_build_lists(b);
}

int gem_batch_step(gem_batch* b, void* stream) {
  if (!b) return set_err(GEM_EINVAL, "null batch");
  cudaStream_t st = S(stream);
  if (!b->use_graph) return batch_enqueue(b, st);
  if (!b->exec) {
    GEM_CUDA(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal));
    const int rc = batch_enqueue(b, b->cap_stream);
    cudaGraph_t gph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->cap_stream, &gph);
    if (rc) {
      if (gph) cudaGraphDestroy(gph);
      return rc;
    }
    if (e != cudaSuccess) return set_err(GEM_ECUDA, "stream capture of the batched step failed: %s", cudaGetErrorString(e));
    b->graph = gph;
    GEM_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
  }
  GEM_CUDA(cudaGraphLaunch(b->exec, st));
  return GEM_OK;
}

int gem_batch_step_fixed_dt(gem_batch* b, const double* host_dts, void* stream) {
  if (!b || !host_dts) return set_err(GEM_EINVAL, "null argument");
  cudaStream_t st = S(stream);
  if (!b->d_dt_in && cudaMalloc(&b->d_dt_in, sizeof(double) * b->n) != cudaSuccess) {
    b->d_dt_in = nullptr;
    return set_err(GEM_ENOMEM, "cudaMalloc of the prescribed-dt buffer failed");
  }
  GEM_CUDA(cudaMemcpyAsync(b->d_dt_in, host_dts, sizeof(double) * b->n, cudaMemcpyHostToDevice, st));
  if (!b->use_graph) return batch_enqueue(b, st, true);
  if (!b->exec_fixed) {
    GEM_CUDA(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal));
    const int rc = batch_enqueue(b, b->cap_stream, true);
    cudaGraph_t gph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->cap_stream, &gph);
    if (rc) {
      if (gph) cudaGraphDestroy(gph);
      return rc;
    }
    if (e != cudaSuccess) return set_err(GEM_ECUDA, "stream capture of the batched step failed: %s", cudaGetErrorString(e));
    b->graph_fixed = gph;
    GEM_CUDA(cudaGraphInstantiate(&b->exec_fixed, b->graph_fixed, 0));
  }
  GEM_CUDA(cudaGraphLaunch(b->exec_fixed, st));
  return GEM_OK;
}

int gem_batch_dts(const gem_batch* b, double* host_dt) {
  if (!b || !host_dt) return set_err(GEM_EINVAL, "null argument");
  for (int i = 0; i < b->n; ++i) GEM_CUDA(cudaMemcpy(host_dt + i, b->works[i]->dt, sizeof(double), cudaMemcpyDeviceToHost));
  return GEM_OK;
}

int gem_batch_info(const gem_batch* b, int* launches_per_step, long long* items_per_step) {
  if (!b) return set_err(GEM_EINVAL, "null batch");
  long long it = 0;
  for (const auto& L : b->launches) it += (long long)L.items.size();
  if (launches_per_step) *launches_per_step = (int)b->launches.size() + 2;  // + zero, dt finalize
  if (items_per_step) *items_per_step = it;
  return GEM_OK;
}

}  // extern "C"
