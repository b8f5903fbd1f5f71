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
  DiffArgs df;   // fused-diffusion arguments (Mslot = the batch's slot size)
  unsigned long long* acc;
  double tcfl;
};

// work item: instance, block x, block y, the instance's own grid x extent
using Item = int4;

__global__ void __launch_bounds__(32 * LSP, 4) kb_dt_reduce(const InstDev* __restrict__ inst, const Item* __restrict__ it, int n) {
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const Item q = it[w];
    const InstDev& I = inst[q.x];
    const VB vb{q.y, q.z, q.w};
    if (I.sw.G.unit)
      b_dt_reduce<true, 0>(I.sw.G, I.sw.B, I.acc, nullptr, vb);
    else
      b_dt_reduce<false, 0>(I.sw.G, I.sw.B, I.acc, nullptr, vb);
  }
}

__global__ void kb_zero_acc(const InstDev* inst, int ninst) {
  const int i = blockIdx.x;
  if (i < ninst && threadIdx.x < 3 * LSP) inst[i].acc[threadIdx.x] = 0ull;
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

template <int DIM>
__global__ void __launch_bounds__(224, 2) kb_sweep_march(const InstDev* __restrict__ inst, const Item* __restrict__ it, int n) {
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const Item q = it[w];
    const InstDev& I = inst[q.x];
    const VB vb{q.y, q.z, q.w};
    if (I.sw.G.unit)
      b_sweep_march<DIM, true, true>(I.sw, vb);
    else
      b_sweep_march<DIM, false, true>(I.sw, vb);
    if (DIM == 2) __syncthreads();  // the epilogue's shared buffers are reused by the next item
  }
}

__global__ void __launch_bounds__(224) kb_sweep_x1(const InstDev* __restrict__ inst, const Item* __restrict__ it, int n) {
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const Item q = it[w];
    const InstDev& I = inst[q.x];
    const VB vb{q.y, q.z, q.w};
    if (I.sw.G.unit)
      b_sweep_x1<true, true>(I.sw, vb);
    else
      b_sweep_x1<false, true>(I.sw, vb);
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

__global__ void __launch_bounds__(128) kb_diffusion(const InstDev* __restrict__ inst, const Item* __restrict__ it, int n) {
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const Item q = it[w];
    const InstDev& I = inst[q.x];
    if (I.df.G.unit)
      b_diffusion<true>(I.df, VB{q.y, q.z, q.w});
    else
      b_diffusion<false>(I.df, VB{q.y, q.z, q.w});
  }
}

}  // namespace gemk

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
namespace {

enum BatchPhase {
  BP_DT = 0, BP_GX1, BP_GX2, BP_GX3, BP_SW3, BP_SW1, BP_SW2, BP_EPI, BP_CVE, BP_DIFF, BP_N
};

struct PhaseList {
  std::vector<Item> items;
  Item* d_items = nullptr;
  int grid = 0;  // persistent blocks
};

}  // namespace

struct gem_batch {
  int n = 0;
  std::vector<const gem_grid*> grids;
  std::vector<gem_work*> works;
  InstDev* d_inst = nullptr;
  PhaseList ph[BP_N];
  int Mmax = 2, wpb = 4;
  size_t diff_smem = 0;
  int per_sm_scale = 100;  // percent of the occupancy-limited persistent grid
  cudaStream_t cap_stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int use_graph = 1;
};

namespace {

// per-instance block counts of each phase, as the plain launchers size them
void instance_items(const gem_grid* g, int idx, int wpb, std::vector<Item>* out) {
  const Dims& d = g->dev.d;
  auto add1 = [&](int ph, long long nb) {
    for (long long b = 0; b < nb; ++b) out[ph].push_back(make_int4(idx, (int)b, 0, (int)nb));
  };
  add1(BP_DT, std::min<long long>((long long)d.lx2 * d.lx3, (long long)num_sms() * 8));
  add1(BP_GX1, grid_for((long long)(d.lx2 + 4) * (d.lx3 + 4) * LSP, 128));
  add1(BP_GX2, grid_for((long long)(d.lx1 + 4) * (d.lx3 + 4) * LSP, 128));
  add1(BP_GX3, grid_for((long long)(d.lx1 + 4) * (d.lx2 + 4) * LSP, 128));
  const int gx13 = (d.lx1 + 31) / 32;
  for (int by = 0; by < d.lx2; ++by)
    for (int bx = 0; bx < gx13; ++bx) out[BP_SW3].push_back(make_int4(idx, bx, by, gx13));
  for (int by = 0; by < d.lx3; ++by)
    for (int bx = 0; bx < d.lx2; ++bx) out[BP_SW1].push_back(make_int4(idx, bx, by, d.lx2));
  for (int by = 0; by < d.lx3; ++by)
    for (int bx = 0; bx < gx13; ++bx) out[BP_SW2].push_back(make_int4(idx, bx, by, gx13));
  add1(BP_EPI, grid_for(d.ng, 256));
  if (g->dev.has_null && (g->dev.gridflag == 0 || g->dev.gridflag == 1))
    add1(BP_CVE, grid_for((long long)d.lx2 * d.lx3 * LSP, 128));
  const long long ncs = (long long)d.lx2 * d.lx3 * LSP;
  add1(BP_DIFF, std::min<long long>((ncs + wpb - 1) / wpb, (long long)num_sms() * 2));
}

template <class K>
int persistent_grid(K kernel, int threads, size_t smem, size_t nitems, int scale_pct, int* out) {
  int per_sm = 0;
  GEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
  if (per_sm < 1) per_sm = 1;
  long long g = (long long)num_sms() * per_sm * scale_pct / 100;
  if (g < 1) g = 1;
  if (g > (long long)nitems) g = (long long)nitems;
  *out = (int)std::max<long long>(g, 1);
  return GEM_OK;
}

int batch_build_lists(gem_batch* b) {
  std::vector<Item> lists[BP_N];
  // largest instances first, so the long items start early
  std::vector<int> order(b->n);
  for (int i = 0; i < b->n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    return b->grids[x]->dev.d.ng > b->grids[y]->dev.d.ng;
  });
  for (int i : order) instance_items(b->grids[i], i, b->wpb, lists);
  for (int p = 0; p < BP_N; ++p) {
    PhaseList& L = b->ph[p];
    if (L.d_items) cudaFree(L.d_items);
    L.d_items = nullptr;
    L.items = lists[p];
    if (!L.items.empty()) {
      if (cudaMalloc(&L.d_items, L.items.size() * sizeof(Item)) != cudaSuccess)
        return set_err(GEM_ENOMEM, "cudaMalloc of a batch work list failed");
      GEM_CUDA(cudaMemcpy(L.d_items, L.items.data(), L.items.size() * sizeof(Item), cudaMemcpyHostToDevice));
    }
  }
  b->diff_smem = (size_t)DNA * b->Mmax * 32 * sizeof(double) * b->wpb;
  GEM_CUDA(cudaFuncSetAttribute(kb_diffusion, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->diff_smem));
  int rc = GEM_OK;
  const int sc = b->per_sm_scale;
  if ((rc = persistent_grid(kb_dt_reduce, 32 * LSP, 0, b->ph[BP_DT].items.size(), sc, &b->ph[BP_DT].grid))) return rc;
  if ((rc = persistent_grid(kb_ghost_x1, 128, 0, b->ph[BP_GX1].items.size(), sc, &b->ph[BP_GX1].grid))) return rc;
  if ((rc = persistent_grid(kb_ghost_x2, 128, 0, b->ph[BP_GX2].items.size(), sc, &b->ph[BP_GX2].grid))) return rc;
  if ((rc = persistent_grid(kb_ghost_x3, 128, 0, b->ph[BP_GX3].items.size(), sc, &b->ph[BP_GX3].grid))) return rc;
  if ((rc = persistent_grid(kb_sweep_march<3>, 32 * LSP, 0, b->ph[BP_SW3].items.size(), sc, &b->ph[BP_SW3].grid))) return rc;
  if ((rc = persistent_grid(kb_sweep_x1, 32 * LSP, 0, b->ph[BP_SW1].items.size(), sc, &b->ph[BP_SW1].grid))) return rc;
  if ((rc = persistent_grid(kb_sweep_march<2>, 32 * LSP, 0, b->ph[BP_SW2].items.size(), sc, &b->ph[BP_SW2].grid))) return rc;
  if ((rc = persistent_grid(kb_ghost_epilogue, 256, 0, b->ph[BP_EPI].items.size(), sc, &b->ph[BP_EPI].grid))) return rc;
  if ((rc = persistent_grid(kb_clean_vel_edges, 128, 0, std::max<size_t>(1, b->ph[BP_CVE].items.size()), sc,
                            &b->ph[BP_CVE].grid))) return rc;
  if ((rc = persistent_grid(kb_diffusion, 32 * b->wpb, b->diff_smem, b->ph[BP_DIFF].items.size(), sc,
                            &b->ph[BP_DIFF].grid))) return rc;
  return GEM_OK;
}

void batch_drop_graph(gem_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

// the eleven launches of one batched step
int batch_enqueue(gem_batch* b, cudaStream_t st) {
  const InstDev* I = b->d_inst;
  auto n = [&](int p) { return (int)b->ph[p].items.size(); };
  kb_zero_acc<<<b->n, 32, 0, st>>>(I, b->n);
  kb_dt_reduce<<<b->ph[BP_DT].grid, dim3(32, LSP), 0, st>>>(I, b->ph[BP_DT].d_items, n(BP_DT));
  kb_dt_finalize<<<(b->n + 63) / 64, 64, 0, st>>>(I, b->n);
  kb_ghost_x1<<<b->ph[BP_GX1].grid, 128, 0, st>>>(I, b->ph[BP_GX1].d_items, n(BP_GX1));
  kb_ghost_x2<<<b->ph[BP_GX2].grid, 128, 0, st>>>(I, b->ph[BP_GX2].d_items, n(BP_GX2));
  kb_ghost_x3<<<b->ph[BP_GX3].grid, 128, 0, st>>>(I, b->ph[BP_GX3].d_items, n(BP_GX3));
  kb_sweep_march<3><<<b->ph[BP_SW3].grid, dim3(32, LSP), 0, st>>>(I, b->ph[BP_SW3].d_items, n(BP_SW3));
  kb_sweep_x1<<<b->ph[BP_SW1].grid, dim3(32, LSP), 0, st>>>(I, b->ph[BP_SW1].d_items, n(BP_SW1));
  kb_sweep_march<2><<<b->ph[BP_SW2].grid, dim3(32, LSP), 0, st>>>(I, b->ph[BP_SW2].d_items, n(BP_SW2));
  kb_ghost_epilogue<<<b->ph[BP_EPI].grid, 256, 0, st>>>(I, b->ph[BP_EPI].d_items, n(BP_EPI));
  if (n(BP_CVE) > 0)
    kb_clean_vel_edges<<<b->ph[BP_CVE].grid, 128, 0, st>>>(I, b->ph[BP_CVE].d_items, n(BP_CVE));
  kb_diffusion<<<b->ph[BP_DIFF].grid, 32 * b->wpb, b->diff_smem, st>>>(I, b->ph[BP_DIFF].d_items, n(BP_DIFF));
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
  int Mmax = 2;
  for (int i = 0; i < n; ++i) {
    const gem_grid* g = grids[i];
    gem_work* w = works[i];
    if (!g || !w || !fluidvars[i] || !fluidauxvars[i] || !electrovars[i]) {
      delete b;
      return set_err(GEM_EINVAL, "gem_batch_create: instance %d has a null argument", i);
    }
    int rc = check_step(g);
    if (rc) {
      delete b;
      return set_err(rc, "gem_batch_create: instance %d: %s", i, g_err.c_str());
    }
    if (cfgs[i].diffsolvetype != 1 && cfgs[i].diffsolvetype != 2) {
      delete b;
      return set_err(GEM_EINVAL, "gem_batch_create: instance %d: diffsolvetype %d (1 or 2)", i,
                     cfgs[i].diffsolvetype);
    }
    if (w->lx1 != g->dev.d.lx1 || w->lx2 != g->dev.d.lx2 || w->lx3 != g->dev.d.lx3) {
      delete b;
      return set_err(GEM_EINVAL, "gem_batch_create: instance %d: work and grid sizes differ", i);
    }
    const int M = std::max(2, (g->dev.d.lx1 + 31) / 32);
    Mmax = std::max(Mmax, M);
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
    I.df.solver = cfgs[i].diffsolvetype;
    I.df.M = M;
    I.df.fused = 1;
    I.acc = w->acc;
    I.tcfl = cfgs[i].tcfl;
    b->grids.push_back(g);
    b->works.push_back(w);
  }
  b->Mmax = Mmax;
  for (int i = 0; i < n; ++i) h[i].df.Mslot = Mmax;  // one slot size: warps move between instances
  const size_t per_warp = (size_t)DNA * Mmax * 32 * sizeof(double);
  b->wpb = (int)std::min<size_t>(4, (227 * 1024) / per_warp);
  if (b->wpb < 1) {
    delete b;
    return set_err(GEM_EINVAL, "gem_batch_create: lx1 too long for the on-chip column solver");
  }
  int rc = GEM_OK;
  if (cudaMalloc(&b->d_inst, sizeof(InstDev) * n) != cudaSuccess) {
    delete b;
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
  for (int p = 0; p < BP_N; ++p)
    if (b->ph[p].d_items) cudaFree(b->ph[p].d_items);
  if (b->d_inst) cudaFree(b->d_inst);
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
  if (param == GEM_BATCH_DIFF_WARPS) {
    const size_t per_warp = (size_t)DNA * b->Mmax * 32 * sizeof(double);
    if (value < 1 || value > 4 || per_warp * value > 227 * 1024)
      return set_err(GEM_EINVAL, "diffusion warps per block %d: 1..4 within 227 KB of shared memory", value);
    b->wpb = value;
  } else if (param == GEM_BATCH_GRID_PCT) {
    if (value < 10 || value > 400) return set_err(GEM_EINVAL, "persistent grid percentage %d: 10..400", value);
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

int gem_batch_dts(const gem_batch* b, double* host_dt) {
  if (!b || !host_dt) return set_err(GEM_EINVAL, "null argument");
  for (int i = 0; i < b->n; ++i) GEM_CUDA(cudaMemcpy(host_dt + i, b->works[i]->dt, sizeof(double), cudaMemcpyDeviceToHost));
  return GEM_OK;
}

int gem_batch_info(const gem_batch* b, int* launches_per_step, long long* items_per_step) {
  if (!b) return set_err(GEM_EINVAL, "null batch");
  int l = 3;  // zero, dt reduce, dt finalize
  long long it = 0;
  for (int p = 0; p < BP_N; ++p) {
    it += (long long)b->ph[p].items.size();
    if (p != BP_DT && !b->ph[p].items.empty()) ++l;
  }
  if (launches_per_step) *launches_per_step = l;
  if (items_per_step) *items_per_step = it;
  return GEM_OK;
}

}  // extern "C"
