// Host side of libgemini_b200: device grid/work objects, kernel launchers and the
// device-resident C ABI declared in include/gem_fluid.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gem_fluid.h"
#include "gem_kernels.cuh"

using namespace gemk;

extern "C" void gem_capi_bind_grid(gem_grid* g);
extern "C" void gem_capi_forget_grid(gem_grid* g);

namespace {

thread_local std::string g_err;

int set_err(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define GEM_CUDA(call)                                                                    \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return set_err(GEM_ECUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                     __FILE__, __LINE__);                                                 \
  } while (0)

#define GEM_LAUNCHED(name)                                                                    \
  do {                                                                                        \
    cudaError_t e_ = cudaGetLastError();                                                      \
    if (e_ != cudaSuccess) return set_err(GEM_ECUDA, "launch of %s failed: %s", name, cudaGetErrorString(e_)); \
  } while (0)

int num_sms() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms;
}

// |y| in [2^-400, 2^400] (as the device's exact-quotient range test reads the exponent)
bool y_in_range(double y) {
  unsigned long long u;
  std::memcpy(&u, &y, 8);
  const unsigned h = (unsigned)(u >> 32) & 0x7fffffffu;
  return h - (623u << 20) < (800u << 20);
}

// cells of the ghost shell (the ghost epilogue's work items)
long long ghost_cells(const Dims& d) {
  const long long a1 = d.lx1 + 4, a2 = d.lx2 + 4;
  return 4 * (a1 * a2 + a1 * d.lx3 + (long long)d.lx2 * d.lx3);
}

unsigned grid_for(long long n, int threads, int per_sm = 8) {
  long long b = (n + threads - 1) / threads;
  const long long cap = (long long)num_sms() * per_sm;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (unsigned)b;
}

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace

struct gem_grid {
  GridDev dev;
  int lnull;
  std::vector<void*> allocs;
};

// Per-step CUDA events at the phase boundaries of dt_calc + the fused step (optional):
// E0 dt_calc E1 ghost fill E2 sweep x3 E3 sweep x1 E4 sweep x2 E5 ghost epilogue E6
// diffusion E7
constexpr int NPHASE = 7;
struct PhaseTimer {
  int cap = 0;
  long long step = 0;
  std::vector<cudaEvent_t> ev;  // cap * (NPHASE + 1)
  void record(int k, cudaStream_t st) {
    if (cap > 0) cudaEventRecord(ev[(size_t)(step % cap) * (NPHASE + 1) + k], st);
  }
};

struct gem_work {
  PhaseTimer timer;
  int lx1, lx2, lx3;
  double *vs1i, *vs2i, *vs3i, *nn, *Tn, *dt;
  double* Ttop;             // per-column exospheric temperature (lx2*lx3), or null for Teinf
  double* lu;               // band-solve scratch of k_diffusion_lu (lu_slots() slots of lx1 rows)
  // the reference work object's sub-step contents for the host-memory *_C routines, allocated
  // on first use: the neutral state and ionization rates (gem_work_set_sources) and the
  // artificial viscosity Q, production and loss rates Pr, Lo
  double* sub;
  gem_source_inputs src;
  int has_src;
  double *Q, *Pr, *Lo;
  unsigned long long* acc;  // 32 slots: CFL maxima / counters
  long long nf1, nf2, nf3;
  // device staging of the host blocks for gem_fluid_adv_host, and its copy-out stream with
  // the events after the ghost fill, the ghost epilogue and the diffusion
  double *F, *A, *E;
  size_t nF, nA, nE;
  cudaStream_t cs;
  cudaEvent_t ev[4];
};

namespace {

int dev_copy(const double* h, size_t n, const double** out, std::vector<void*>& allocs) {
  void* p = nullptr;
  if (cudaMalloc(&p, n * sizeof(double)) != cudaSuccess)
    return set_err(GEM_ENOMEM, "cudaMalloc of %zu doubles failed", n);
  allocs.push_back(p);
  GEM_CUDA(cudaMemcpy(p, h, n * sizeof(double), cudaMemcpyHostToDevice));
  *out = static_cast<const double*>(p);
  return GEM_OK;
}

int check_grid(const gem_grid* g) {
  if (!g) return set_err(GEM_EINVAL, "null grid");
  return GEM_OK;
}

Blocks blocks(const gem_grid* g, double* F, double* A) {
  Blocks b;
  b.F = F;
  b.A = A;
  b.ng = g->dev.d.ng;
  return b;
}

// fused step requirements shared by several launchers
int check_step(const gem_grid* g) {
  const Dims& d = g->dev.d;
  if (d.lx1 < 4) return set_err(GEM_EINVAL, "lx1=%d: the x1 boundary and diffusion stencils need lx1 >= 4", d.lx1);
  if (g->dev.flagper && d.lx3 < 2) return set_err(GEM_EINVAL, "periodic x3 needs lx3 >= 2 (lx3=%d)", d.lx3);
  return GEM_OK;
}

template <int DIM, bool FUSED>
int launch_sweep_t(const gem_grid* g, SweepArgs a, int nsp, cudaStream_t st) {
  const Dims& d = g->dev.d;
  dim3 block(32, nsp);
  if (DIM == 1) {
    // one warp per (x1 column, species)
    dim3 grid(d.lx2, d.lx3);
    if (g->dev.unit)
      k_sweep_x1<true, FUSED><<<grid, block, 0, st>>>(a);
    else
      k_sweep_x1<false, FUSED><<<grid, block, 0, st>>>(a);
    GEM_LAUNCHED("k_sweep_x1");
    return GEM_OK;
  }
  // one thread per (x2 or x3 line, species), 32 adjacent x1 per warp
  dim3 grid((d.lx1 + 31) / 32, (DIM == 3) ? d.lx2 : d.lx3);
  if (DIM == 3 && FUSED) {  // periodicity as a template parameter
    const bool per = g->dev.flagper != 0;
    if (g->dev.unit) {
      if (per) k_sweep_march<3, true, true, 1><<<grid, block, 0, st>>>(a);
      else k_sweep_march<3, true, true, 0><<<grid, block, 0, st>>>(a);
    } else {
      if (per) k_sweep_march<3, false, true, 1><<<grid, block, 0, st>>>(a);
      else k_sweep_march<3, false, true, 0><<<grid, block, 0, st>>>(a);
    }
    GEM_LAUNCHED("k_sweep_march");
    return GEM_OK;
  }
  if (g->dev.unit)
    k_sweep_march<DIM == 3 ? 3 : 2, true, FUSED><<<grid, block, 0, st>>>(a);
  else
    k_sweep_march<DIM == 3 ? 3 : 2, false, FUSED><<<grid, block, 0, st>>>(a);
  GEM_LAUNCHED("k_sweep_march");
  return GEM_OK;
}

int launch_sweep(const gem_grid* g, int dim, bool fused, SweepArgs a, int nsp, cudaStream_t st) {
  if (fused) {
    if (dim == 1) return launch_sweep_t<1, true>(g, a, nsp, st);
    if (dim == 2) return launch_sweep_t<2, true>(g, a, nsp, st);
    return launch_sweep_t<3, true>(g, a, nsp, st);
  }
  if (dim == 1) return launch_sweep_t<1, false>(g, a, nsp, st);
  if (dim == 2) return launch_sweep_t<2, false>(g, a, nsp, st);
  return launch_sweep_t<3, false>(g, a, nsp, st);
}

int launch_ghost_fill(const gem_grid* g, Blocks B, const double* vs1i, int lsp, bool fused,
                      cudaStream_t st) {
  const Dims& d = g->dev.d;
  const GridDev& G = g->dev;
  const long long ncol = (long long)(d.lx2 + 4) * (d.lx3 + 4) * lsp;
  const long long nrow2 = (long long)(d.lx1 + 4) * (d.lx3 + 4) * lsp;
  const long long nrow3 = (long long)(d.lx1 + 4) * (d.lx2 + 4) * lsp;
  if (fused) {
    k_ghost_x1<true><<<grid_for(ncol, 128), 128, 0, st>>>(G, B, vs1i, lsp);
    k_ghost_x2<true><<<grid_for(nrow2, 128), 128, 0, st>>>(G, B, lsp);
    if (G.flagper)
      k_ghost_x3<true, true><<<grid_for(nrow3, 128), 128, 0, st>>>(G, B, lsp);
    else
      k_ghost_x3<true, false><<<grid_for(nrow3, 128), 128, 0, st>>>(G, B, lsp);
  } else {
    k_ghost_x1<false><<<grid_for(ncol, 128), 128, 0, st>>>(G, B, vs1i, lsp);
    k_ghost_x2<false><<<grid_for(nrow2, 128), 128, 0, st>>>(G, B, lsp);
    if (!G.flagper) k_ghost_x3<false, false><<<grid_for(nrow3, 128), 128, 0, st>>>(G, B, lsp);
  }
  GEM_LAUNCHED("ghost fill");
  return GEM_OK;
}

// Resident warps per SM of k_diffusion_lu, which is also the number of its scratch slots
// per SM: the occupancy limit of the launch, at most LU_MAX_WARPS_PER_SM.
constexpr int LU_MAX_WARPS_PER_SM = 16;
int lu_warps_per_sm() {
  static int wps = 0;
  if (!wps) {
    int a = 0, b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_diffusion_lu<true>, 32 * LU_WPB, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_diffusion_lu<false>, 32 * LU_WPB, 0);
    const int w = std::min(a, b) * LU_WPB;
    wps = std::max(LU_WPB, std::min(w, LU_MAX_WARPS_PER_SM));
  }
  return wps;
}
long long lu_slots() { return (long long)num_sms() * lu_warps_per_sm(); }
long long lu_slot_doubles(int lx1) { return (long long)lx1 * gemd::LU_ROW * 32; }
// warp tasks of one grid's diffusion, rounded up to whole blocks
long long lu_tasks(const Dims& d) {
  const long long ntask = (((long long)d.lx2 * d.lx3 + 31) / 32) * LSP;
  return ((ntask + LU_WPB - 1) / LU_WPB) * LU_WPB;
}
// scratch slots a grid's launches use: one per resident warp, no more than it has tasks
long long lu_slots_for(const Dims& d) { return std::min(lu_slots(), lu_tasks(d)); }

// The work object's band-solve scratch, allocated by the first diffusion launch that uses
// the work object (the batched step uses its own; a work object only ever batched needs none).
int work_lu(gem_work* w, const gem_grid* g, double** out) {
  if (!w->lu) {
    const size_t bytes = sizeof(double) * lu_slots_for(g->dev.d) * lu_slot_doubles(g->dev.d.lx1);
    if (cudaMalloc(&w->lu, bytes) != cudaSuccess) {
      w->lu = nullptr;
      return set_err(GEM_ENOMEM, "cudaMalloc of %zu bytes for the diffusion's band-solve scratch failed", bytes);
    }
  }
  *out = w->lu;
  return GEM_OK;
}

int launch_diffusion_lu(const gem_grid* g, DiffArgs a, cudaStream_t st) {
  const Dims& d = g->dev.d;
  if (!a.lu) return set_err(GEM_EINVAL, "diffusion without a band-solve scratch");
  a.lu_slot = lu_slot_doubles(d.lx1);
  a.x3fast = (!g->dev.unit && g->dev.c3 == 0) ? 1 : 0;
  const long long nblk = lu_slots_for(d) / LU_WPB;  // the work object holds this many slots
  if (g->dev.unit)
    k_diffusion_lu<true><<<(unsigned)nblk, 32 * LU_WPB, 0, st>>>(a);
  else
    k_diffusion_lu<false><<<(unsigned)nblk, 32 * LU_WPB, 0, st>>>(a);
  GEM_LAUNCHED("k_diffusion_lu");
  return GEM_OK;
}

int launch_diffusion(const gem_grid* g, DiffArgs a, cudaStream_t st) { return launch_diffusion_lu(g, a, st); }

// x2 / x3 sweep adjoints of up to three fields sharing the face velocities v: one marching
// thread per (line, segment of SVM_TJ cells, species, field).
int launch_sweep_vjp_march(const gem_grid* g, int dim, const SweepVjpFields& FS, const double* v, const double* dt,
                           double* vbar, int vacc, cudaStream_t st) {
  SweepVjpArgs a;
  a.G = g->dev;
  a.f = nullptr;
  a.v = v;
  a.dtp = dt;
  a.obar = nullptr;
  a.fbar = nullptr;
  a.vbar = vbar;
  a.frank = 0;
  a.nsp = 0;
  a.vacc = vacc;
  const Dims& d = g->dev.d;
  const int lx = (dim == 2) ? d.lx2 : d.lx3;
  const int nseg = (lx + 4 + SVM_TJ - 1) / SVM_TJ;
  const long long nl = (long long)d.lx1 * ((dim == 2) ? d.lx3 : d.lx2);
  const unsigned nb = grid_for(nl * nseg * FS.nfs, 256, 8);
  if (g->dev.unit) {
    if (dim == 2) k_sweep_vjp_march<2, true><<<nb, 256, 0, st>>>(a, FS, nseg);
    else k_sweep_vjp_march<3, true><<<nb, 256, 0, st>>>(a, FS, nseg);
  } else {
    if (dim == 2) k_sweep_vjp_march<2, false><<<nb, 256, 0, st>>>(a, FS, nseg);
    else k_sweep_vjp_march<3, false><<<nb, 256, 0, st>>>(a, FS, nseg);
  }
  GEM_LAUNCHED("k_sweep_vjp_march");
  return GEM_OK;
}

// x1 sweep adjoints of up to three fields sharing the face velocities v: one warp per
// (x1 line, species, field); FS.vbar[f] (optional) receives field f's velocity cotangent.
int launch_sweep_vjp_x1(const gem_grid* g, const SweepVjpFields& FS, const double* v, const double* dt, int vacc,
                        cudaStream_t st) {
  SweepVjpArgs a;
  a.G = g->dev;
  a.f = nullptr;
  a.v = v;
  a.dtp = dt;
  a.obar = nullptr;
  a.fbar = nullptr;
  a.vbar = nullptr;
  a.frank = 0;
  a.nsp = 0;
  a.vacc = vacc;
  const Dims& d = g->dev.d;
  const long long nwarp = (long long)d.lx2 * d.lx3 * FS.nfs;
  const unsigned nb = (unsigned)std::min<long long>((nwarp + 7) / 8, (long long)num_sms() * 8);
  if (g->dev.unit)
    k_sweep_vjp_x1<true><<<nb, 256, 0, st>>>(a, FS);
  else
    k_sweep_vjp_x1<false><<<nb, 256, 0, st>>>(a, FS);
  GEM_LAUNCHED("k_sweep_vjp_x1");
  return GEM_OK;
}

// Vector-Jacobian product of one field sweep (differentiable path): x1 by warps along the
// lines, x2 / x3 by marching threads.
int launch_sweep_vjp(const gem_grid* g, int dim, int frank, int nsp, const double* f, const double* v,
                     const double* dt, const double* obar, double* fbar, double* vbar, int vacc, cudaStream_t st) {
  SweepVjpFields FS;
  FS.f[0] = f;
  FS.obar[0] = obar;
  FS.fbar[0] = fbar;
  FS.vbar[0] = vbar;
  FS.nsp[0] = nsp;
  FS.frank[0] = (dim == 1) ? 0 : frank;
  FS.nfld = 1;
  FS.nfs = nsp;
  if (dim == 1) return launch_sweep_vjp_x1(g, FS, v, dt, vacc, st);
  return launch_sweep_vjp_march(g, dim, FS, v, dt, vbar, vacc, st);
}

// Vector-Jacobian product of the energy diffusion: one warp per (column, species), VNA
// per-row arrays of M rows per lane in shared memory.
int launch_diffusion_vjp(const gem_grid* g, DiffAdjArgs a, cudaStream_t st) {
  const Dims& d = g->dev.d;
  const int M = std::max(2, (d.lx1 + 31) / 32);
  a.M = M;
  const size_t per_warp = (size_t)VNA * M * 32 * sizeof(double);
  if (per_warp > 227 * 1024) return set_err(GEM_EINVAL, "lx1=%d too long for the on-chip column adjoint", d.lx1);
  auto kern = g->dev.unit ? k_diffusion_vjp<true> : k_diffusion_vjp<false>;
  // warps per block: the choice (4, 2 or 1) that keeps the most warps resident per SM
  int wpb = 1, best = 0, best_per_sm = 1;
  for (int w : {4, 2, 1}) {
    const size_t sm = per_warp * w;
    if (sm > 227 * 1024) continue;
    GEM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int per_sm = 0;
    GEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * w, sm));
    if (per_sm * w > best) {
      best = per_sm * w;
      wpb = w;
      best_per_sm = per_sm;
    }
  }
  const size_t smem = per_warp * wpb;
  GEM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long long ncs = (long long)d.lx2 * d.lx3 * LSP;
  long long nblk = (ncs + wpb - 1) / wpb;
  const long long cap = (long long)num_sms() * std::max(best_per_sm, 1);
  if (nblk > cap) nblk = cap;
  kern<<<(unsigned)nblk, 32 * wpb, smem, st>>>(a);
  GEM_LAUNCHED("k_diffusion_vjp");
  return GEM_OK;
}

}  // namespace

// Static scratch of gem_dt_calc_noalloc_dev: 3*LSP partial maxima per x3 plane.
static __device__ __align__(256) double g_dt_noalloc_part[GEM_DT_NOALLOC_MAX_PLANES * 3 * LSP];
namespace {
constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_part_ptr[kNoallocMaxDevices] = {};
}  // namespace

extern "C" {

const char* gem_last_error(void) { return g_err.c_str(); }
int gem_version(void) { return 1; }

int gem_grid_create(const gem_grid_desc* desc, gem_grid** out) {
  if (!desc || !out) return set_err(GEM_EINVAL, "null argument");
  *out = nullptr;
  const int lx1 = desc->lx1, lx2 = desc->lx2, lx3 = desc->lx3;
  if (lx1 < 1 || lx2 < 1 || lx3 < 1) return set_err(GEM_EINVAL, "grid sizes must be positive");
  if (desc->gridflag < 0 || desc->gridflag > 2) return set_err(GEM_EINVAL, "gridflag must be 0, 1 or 2");
  gem_grid* g = new gem_grid();
  GridDev& G = g->dev;
  G.d = make_dims(lx1, lx2, lx3);
  G.gridflag = desc->gridflag;
  G.flagper = desc->flagper ? 1 : 0;
  G.unit = desc->unit_metrics ? 1 : 0;
  const size_t ng = (size_t)G.d.ng;
  int rc = GEM_OK;
  G.c3 = G.d.s3;
  auto cp = [&](const double* h, size_t n, const double** o) {
    if (rc != GEM_OK) return;
    if (!h) {
      rc = set_err(GEM_EINVAL, "missing grid array");
      return;
    }
    rc = dev_copy(h, n, o, g->allocs);
  };
  const size_t n1 = (size_t)(lx1 + 1) * lx2 * lx3, n2 = (size_t)lx1 * (lx2 + 1) * lx3,
               n3 = (size_t)lx1 * lx2 * (lx3 + 1);
  const double* need[] = {desc->dx1, desc->dx1i, desc->dx2, desc->dx2i, desc->dx3, desc->dx3i,
                          desc->h1, desc->h2, desc->h3, desc->h1x1i, desc->h2x1i, desc->h3x1i,
                          desc->h1x2i, desc->h2x2i, desc->h3x2i, desc->h1x3i, desc->h2x3i, desc->h3x3i};
  for (const double* p : need)
    if (!p) rc = set_err(GEM_EINVAL, "missing grid array");
  // 1-D tables per direction: dx, dx(j)+dx(j+1), dxi and their reciprocals
  const double* dxs_in[3] = {desc->dx1, desc->dx2, desc->dx3};
  const double* dxi_in[3] = {desc->dx1i, desc->dx2i, desc->dx3i};
  const int lxs[3] = {lx1, lx2, lx3};
  for (int dd = 0; dd < 3 && rc == GEM_OK; ++dd) {
    const int l = lxs[dd];
    std::vector<double> dx(dxs_in[dd], dxs_in[dd] + l + 3), ydx(l + 3), dxs(l + 2), ydxs(l + 2),
        dxi(dxi_in[dd], dxi_in[dd] + l), ydxi(l);
    for (int j = 0; j < l + 3; ++j) ydx[j] = 1.0 / dx[j];
    for (int j = 0; j < l + 2; ++j) {
      dxs[j] = dx[j] + dx[j + 1];
      ydxs[j] = 1.0 / dxs[j];
    }
    for (int j = 0; j < l; ++j) ydxi[j] = 1.0 / dxi[j];
    if (l > 1) {  // the exact quotients of the sweeps and the diffusion assume these are in range
      bool ok = true;
      for (int j = 0; j <= l + 2; ++j) ok = ok && y_in_range(ydx[j]);
      for (int j = 0; j <= l - 1; ++j) ok = ok && y_in_range(ydxi[j]);
      for (int j = 0; j <= l + 1; ++j) ok = ok && y_in_range(ydxs[j]);
      if (!ok) rc = set_err(GEM_EINVAL, "x%d grid spacings (ghosts included) outside [2^-400, 2^400]", dd + 1);
    }
    Line1D& L = G.L[dd];
    cp(dx.data(), dx.size(), &L.dx);
    cp(ydx.data(), ydx.size(), &L.ydx);
    cp(dxs.data(), dxs.size(), &L.dxs);
    cp(ydxs.data(), ydxs.size(), &L.ydxs);
    cp(dxi.data(), dxi.size(), &L.dxi);
    cp(ydxi.data(), ydxi.size(), &L.ydxi);
  }
  // Metric tables.  When no metric factor varies along x3 (checked bit for bit over the
  // interior x3 range, the only one the kernels read), one x3 slice is stored and the x3
  // strides are 0, so the tables of a large grid stay resident in L2.
  const long long s2 = G.d.s2, s3 = G.d.s3;
  bool inv = lx3 > 1 && rc == GEM_OK && !G.unit;
  auto same_x3 = [&](const double* a, long long t3, long long inner, int i3lo, int i3hi) {
    for (int i3 = i3lo + 1; i3 <= i3hi; ++i3)
      if (std::memcmp(a + t3 * (i3 - i3lo), a, sizeof(double) * inner) != 0) return false;
    return true;
  };
  if (inv) {
    const long long inner_c = s2 * (lx2 + 4);
    for (const double* h : {desc->h1, desc->h2, desc->h3}) inv = inv && same_x3(h + s3 * 2, s3, inner_c, 1, lx3);
    const long long in1 = (long long)(lx1 + 1) * lx2, in2 = (long long)lx1 * (lx2 + 1), in3 = (long long)lx1 * lx2;
    for (const double* f : {desc->h1x1i, desc->h2x1i, desc->h3x1i}) inv = inv && same_x3(f, in1, in1, 1, lx3);
    for (const double* f : {desc->h1x2i, desc->h2x2i, desc->h3x2i}) inv = inv && same_x3(f, in2, in2, 1, lx3);
    for (const double* f : {desc->h1x3i, desc->h2x3i, desc->h3x3i}) inv = inv && same_x3(f, in3, in3, 1, lx3 + 1);
  }
  G.c3 = inv ? 0 : s3;
  if (rc == GEM_OK && !G.unit) {
    // cell tables (ghosted layout; one slice at ghosted x3 index 2 when invariant)
    const size_t ncell = inv ? (size_t)(s2 * (lx2 + 4)) : ng;
    const size_t off = inv ? (size_t)(s3 * 2) : 0;
    std::vector<double> h1(desc->h1 + off, desc->h1 + off + ncell), h2(desc->h2 + off, desc->h2 + off + ncell),
        h3(desc->h3 + off, desc->h3 + off + ncell), a0(ncell), a1(ncell), y0(ncell), y1(ncell), yh1(ncell);
    for (size_t k = 0; k < ncell; ++k) {
      a0[k] = h1[k] * h2[k] * h3[k];          // advec.f90:312 (frank 0)
      a1[k] = h1[k] * h1[k] * h2[k] * h3[k];  // advec.f90:310 (frank 1)
      y0[k] = 1.0 / a0[k];
      y1[k] = 1.0 / a1[k];
      yh1[k] = 1.0 / h1[k];
    }
    {  // interior cells: the exact quotients of the sweeps and the diffusion assume these
       // reciprocals are in range
      bool ok = true;
      const int n3 = inv ? 1 : lx3;
      for (int i3 = 1; i3 <= n3 && ok; ++i3)
        for (int i2 = 1; i2 <= lx2 && ok; ++i2)
          for (int i1 = 1; i1 <= lx1; ++i1) {
            const size_t k = (size_t)((i1 + 1) + s2 * (i2 + 1) + (inv ? 0 : s3 * (i3 + 1)));
            ok = ok && y_in_range(y0[k]) && y_in_range(y1[k]) && y_in_range(yh1[k]);
          }
      if (!ok) rc = set_err(GEM_EINVAL, "metric factors outside [2^-400, 2^400]");
    }
    cp(h1.data(), ncell, &G.h1);
    cp(h2.data(), ncell, &G.h2);
    cp(h3.data(), ncell, &G.h3);
    cp(yh1.data(), ncell, &G.yh1);
    // dx{d}i*h{d} (multifluid.f90:764-770) and reciprocals; x1 ghosts are never read
    {
      const long long ncol = (long long)ncell / (lx1 + 4);  // (i2, i3) rows in the table
      std::vector<double> dl(ncell), ydl(ncell);
      const std::vector<double>* hs[3] = {&h1, &h2, &h3};
      // with one stored x3 slice, dx3i*h3 is tabulated only when dx3i is uniform
      bool dx3_uniform = true;
      for (int j = 1; j < lx3; ++j) dx3_uniform = dx3_uniform && desc->dx3i[j] == desc->dx3i[0];
      G.dl3_tab = (!inv || dx3_uniform) ? 1 : 0;
      for (int dd = 0; dd < 3 && rc == GEM_OK; ++dd) {
        if (dd == 2 && !G.dl3_tab) {
          G.dl[2] = G.ydl[2] = nullptr;
          break;
        }
        for (long long r = 0; r < ncol; ++r) {
          const int i2 = (int)(r % (lx2 + 4)) - 1, i3 = inv ? 1 : (int)(r / (lx2 + 4)) - 1;
          for (int i1 = -1; i1 <= lx1 + 2; ++i1) {
            const size_t k = (size_t)(i1 + 1) + (size_t)r * (lx1 + 4);
            const int ii = (dd == 0) ? i1 : (dd == 1) ? i2 : i3;
            const int li = lxs[dd];
            double v = 0.0;
            if (ii >= 1 && ii <= li) v = dxi_in[dd][ii - 1] * (*hs[dd])[k];
            dl[k] = v;
            ydl[k] = 1.0 / v;
          }
        }
        cp(dl.data(), ncell, &G.dl[dd]);
        cp(ydl.data(), ncell, &G.ydl[dd]);
      }
    }
    cp(a0.data(), ncell, &G.ha1_0);
    cp(a1.data(), ncell, &G.ha1_1);
    cp(y0.data(), ncell, &G.yha1_0);
    cp(y1.data(), ncell, &G.yha1_1);
    // face tables: sweep x1 uses h2x1i*h3x1i and h1x1i, x2 h1x2i*h3x2i and h2x2i, x3
    // h1x3i*h2x3i and h3x3i (advec.f90:302-304, 333-340, 369-376)
    struct Fam {
      const double *ha, *hb, *hc;
      long long e1, e2, e3;  // extents
    } fam[3] = {{desc->h2x1i, desc->h3x1i, desc->h1x1i, lx1 + 1, lx2, lx3},
                {desc->h1x2i, desc->h3x2i, desc->h2x2i, lx1, lx2 + 1, lx3},
                {desc->h1x3i, desc->h2x3i, desc->h3x3i, lx1, lx2, lx3 + 1}};
    for (int dd = 0; dd < 3 && rc == GEM_OK; ++dd) {
      const Fam& f = fam[dd];
      const size_t nfc = inv ? (size_t)(f.e1 * f.e2) : (size_t)(f.e1 * f.e2 * f.e3);
      std::vector<double> p0(nfc), p1(nfc), hc(f.hc, f.hc + nfc), yhc(nfc);
      bool ok = true;
      for (size_t k = 0; k < nfc; ++k) {
        p0[k] = f.ha[k] * f.hb[k];
        p1[k] = f.ha[k] * f.ha[k] * f.hb[k];
        yhc[k] = 1.0 / hc[k];
        ok = ok && y_in_range(yhc[k]);
      }
      if (!ok) rc = set_err(GEM_EINVAL, "x%d face metric factors outside [2^-400, 2^400]", dd + 1);
      FaceTab& T = G.F[dd];
      T.t1 = 1;
      T.t2 = f.e1;
      T.t3 = inv ? 0 : f.e1 * f.e2;
      cp(p0.data(), nfc, &T.ha2i0);
      cp(p1.data(), nfc, &T.ha2i1);
      cp(hc.data(), nfc, &T.hc);
      cp(yhc.data(), nfc, &T.yhc);
    }
  } else if (rc == GEM_OK) {
    // unit metrics: the kernels read no metric table
    G.h1 = G.h2 = G.h3 = G.yh1 = G.ha1_0 = G.ha1_1 = G.yha1_0 = G.yha1_1 = nullptr;
    for (int dd = 0; dd < 3; ++dd) G.dl[dd] = G.ydl[dd] = nullptr;
    for (int dd = 0; dd < 3; ++dd) G.F[dd] = FaceTab{nullptr, nullptr, nullptr, nullptr, 1, 0, 0};
  }
  g->lnull = 0;
  G.has_null = 0;
  G.nullpts = nullptr;
  if (rc == GEM_OK && desc->nullpts) {
    const size_t nc = (size_t)lx1 * lx2 * lx3;
    for (size_t k = 0; k < nc; ++k) g->lnull += desc->nullpts[k] ? 1 : 0;
    if (g->lnull > 0) {
      void* p = nullptr;
      if (cudaMalloc(&p, nc) != cudaSuccess) {
        rc = set_err(GEM_ENOMEM, "cudaMalloc for nullpts failed");
      } else {
        g->allocs.push_back(p);
        if (cudaMemcpy(p, desc->nullpts, nc, cudaMemcpyHostToDevice) != cudaSuccess)
          rc = set_err(GEM_ECUDA, "copy of nullpts failed");
        G.nullpts = static_cast<const unsigned char*>(p);
        G.has_null = 1;
      }
    }
  }
  if (rc != GEM_OK) {
    gem_grid_destroy(g);
    return rc;
  }
  *out = g;
  gem_capi_bind_grid(g);  // the grid sizes the size-less *_C entry points use
  return GEM_OK;
}

int gem_grid_destroy(gem_grid* g) {
  if (!g) return GEM_OK;
  gem_capi_forget_grid(g);
  for (void* p : g->allocs) cudaFree(p);
  delete g;
  return GEM_OK;
}

int gem_grid_dims(const gem_grid* g, int* lx1, int* lx2, int* lx3) {
  if (check_grid(g)) return GEM_EINVAL;
  if (lx1) *lx1 = g->dev.d.lx1;
  if (lx2) *lx2 = g->dev.d.lx2;
  if (lx3) *lx3 = g->dev.d.lx3;
  return GEM_OK;
}

int gem_work_create(const gem_grid* g, gem_work** out) {
  if (check_grid(g) || !out) return set_err(GEM_EINVAL, "null argument");
  *out = nullptr;
  const Dims& d = g->dev.d;
  gem_work* w = new gem_work();
  w->vs1i = w->vs2i = w->vs3i = w->nn = w->Tn = w->dt = nullptr;
  w->acc = nullptr;
  w->Ttop = nullptr;
  w->lu = nullptr;
  w->sub = nullptr;
  std::memset(&w->src, 0, sizeof(w->src));
  w->has_src = 0;
  w->Q = w->Pr = w->Lo = nullptr;
  w->F = w->A = w->E = nullptr;
  w->nF = w->nA = w->nE = 0;
  w->cs = nullptr;
  for (auto& e : w->ev) e = nullptr;
  w->lx1 = d.lx1;
  w->lx2 = d.lx2;
  w->lx3 = d.lx3;
  w->nf1 = (long long)(d.lx1 + 1) * d.lx2 * d.lx3;
  w->nf2 = (long long)d.lx1 * (d.lx2 + 1) * d.lx3;
  w->nf3 = (long long)d.lx1 * d.lx2 * (d.lx3 + 1);
  const long long nc = (long long)d.lx1 * d.lx2 * d.lx3;
  struct A {
    void** p;
    size_t bytes;
  } al[] = {{(void**)&w->vs1i, sizeof(double) * w->nf1 * LSP},
            {(void**)&w->vs2i, sizeof(double) * w->nf2 * LSP},
            {(void**)&w->vs3i, sizeof(double) * w->nf3 * LSP},
            {(void**)&w->nn, sizeof(double) * nc * 3},
            {(void**)&w->Tn, sizeof(double) * nc},
            {(void**)&w->dt, sizeof(double) * 4},
            {(void**)&w->acc, sizeof(unsigned long long) * 32}};
  for (auto& a : al) {
    if (cudaMalloc(a.p, a.bytes) != cudaSuccess) {
      gem_work_destroy(w);
      return set_err(GEM_ENOMEM, "cudaMalloc of %zu bytes for the work object failed", a.bytes);
    }
    // libgemini.f90:288-291: interface velocities start at zero
    if (cudaMemset(*a.p, 0, a.bytes) != cudaSuccess) {
      gem_work_destroy(w);
      return set_err(GEM_ECUDA, "cudaMemset failed");
    }
  }
  *out = w;
  return GEM_OK;
}

int gem_work_destroy(gem_work* w) {
  if (!w) return GEM_OK;
  for (cudaEvent_t e : w->timer.ev) cudaEventDestroy(e);
  for (cudaEvent_t e : w->ev)
    if (e) cudaEventDestroy(e);
  if (w->cs) cudaStreamDestroy(w->cs);
  void* ps[] = {w->vs1i, w->vs2i, w->vs3i, w->nn, w->Tn, w->dt, w->acc, w->F, w->A, w->E, w->Ttop, w->lu, w->sub};
  for (void* p : ps)
    if (p) cudaFree(p);
  delete w;
  return GEM_OK;
}

namespace {
// the sub-step buffers of a work object (one allocation): Q, Pr, Lo (LSP*nc each), then the
// source inputs nn (6*nc), vn1, vn2, vn3, Tn, alt, g1 (nc each), Prionize ((LSP-1)*nc), Qeionize (nc)
int work_sub_alloc(gem_work* w) {
  if (w->sub) return GEM_OK;
  const size_t nc = (size_t)w->lx1 * w->lx2 * w->lx3;
  const size_t n = nc * (3 * LSP + 6 + 6 + (LSP - 1) + 1);
  if (cudaMalloc(&w->sub, n * sizeof(double)) != cudaSuccess) {
    w->sub = nullptr;
    return set_err(GEM_ENOMEM, "cudaMalloc of %zu doubles for the sub-step buffers failed", n);
  }
  double* p = w->sub;
  w->Q = p;
  p += LSP * nc;
  w->Pr = p;
  p += LSP * nc;
  w->Lo = p;
  p += LSP * nc;
  double* nn = p;
  p += 6 * nc;
  double* v1 = p;
  p += nc;
  double* v2 = p;
  p += nc;
  double* v3 = p;
  p += nc;
  double* tn = p;
  p += nc;
  double* al = p;
  p += nc;
  double* g1 = p;
  p += nc;
  double* pri = p;
  p += (LSP - 1) * nc;
  double* qei = p;
  w->src.nn = nn;
  w->src.vn1 = v1;
  w->src.vn2 = v2;
  w->src.vn3 = v3;
  w->src.Tn = tn;
  w->src.alt = al;
  w->src.g1 = g1;
  w->src.Prionize = pri;
  w->src.Qeionize = qei;
  return GEM_OK;
}
}  // namespace

int gem_work_set_sources(gem_work* w, const gem_source_inputs* host) {
  if (!w || !host || !host->nn || !host->vn1 || !host->vn2 || !host->vn3 || !host->Tn || !host->alt || !host->g1 ||
      !host->Prionize || !host->Qeionize)
    return set_err(GEM_EINVAL, "null argument");
  int rc = work_sub_alloc(w);
  if (rc) return rc;
  const size_t nc = (size_t)w->lx1 * w->lx2 * w->lx3, b = nc * sizeof(double);
  const gem_source_inputs& d = w->src;
  GEM_CUDA(cudaMemcpy((void*)d.nn, host->nn, 6 * b, cudaMemcpyHostToDevice));
  GEM_CUDA(cudaMemcpy((void*)d.vn1, host->vn1, b, cudaMemcpyHostToDevice));
  GEM_CUDA(cudaMemcpy((void*)d.vn2, host->vn2, b, cudaMemcpyHostToDevice));
  GEM_CUDA(cudaMemcpy((void*)d.vn3, host->vn3, b, cudaMemcpyHostToDevice));
  GEM_CUDA(cudaMemcpy((void*)d.Tn, host->Tn, b, cudaMemcpyHostToDevice));
  GEM_CUDA(cudaMemcpy((void*)d.alt, host->alt, b, cudaMemcpyHostToDevice));
  GEM_CUDA(cudaMemcpy((void*)d.g1, host->g1, b, cudaMemcpyHostToDevice));
  GEM_CUDA(cudaMemcpy((void*)d.Prionize, host->Prionize, (LSP - 1) * b, cudaMemcpyHostToDevice));
  GEM_CUDA(cudaMemcpy((void*)d.Qeionize, host->Qeionize, b, cudaMemcpyHostToDevice));
  // the diffusion reads the same atmosphere: O, N2, O2 and Tn
  GEM_CUDA(cudaMemcpy(w->nn, host->nn, 3 * b, cudaMemcpyHostToDevice));
  GEM_CUDA(cudaMemcpy(w->Tn, host->Tn, b, cudaMemcpyHostToDevice));
  w->has_src = 1;
  return GEM_OK;
}

int gem_work_prepare(gem_work* w, const gem_grid* g) {
  if (!w || check_grid(g)) return set_err(GEM_EINVAL, "null argument");
  if (w->lx1 != g->dev.d.lx1 || w->lx2 != g->dev.d.lx2 || w->lx3 != g->dev.d.lx3)
    return set_err(GEM_EINVAL, "work object and grid sizes differ");
  double* p = nullptr;
  return work_lu(w, g, &p);
}

int gem_work_substep_buffers(gem_work* w, const gem_source_inputs** src, double** Q, double** Pr, double** Lo) {
  if (!w) return set_err(GEM_EINVAL, "null work object");
  int rc = work_sub_alloc(w);
  if (rc) return rc;
  if (src) *src = w->has_src ? &w->src : nullptr;
  if (Q) *Q = w->Q;
  if (Pr) *Pr = w->Pr;
  if (Lo) *Lo = w->Lo;
  return GEM_OK;
}

int gem_work_set_neutrals(gem_work* w, const double* nn, const double* Tn) {
  if (!w || !nn || !Tn) return set_err(GEM_EINVAL, "null argument");
  const size_t nc = (size_t)w->lx1 * w->lx2 * w->lx3;
  GEM_CUDA(cudaMemcpy(w->nn, nn, nc * 3 * sizeof(double), cudaMemcpyHostToDevice));
  GEM_CUDA(cudaMemcpy(w->Tn, Tn, nc * sizeof(double), cudaMemcpyHostToDevice));
  return GEM_OK;
}

int gem_work_interface_vels(gem_work* w, int which, double* host, int dir) {
  if (!w || !host || which < 1 || which > 3) return set_err(GEM_EINVAL, "bad argument");
  double* p = which == 1 ? w->vs1i : which == 2 ? w->vs2i : w->vs3i;
  const long long n = (which == 1 ? w->nf1 : which == 2 ? w->nf2 : w->nf3) * LSP;
  if (dir == 0)
    GEM_CUDA(cudaMemcpy(p, host, n * sizeof(double), cudaMemcpyHostToDevice));
  else
    GEM_CUDA(cudaMemcpy(host, p, n * sizeof(double), cudaMemcpyDeviceToHost));
  return GEM_OK;
}

double* gem_work_array(gem_work* w, int which) {
  if (!w) return nullptr;
  switch (which) {
    case 1: return w->vs1i;
    case 2: return w->vs2i;
    case 3: return w->vs3i;
    case 4: return w->nn;
    case 5: return w->Tn;
    default: return nullptr;
  }
}

double* gem_work_dt(gem_work* w) { return w ? w->dt : nullptr; }

int gem_work_set_top_temperature(gem_work* w, const double* Ttop, int on_device) {
  if (!w) return set_err(GEM_EINVAL, "null work object");
  if (!Ttop) {
    if (w->Ttop) cudaFree(w->Ttop);
    w->Ttop = nullptr;
    return GEM_OK;
  }
  const size_t n = (size_t)w->lx2 * w->lx3;
  if (!w->Ttop && cudaMalloc(&w->Ttop, n * sizeof(double)) != cudaSuccess) {
    w->Ttop = nullptr;
    return set_err(GEM_ENOMEM, "cudaMalloc of the top-temperature array failed");
  }
  GEM_CUDA(cudaMemcpy(w->Ttop, Ttop, n * sizeof(double), on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice));
  return GEM_OK;
}

// ---- conversions ---------------------------------------------------------------------
#define ELEMWISE(name, kern, Fp, Ap)                                                   \
  int name(const gem_grid* g, Fp fluidvars, Ap fluidauxvars, void* stream) {           \
    if (check_grid(g) || !fluidvars || !fluidauxvars) return set_err(GEM_EINVAL, "null argument"); \
    Blocks B = blocks(g, const_cast<double*>(fluidvars), const_cast<double*>(fluidauxvars)); \
    kern<<<grid_for(g->dev.d.ng, 256), 256, 0, S(stream)>>>(B);                        \
    GEM_LAUNCHED(#kern);                                                               \
    return GEM_OK;                                                                     \
  }
ELEMWISE(gem_v12rhov1_dev, k_v12rhov1, const double*, double*)
ELEMWISE(gem_T2rhoe_dev, k_T2rhoe, const double*, double*)
ELEMWISE(gem_rhov12v1_dev, k_rhov12v1, double*, const double*)
ELEMWISE(gem_rhoe2T_dev, k_rhoe2T, double*, const double*)
#undef ELEMWISE

int gem_set_global_boundaries_allspec_dev(const gem_grid* g, double* fluidvars, double* fluidauxvars,
                                          const gem_work* w, int lsp, void* stream) {
  if (check_grid(g) || !fluidvars || !fluidauxvars || !w) return set_err(GEM_EINVAL, "null argument");
  if (lsp < 1 || lsp > LSP) return set_err(GEM_EINVAL, "number of global boundaries must be in 1..%d", LSP);
  if (g->dev.d.lx1 < 3) return set_err(GEM_EINVAL, "lx1 must be >= 3 for the x1 boundary extrapolation");
  return launch_ghost_fill(g, blocks(g, fluidvars, fluidauxvars), w->vs1i, lsp, false, S(stream));
}

int gem_halo_fluidvars_dev(const gem_grid* g, double* fluidvars, double* fluidauxvars, void* stream) {
  if (check_grid(g) || !fluidvars || !fluidauxvars) return set_err(GEM_EINVAL, "null argument");
  if (!g->dev.flagper) return GEM_OK;
  if (g->dev.d.lx3 < 2) return set_err(GEM_EINVAL, "periodic x3 needs lx3 >= 2");
  const long long n = (long long)(g->dev.d.lx1 + 4) * g->dev.d.lx2 * LSP;
  k_halo_wrap<<<grid_for(n, 128), 128, 0, S(stream)>>>(g->dev, blocks(g, fluidvars, fluidauxvars), 1);
  GEM_LAUNCHED("k_halo_wrap");
  return GEM_OK;
}

int gem_halo_allparams_dev(const gem_grid* g, double* fluidvars, double* fluidauxvars, void* stream) {
  if (check_grid(g) || !fluidvars || !fluidauxvars) return set_err(GEM_EINVAL, "null argument");
  if (!g->dev.flagper) return GEM_OK;
  if (g->dev.d.lx3 < 2) return set_err(GEM_EINVAL, "periodic x3 needs lx3 >= 2");
  const long long n = (long long)(g->dev.d.lx1 + 4) * g->dev.d.lx2 * LSP;
  k_halo_wrap<<<grid_for(n, 128), 128, 0, S(stream)>>>(g->dev, blocks(g, fluidvars, fluidauxvars), 0);
  GEM_LAUNCHED("k_halo_wrap");
  return GEM_OK;
}

int gem_interface_vels_allspec_dev(const gem_grid* g, const double* fluidvars, gem_work* w, int lsp,
                                   void* stream) {
  if (check_grid(g) || !fluidvars || !w) return set_err(GEM_EINVAL, "null argument");
  if (lsp < 1 || lsp > LSP) return set_err(GEM_EINVAL, "number of interface vels must be in 1..%d", LSP);
  const Dims& d = g->dev.d;
  k_interface_vels<<<dim3(grid_for(nf1(d) + nf2(d) + nf3(d), 256, 4), lsp), 256, 0, S(stream)>>>(
      g->dev, blocks(g, const_cast<double*>(fluidvars), nullptr), w->vs1i, w->vs2i, w->vs3i);
  GEM_LAUNCHED("k_interface_vels");
  return GEM_OK;
}

int gem_sweep_allspec_dev(const gem_grid* g, int dim, int which, double* fluidvars, double* fluidauxvars,
                          const gem_work* w, const double* dt, void* stream) {
  if (check_grid(g) || !fluidvars || !fluidauxvars || !w || !dt) return set_err(GEM_EINVAL, "null argument");
  if (dim < 1 || dim > 3 || which < 0 || which > 2) return set_err(GEM_EINVAL, "dim must be 1..3, which 0..2");
  SweepArgs a;
  a.G = g->dev;
  a.B = blocks(g, fluidvars, fluidauxvars);
  a.vsi = dim == 1 ? w->vs1i : dim == 2 ? w->vs2i : w->vs3i;
  a.vs1i = nullptr;
  a.dtp = dt;
  a.which = which;
  const int nsp = (which == 2) ? LSP : LSP - 1;  // multifluid.f90:55,63,71
  return launch_sweep(g, dim, false, a, nsp, S(stream));
}

int gem_clean_param_dev(const gem_grid* g, int iparm, double* fluidvars, void* stream) {
  if (check_grid(g) || !fluidvars) return set_err(GEM_EINVAL, "null argument");
  if (iparm < 1 || iparm > 3) return set_err(GEM_EINVAL, "non-standard parameter selected in clean_params");
  const long long ng = g->dev.d.ng;
  double* param = fluidvars + (iparm == 1 ? 0 : iparm == 2 ? LSP : 4 * LSP) * ng;
  k_clean_elementwise<<<grid_for(ng, 256), 256, 0, S(stream)>>>(g->dev, param, iparm);
  GEM_LAUNCHED("k_clean_elementwise");
  if (iparm == 2 && g->dev.has_null && (g->dev.gridflag == 0 || g->dev.gridflag == 1)) {
    const long long n = (long long)g->dev.d.lx2 * g->dev.d.lx3 * LSP;
    k_clean_vel_edges<<<grid_for(n, 128), 128, 0, S(stream)>>>(g->dev, param);
    GEM_LAUNCHED("k_clean_vel_edges");
  }
  return GEM_OK;
}

int gem_energy_diffusion_dev(const gem_cfg* cfg, const gem_grid* g, double* fluidvars,
                             const double* electrovars, const gem_work* w, const double* dt, void* stream) {
  if (!cfg || check_grid(g) || !fluidvars || !electrovars || !w || !dt) return set_err(GEM_EINVAL, "null argument");
  if (cfg->diffsolvetype != 1 && cfg->diffsolvetype != 2)
    return set_err(GEM_EINVAL, "Unsupported diffusion solver type/mode: %d. Should be either 1 or 2.", cfg->diffsolvetype);
  if (g->dev.d.lx1 < 4) return set_err(GEM_EINVAL, "diffusion needs lx1 >= 4");
  DiffArgs a;
  a.G = g->dev;
  a.B = blocks(g, fluidvars, nullptr);
  a.J1 = electrovars + 3 * g->dev.d.ng;
  a.nn = w->nn;
  a.Tn = w->Tn;
  a.dtp = dt;
  a.Teinf = cfg->Teinf;
  a.Ttop = w->Ttop;
  if (int rc0 = work_lu(const_cast<gem_work*>(w), g, &a.lu)) return rc0;
  a.solver = cfg->diffsolvetype;
  a.fused = 0;
  int rc = launch_diffusion(g, a, S(stream));
  if (rc) return rc;
  k_diffusion_ghost_floor<<<grid_for(g->dev.d.ng, 256), 256, 0, S(stream)>>>(g->dev, a.B);
  GEM_LAUNCHED("k_diffusion_ghost_floor");
  return GEM_OK;
}

int gem_dt_calc_dev(const gem_grid* g, double tcfl, const double* fluidvars, gem_work* w, double* dt_out,
                    void* stream) {
  if (check_grid(g) || !fluidvars || !w || !dt_out) return set_err(GEM_EINVAL, "null argument");
  cudaStream_t st = S(stream);
  w->timer.record(0, st);
  GEM_CUDA(cudaMemsetAsync(w->acc, 0, 3 * LSP * sizeof(unsigned long long), st));
  Blocks B = blocks(g, const_cast<double*>(fluidvars), nullptr);
  const unsigned nb = (unsigned)std::min<long long>((long long)g->dev.d.lx2 * g->dev.d.lx3, (long long)num_sms() * 8);
  if (g->dev.unit)
    k_dt_reduce<true, 0><<<nb, dim3(32, LSP), 0, st>>>(g->dev, B, w->acc, nullptr);
  else
    k_dt_reduce<false, 0><<<nb, dim3(32, LSP), 0, st>>>(g->dev, B, w->acc, nullptr);
  GEM_LAUNCHED("k_dt_reduce");
  k_dt_finalize<<<1, 32, 0, st>>>(w->acc, tcfl, dt_out);
  GEM_LAUNCHED("k_dt_finalize");
  w->timer.record(1, st);
  return GEM_OK;
}

// One field sweep on a caller-provided field (differentiable path): species 0..nsp-1 of
// the ghosted block f, face velocities v (reference face layout), frank 0 or 1.
int gem_sweep_field_dev(const gem_grid* g, int dim, int frank, int nsp, double* f, const double* v,
                        const double* dt, void* stream) {
  if (check_grid(g) || !f || !v || !dt) return set_err(GEM_EINVAL, "null argument");
  if (dim < 1 || dim > 3 || frank < 0 || frank > 1 || nsp < 1 || nsp > LSP)
    return set_err(GEM_EINVAL, "dim %d / frank %d / nsp %d out of range", dim, frank, nsp);
  SweepArgs a;
  a.G = g->dev;
  Blocks B;
  B.F = f;  // which 0 reads ns(s) = F + s*ng (frank 0); which 1 reads rv(s) = A + s*ng (frank 1)
  B.A = f;
  B.ng = g->dev.d.ng;
  a.B = B;
  a.vsi = v;
  a.vs1i = nullptr;
  a.dtp = dt;
  a.dtp_w = nullptr;
  a.which = (frank == 1 && dim != 1) ? 1 : 0;
  return launch_sweep(g, dim, false, a, nsp, S(stream));
}

int gem_sweep_field_vjp_dev(const gem_grid* g, int dim, int frank, int nsp, const double* f, const double* v,
                            const double* dt, const double* obar, double* fbar, double* vbar, void* stream) {
  if (check_grid(g) || !f || !v || !dt || !obar || !fbar) return set_err(GEM_EINVAL, "null argument");
  if (dim < 1 || dim > 3 || frank < 0 || frank > 1 || nsp < 1 || nsp > LSP)
    return set_err(GEM_EINVAL, "dim %d / frank %d / nsp %d out of range", dim, frank, nsp);
  return launch_sweep_vjp(g, dim, frank, nsp, f, v, dt, obar, fbar, vbar, 0, S(stream));
}

// Vector-Jacobian product of the energy diffusion (differentiable path).
int gem_diffusion_vjp_dev(const gem_cfg* cfg, const gem_grid* g, const double* Ts, const double* ns,
                          const double* electrovars, const gem_work* w, const double* dt, const double* Ybar,
                          double* Tbar, double* nbar, double* Ttop_bar, void* stream) {
  if (!cfg || check_grid(g) || !Ts || !ns || !electrovars || !w || !dt || !Ybar || !Tbar || !nbar)
    return set_err(GEM_EINVAL, "null argument");
  if (cfg->diffsolvetype != 1 && cfg->diffsolvetype != 2)
    return set_err(GEM_EINVAL, "Unsupported diffusion solver type/mode: %d. Should be either 1 or 2.", cfg->diffsolvetype);
  const Dims& d = g->dev.d;
  if (d.lx1 < 4) return set_err(GEM_EINVAL, "lx1=%d: the diffusion needs lx1 >= 4", d.lx1);
  DiffAdjArgs a;
  a.G = g->dev;
  a.T = Ts;
  a.ns = ns;
  a.J1 = electrovars + 3 * d.ng;
  a.nn = w->nn;
  a.Tn = w->Tn;
  a.Ttop = w->Ttop;
  a.Teinf = cfg->Teinf;
  a.dtp = dt;
  a.solver = cfg->diffsolvetype;
  a.Ybar = Ybar;
  a.Tbar = Tbar;
  a.nbar = nbar;
  a.Ttop_bar = Ttop_bar;
  return launch_diffusion_vjp(g, a, S(stream));
}

// dt_calc variant that allocates nothing: its scratch (per-x3-plane partial maxima) is
// the file-scope device array below, whose address is resolved once per device.
int gem_dt_calc_noalloc_dev(const gem_grid* g, double tcfl, const double* fluidvars, double* dt_out,
                            void* stream) {
  if (check_grid(g) || !fluidvars || !dt_out) return set_err(GEM_EINVAL, "null argument");
  const Dims& d = g->dev.d;
  if (d.lx3 > GEM_DT_NOALLOC_MAX_PLANES)
    return set_err(GEM_EINVAL,
                   "gem_dt_calc_noalloc_dev: lx3=%d x3 planes exceed its static scratch of %d planes "
                   "(use gem_dt_calc_dev)",
                   d.lx3, GEM_DT_NOALLOC_MAX_PLANES);
  int dev = 0;
  GEM_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoallocMaxDevices)
    return set_err(GEM_EINVAL, "gem_dt_calc_noalloc_dev: device ordinal %d out of range", dev);
  double* part = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    part = g_noalloc_part_ptr[dev];
    if (!part) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_dt_noalloc_part);
      if (e != cudaSuccess || !p)
        return set_err(GEM_ECUDA, "cudaGetSymbolAddress of the no-alloc dt scratch failed: %s",
                       cudaGetErrorString(e));
      part = static_cast<double*>(p);
      g_noalloc_part_ptr[dev] = part;
    }
  }
  // every partial slot that the finalize reads is written by the reduce: nothing in the
  // scratch has to start at zero
  cudaStream_t st = S(stream);
  Blocks B = blocks(g, const_cast<double*>(fluidvars), nullptr);
  if (g->dev.unit)
    k_dt_reduce_planes<true><<<d.lx3, dim3(32, LSP), 0, st>>>(g->dev, B, part);
  else
    k_dt_reduce_planes<false><<<d.lx3, dim3(32, LSP), 0, st>>>(g->dev, B, part);
  GEM_LAUNCHED("k_dt_reduce_planes");
  k_dt_finalize_planes<<<1, 32, 0, st>>>(part, d.lx3, tcfl, dt_out);
  GEM_LAUNCHED("k_dt_finalize_planes");
  return GEM_OK;
}

int gem_maxcfl_dev(const gem_grid* g, const double* fluidvars, gem_work* w, const double* dt,
                   double* maxcfl_out, void* stream) {
  if (check_grid(g) || !fluidvars || !w || !dt || !maxcfl_out) return set_err(GEM_EINVAL, "null argument");
  cudaStream_t st = S(stream);
  GEM_CUDA(cudaMemsetAsync(w->acc + 24, 0, sizeof(unsigned long long), st));
  Blocks B = blocks(g, const_cast<double*>(fluidvars), nullptr);
  const unsigned nb = (unsigned)std::min<long long>((long long)g->dev.d.lx2 * g->dev.d.lx3, (long long)num_sms() * 8);
  if (g->dev.unit)
    k_dt_reduce<true, 1><<<nb, dim3(32, LSP), 0, st>>>(g->dev, B, w->acc + 24, dt);
  else
    k_dt_reduce<false, 1><<<nb, dim3(32, LSP), 0, st>>>(g->dev, B, w->acc + 24, dt);
  GEM_LAUNCHED("k_dt_reduce");
  k_maxcfl_finalize<<<1, 32, 0, st>>>(w->acc + 24, maxcfl_out);
  GEM_LAUNCHED("k_maxcfl_finalize");
  return GEM_OK;
}

// The fused step; after_fill / after_epi (optional) are recorded once the ghost fill (vs2,
// vs3 final from there on) and the ghost epilogue (ns, vs1, rhovs1 final) are done.
static int fluid_adv_impl(const gem_cfg* cfg, const gem_grid* g, double* fluidvars, double* fluidauxvars,
                          const double* electrovars, gem_work* w, const double* dt, cudaStream_t st,
                          cudaEvent_t after_fill, cudaEvent_t after_epi);

int gem_fluid_adv_dev(const gem_cfg* cfg, const gem_grid* g, double* fluidvars, double* fluidauxvars,
                      const double* electrovars, gem_work* w, const double* dt, void* stream) {
  if (!cfg || check_grid(g) || !fluidvars || !fluidauxvars || !electrovars || !w || !dt)
    return set_err(GEM_EINVAL, "null argument");
  if (cfg->diffsolvetype != 1 && cfg->diffsolvetype != 2)
    return set_err(GEM_EINVAL, "Unsupported diffusion solver type/mode: %d. Should be either 1 or 2.", cfg->diffsolvetype);
  return fluid_adv_impl(cfg, g, fluidvars, fluidauxvars, electrovars, w, dt, S(stream), nullptr, nullptr);
}

static int fluid_adv_impl(const gem_cfg* cfg, const gem_grid* g, double* fluidvars, double* fluidauxvars,
                          const double* electrovars, gem_work* w, const double* dt, cudaStream_t st,
                          cudaEvent_t after_fill, cudaEvent_t after_epi) {
  int rc = check_step(g);
  if (rc) return rc;
  Blocks B = blocks(g, fluidvars, fluidauxvars);
  w->timer.record(1, st);
  // v12rhov1 + T2rhoe + set_global_boundaries + halo_fluidvars (the interior conversions
  // are folded into the x3 sweep)
  rc = launch_ghost_fill(g, B, w->vs1i, LSP, true, st);
  if (rc) return rc;
  if (after_fill) GEM_CUDA(cudaEventRecord(after_fill, st));
  w->timer.record(2, st);
  SweepArgs a;
  a.G = g->dev;
  a.B = B;
  a.vsi = nullptr;
  a.vs1i = w->vs1i;
  a.dtp = dt;
  a.which = 0;
  if ((rc = launch_sweep(g, 3, true, a, LSP, st))) return rc;
  w->timer.record(3, st);
  if ((rc = launch_sweep(g, 1, true, a, LSP, st))) return rc;
  w->timer.record(4, st);
  if ((rc = launch_sweep(g, 2, true, a, LSP, st))) return rc;
  w->timer.record(5, st);
  k_ghost_epilogue<<<grid_for(ghost_cells(g->dev.d), 256), 256, 0, st>>>(g->dev, B);
  GEM_LAUNCHED("k_ghost_epilogue");
  if (g->dev.has_null && (g->dev.gridflag == 0 || g->dev.gridflag == 1)) {
    const long long n = (long long)g->dev.d.lx2 * g->dev.d.lx3 * LSP;
    k_clean_vel_edges<<<grid_for(n, 128), 128, 0, st>>>(g->dev, fluidvars + LSP * g->dev.d.ng);
    GEM_LAUNCHED("k_clean_vel_edges");
  }
  if (after_epi) GEM_CUDA(cudaEventRecord(after_epi, st));
  DiffArgs d;
  d.G = g->dev;
  d.B = B;
  d.J1 = electrovars + 3 * g->dev.d.ng;
  d.nn = w->nn;
  d.Tn = w->Tn;
  d.dtp = dt;
  d.Teinf = cfg->Teinf;
  d.Ttop = w->Ttop;
  if ((rc = work_lu(w, g, &d.lu))) return rc;
  d.solver = cfg->diffsolvetype;
  d.fused = 1;
  w->timer.record(6, st);
  rc = launch_diffusion(g, d, st);
  if (rc) return rc;
  w->timer.record(7, st);
  if (w->timer.cap > 0) w->timer.step++;
  return GEM_OK;
}

// The advection of the step with compression through the fused kernels: the ghost fill, the
// fused x3 and x1 sweeps, the fused x2 sweep whose epilogue stops after rhov12v1 and
// clean_param(1), (2) (the swept energy densities stay for the compression sub-step), and
// that part of the ghost shell.  Bit for bit what v12rhov1, T2rhoe,
// set_global_boundaries_allspec, halo_fluidvars, interface_vels_allspec, the nine sweeps,
// halo_allparams, rhov12v1 and clean_param(1), (2) leave for the compression sub-step (which
// converts rhoes and resets the ghost temperatures before anything reads them).  Needs what
// the fused step needs (check_step).
static int advection_keepre(const gem_grid* g, double* fluidvars, double* fluidauxvars, gem_work* w,
                            const double* dt, cudaStream_t st) {
  const Dims& d = g->dev.d;
  Blocks B = blocks(g, fluidvars, fluidauxvars);
  int rc = launch_ghost_fill(g, B, w->vs1i, LSP, true, st);
  if (rc) return rc;
  SweepArgs a;
  a.G = g->dev;
  a.B = B;
  a.vsi = nullptr;
  a.vs1i = w->vs1i;
  a.dtp = dt;
  a.dtp_w = nullptr;
  a.which = 0;
  if ((rc = launch_sweep(g, 3, true, a, LSP, st))) return rc;
  if ((rc = launch_sweep(g, 1, true, a, LSP, st))) return rc;
  const dim3 block(32, LSP), grid((d.lx1 + 31) / 32, d.lx3);
  if (g->dev.unit)
    k_sweep_march<2, true, true, 2, true><<<grid, block, 0, st>>>(a);
  else
    k_sweep_march<2, false, true, 2, true><<<grid, block, 0, st>>>(a);
  GEM_LAUNCHED("k_sweep_march");
  k_ghost_epilogue<true><<<grid_for(ghost_cells(d), 256), 256, 0, st>>>(g->dev, B);
  GEM_LAUNCHED("k_ghost_epilogue");
  if (g->dev.has_null && (g->dev.gridflag == 0 || g->dev.gridflag == 1)) {
    const long long n = (long long)d.lx2 * d.lx3 * LSP;
    k_clean_vel_edges<<<grid_for(n, 128), 128, 0, st>>>(g->dev, fluidvars + LSP * d.ng);
    GEM_LAUNCHED("k_clean_vel_edges");
  }
  return GEM_OK;
}

// energy_diffusion, clean_param(3) and T2rhoe of the step with compression: the diffusion's
// fused store applies clean_param(3) and T2rhoe to the interior cells and one pass over the
// ghost shell does the rest; bit for bit the three routines in sequence.  Needs lx1 >= 4.
static int diffusion_clean_T2rhoe(const gem_cfg* cfg, const gem_grid* g, double* fluidvars, double* fluidauxvars,
                                  const double* electrovars, gem_work* w, const double* dt, cudaStream_t st) {
  DiffArgs a;
  a.G = g->dev;
  a.B = blocks(g, fluidvars, fluidauxvars);
  a.J1 = electrovars + 3 * g->dev.d.ng;
  a.nn = w->nn;
  a.Tn = w->Tn;
  a.dtp = dt;
  a.Teinf = cfg->Teinf;
  a.Ttop = w->Ttop;
  int rc = work_lu(w, g, &a.lu);
  if (rc) return rc;
  a.solver = cfg->diffsolvetype;
  a.fused = 1;
  if ((rc = launch_diffusion(g, a, st))) return rc;
  k_ghost_T100<<<grid_for(ghost_cells(g->dev.d), 256), 256, 0, st>>>(g->dev, a.B);
  GEM_LAUNCHED("k_ghost_T100");
  return GEM_OK;
}

int gem_work_phase_timing(gem_work* w, int max_steps) {
  if (!w || max_steps < 0) return set_err(GEM_EINVAL, "bad argument");
  for (cudaEvent_t e : w->timer.ev) cudaEventDestroy(e);
  w->timer.ev.clear();
  w->timer.cap = 0;
  w->timer.step = 0;
  if (max_steps == 0) return GEM_OK;
  w->timer.ev.resize((size_t)max_steps * (NPHASE + 1));
  for (auto& e : w->timer.ev) GEM_CUDA(cudaEventCreate(&e));
  w->timer.cap = max_steps;
  return GEM_OK;
}

int gem_work_phase_times(gem_work* w, double* ms, int nphase_max, int* nphase, int* nsteps) {
  if (!w || !ms) return set_err(GEM_EINVAL, "bad argument");
  const int ns = (int)std::min<long long>(w->timer.step, w->timer.cap);
  const int np = std::min(nphase_max, NPHASE);
  for (int p = 0; p < np; ++p) ms[p] = 0.0;
  for (int k = 0; k < ns; ++k) {
    const cudaEvent_t* e = &w->timer.ev[(size_t)k * (NPHASE + 1)];
    GEM_CUDA(cudaEventSynchronize(e[NPHASE]));
    for (int p = 0; p < np; ++p) {
      float t = 0.f;
      GEM_CUDA(cudaEventElapsedTime(&t, e[p], e[p + 1]));
      ms[p] += t;
    }
  }
  for (int p = 0; p < np; ++p) ms[p] = ns ? ms[p] / ns : 0.0;
  if (nphase) *nphase = np;
  if (nsteps) *nsteps = ns;
  w->timer.step = 0;
  return GEM_OK;
}

int gem_fluid_adv_host(const gem_cfg* cfg, const gem_grid* g, double* fluidvars, double* fluidauxvars,
                       const double* electrovars, gem_work* w, double* dt_inout, void* stream) {
  if (!cfg || check_grid(g) || !fluidvars || !fluidauxvars || !electrovars || !w || !dt_inout)
    return set_err(GEM_EINVAL, "null argument");
  const size_t ng = (size_t)g->dev.d.ng;
  const size_t nF = ng * 5 * LSP, nA = ng * (2 * LSP + 9), nE = ng * 7;
  if (!w->F) {
    if (cudaMalloc(&w->F, nF * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&w->A, nA * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&w->E, nE * sizeof(double)) != cudaSuccess)
      return set_err(GEM_ENOMEM, "device staging allocation failed");
    w->nF = nF;
    w->nA = nA;
    w->nE = nE;
  }
  cudaStream_t st = S(stream);
  // Only what the step reads goes in: fluidvars and J1 (electrovars field 4).  rhovs1 and
  // rhoes are recomputed from ns, vs1, Ts over every cell (v12rhov1/T2rhoe), the 9 MHD
  // scalars and the other electrovars fields are not touched.
  GEM_CUDA(cudaMemcpyAsync(w->F, fluidvars, nF * sizeof(double), cudaMemcpyHostToDevice, st));
  GEM_CUDA(cudaMemcpyAsync(w->E + 3 * ng, electrovars + 3 * ng, ng * sizeof(double), cudaMemcpyHostToDevice, st));
  int rc;
  if (*dt_inout < 0) {
    if ((rc = gem_dt_calc_dev(g, cfg->tcfl, w->F, w, w->dt, stream))) return rc;
  } else {
    GEM_CUDA(cudaMemcpyAsync(w->dt, dt_inout, sizeof(double), cudaMemcpyHostToDevice, st));
  }
  // ... and only what it writes comes out: fluidvars and rhovs1|rhoes, each block as soon as
  // the step is done with it, on a copy stream beside the step's kernels: vs2, vs3 after the
  // ghost fill, ns, vs1 and rhovs1 after the ghost epilogue (the diffusion reads ns only),
  // Ts and rhoes at the end
  if (!w->cs) {
    GEM_CUDA(cudaStreamCreateWithFlags(&w->cs, cudaStreamNonBlocking));
    for (auto& e : w->ev) GEM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  if (cfg->diffsolvetype != 1 && cfg->diffsolvetype != 2)
    return set_err(GEM_EINVAL, "Unsupported diffusion solver type/mode: %d. Should be either 1 or 2.", cfg->diffsolvetype);
  if ((rc = fluid_adv_impl(cfg, g, w->F, w->A, w->E, w, w->dt, st, w->ev[0], w->ev[1]))) return rc;
  GEM_CUDA(cudaEventRecord(w->ev[2], st));
  const size_t blk = ng * LSP;  // one field of all species
  GEM_CUDA(cudaStreamWaitEvent(w->cs, w->ev[0], 0));
  {
    // vs2 and vs3 change only in their ghost cells (the ghost fill), so only their ghost shell
    // comes out, as strided copies over the 14 blocks -- the x3 ghost planes, the x2 ghost
    // rows of every plane and the x1 ghost cells of every column -- and the host keeps its
    // unchanged interior
    const Dims& d = g->dev.d;
    const size_t s2 = (size_t)d.lx1 + 4, s3 = s2 * (d.lx2 + 4), nb = 2 * LSP, D = sizeof(double);
    double* hb = fluidvars + 2 * blk;
    const double* db = w->F + 2 * blk;
    const size_t o3 = (size_t)(d.lx3 + 2) * s3, o2 = (size_t)(d.lx2 + 2) * s2, o1 = (size_t)d.lx1 + 2;
    const auto D2H = cudaMemcpyDeviceToHost;
    GEM_CUDA(cudaMemcpy2DAsync(hb, ng * D, db, ng * D, 2 * s3 * D, nb, D2H, w->cs));
    GEM_CUDA(cudaMemcpy2DAsync(hb + o3, ng * D, db + o3, ng * D, 2 * s3 * D, nb, D2H, w->cs));
    GEM_CUDA(cudaMemcpy2DAsync(hb, s3 * D, db, s3 * D, 2 * s2 * D, nb * (d.lx3 + 4), D2H, w->cs));
    GEM_CUDA(cudaMemcpy2DAsync(hb + o2, s3 * D, db + o2, s3 * D, 2 * s2 * D, nb * (d.lx3 + 4), D2H, w->cs));
    GEM_CUDA(cudaMemcpy2DAsync(hb, s2 * D, db, s2 * D, 2 * D, nb * (d.lx2 + 4) * (d.lx3 + 4), D2H, w->cs));
    GEM_CUDA(cudaMemcpy2DAsync(hb + o1, s2 * D, db + o1, s2 * D, 2 * D, nb * (d.lx2 + 4) * (d.lx3 + 4), D2H, w->cs));
  }
  GEM_CUDA(cudaStreamWaitEvent(w->cs, w->ev[1], 0));
  GEM_CUDA(cudaMemcpyAsync(fluidvars, w->F, 2 * blk * sizeof(double), cudaMemcpyDeviceToHost, w->cs));
  GEM_CUDA(cudaMemcpyAsync(fluidauxvars, w->A, blk * sizeof(double), cudaMemcpyDeviceToHost, w->cs));
  GEM_CUDA(cudaStreamWaitEvent(w->cs, w->ev[2], 0));
  GEM_CUDA(cudaMemcpyAsync(fluidvars + 4 * blk, w->F + 4 * blk, blk * sizeof(double), cudaMemcpyDeviceToHost, w->cs));
  GEM_CUDA(cudaMemcpyAsync(fluidauxvars + blk, w->A + blk, blk * sizeof(double), cudaMemcpyDeviceToHost, w->cs));
  GEM_CUDA(cudaMemcpyAsync(dt_inout, w->dt, sizeof(double), cudaMemcpyDeviceToHost, w->cs));
  GEM_CUDA(cudaEventRecord(w->ev[3], w->cs));
  GEM_CUDA(cudaStreamWaitEvent(st, w->ev[3], 0));
  GEM_CUDA(cudaStreamSynchronize(st));
  return GEM_OK;
}

int gem_check_finite(const gem_grid* g, const double* fluidvars, gem_work* w, long long* count, void* stream) {
  if (check_grid(g) || !fluidvars || !w || !count) return set_err(GEM_EINVAL, "null argument");
  cudaStream_t st = S(stream);
  GEM_CUDA(cudaMemsetAsync(w->acc + 28, 0, sizeof(unsigned long long), st));
  k_count_nonfinite<<<grid_for(nci(g->dev.d), 256, 4), 256, 0, st>>>(
      g->dev, blocks(g, const_cast<double*>(fluidvars), nullptr), w->acc + 28);
  GEM_LAUNCHED("k_count_nonfinite");
  unsigned long long c = 0;
  GEM_CUDA(cudaMemcpyAsync(&c, w->acc + 28, sizeof(c), cudaMemcpyDeviceToHost, st));
  GEM_CUDA(cudaStreamSynchronize(st));
  *count = (long long)c;
  return c ? GEM_ENONFINITE : GEM_OK;
}

}  // extern "C"

#include "gem_batch.cuh"
#include "gem_adjoint.cuh"
#include "gem_compression_dev.cuh"
#include "gem_sources_dev.cuh"
#include "gem_rates_dev.cuh"
#include "gem_fullstep_dev.cuh"
#include "gem_clock_dev.cuh"
