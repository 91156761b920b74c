// ensemble.cu — batched ensembles of uneven blocks (FP32 perturbation form).
//
// Many independent mesh blocks (ensemble members of different sizes, same
// physics) advance together: each sweep of an RK stage is ONE persistent
// launch over all members, whose CTAs pull (member, tile) work items from a
// device counter until the queue is drained, so small and large members
// share the SMs without a launch per member and without tail effects at
// member boundaries.  Per stage: x1 sweep, x2 sweep, x3 sweep, implicit
// column, implicit finish, boundary fills — six to seven launches for the
// whole ensemble.  dt is per member and stays on the device (a per-member CFL
// reduction), so a whole step can be captured in one CUDA graph.
//
// The tile shapes (x1 columns per CTA, march segment length, implicit column
// block, persistent CTAs per SM) are parameters of the plan; the project's
// autotuner (snapy_linfel_b200/ensemble.py) times candidates on the live
// ensemble and keeps the fastest.
//
// Reference: each member is one snapy MeshBlock (MeshBlockImpl::forward,
// src/mesh/meshblock.cpp:577-786); the reference has no batched form.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "kernels.cuh"

using namespace snapb;

namespace snapb {

// per-member CFL reduction over the interior: min over cells of
// dx_d / (|v_d| + cs) for the used directions, atomically into slots[3m + d]
__global__ void __launch_bounds__(256) k_cfl32_batch(const Member32* __restrict__ mem, Phys p,
                                                     WorkQueue q,
                                                     unsigned long long* __restrict__ slots,
                                                     int use1, int use2, int use3) {
  __shared__ double red[3][8];
  int m;
  int64_t tile;
  while (queue_next(q, m, tile)) {
    const Geo& g = mem[m].g;
    const float* w = mem[m].b.w;
    const float* rbf = mem[m].b.rbf;
    const float* pbf = mem[m].b.pbf;
    const int ni = g.iu - g.il + 1, nj = g.ju - g.jl + 1, nk = g.ku - g.kl + 1;
    const int64_t n = (int64_t)ni * nj * nk;
    const float gamma = (float)p.gammad;
    float a[3] = {0.f, 0.f, 0.f};
    const int64_t t0 = tile * kCflItem;
    for (int64_t t = t0 + threadIdx.x; t < min(t0 + kCflItem, n); t += blockDim.x) {
      int i = g.il + umod(t, ni);
      int j = g.jl + umod(udiv(t, ni), nj);
      int k = g.kl + udiv(t, (int64_t)ni * nj);
      int64_t o = (int64_t)k * g.s3 + (int64_t)j * g.s2 + i;
      cfl32_speeds(w, g.sv, o, rbf[i], pbf[i], gamma, a);
    }
    double m1, m2, m3;
    cfl32_limits(g, use1, use2, use3, a, m1, m2, m3);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      m1 = fmin(m1, __shfl_xor_sync(0xffffffffu, m1, o));
      m2 = fmin(m2, __shfl_xor_sync(0xffffffffu, m2, o));
      m3 = fmin(m3, __shfl_xor_sync(0xffffffffu, m3, o));
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
      red[0][wid] = m1;
      red[1][wid] = m2;
      red[2][wid] = m3;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
      double x = 1.7e308;
      for (int k = 0; k < (int)(blockDim.x >> 5); ++k) x = fmin(x, red[threadIdx.x][k]);
      atomicMin(&slots[3 * m + threadIdx.x], (unsigned long long)__double_as_longlong(x));
    }
  }
}

// dt_m = f * min(used slots of m)
__global__ void k_cfl_batch_final(const unsigned long long* slots, int M, int use1, int use2,
                                  int use3, double f, double* dts) {
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= M) return;
  double d1 = use1 ? __longlong_as_double((long long)slots[3 * m]) : 1.e9;
  double d2 = use2 ? __longlong_as_double((long long)slots[3 * m + 1]) : 1.e9;
  double d3 = use3 ? __longlong_as_double((long long)slots[3 * m + 2]) : 1.e9;
  dts[m] = f * fmin(d1, fmin(d2, d3));
}

__global__ void k_fill_u64(unsigned long long* p, int n, unsigned long long v) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) p[k] = v;
}

}  // namespace snapb

// ---------------------------------------------------------------------------
// host plan
// ---------------------------------------------------------------------------
enum Phase {
  PH_X1 = 0, PH_X1REV, PH_X2, PH_X3, PH_VCOL, PH_VFIN, PH_VFUSED, PH_VCR, PH_BCU, PH_BCS, PH_CFL,
  PH_COUNT
};

// vic_kernel values of the tuning: the implicit-solve variants
constexpr int kVicColumn = 0, kVicCyclic = 1, kVicFused = 2;

struct snapb_ensemble {
  std::vector<snapb_member_f32> in;
  std::vector<Member32> mem;
  snapb_ensemble_tuning tune;
  Phys p;
  snapb_hydro_config cfg0;
  int M = 0;
  bool a1 = false, a2 = false, a3 = false;
  int use1 = 0, use2 = 0, use3 = 0;
  int sms = 148;
  size_t x1_smem = 0;
  int x1_cols = 8;  // x1 tile width (columns) of every member
  int x1_nc1 = 1;   // longest member column (x1 cells with ghosts): the x1 tile layout
  int vic_kernel = kVicColumn;  // the implicit-solve variant in use
  int max_layers = 0;           // longest member column (cyclic reduction's shared memory)
  std::vector<int64_t> prefix[PH_COUNT];
  // device layout (offsets into the bound workspace)
  size_t o_mem = 0, o_prefix = 0, o_counter = 0, o_dts = 0, o_slots = 0, total = 0;
  char* ws = nullptr;
};

namespace {

int efail(int code, const std::string& msg) { return internal_fail(code, msg); }

size_t al(size_t x) { return (x + 255) & ~(size_t)255; }

int cuda_e(cudaError_t e, const char* where) {
  if (e == cudaSuccess) return SNAPB_OK;
  return efail(SNAPB_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

bool same_physics(const snapb_hydro_config& a, const snapb_hydro_config& b) {
  return a.nghost == b.nghost && a.nvar == b.nvar && a.nscalar == b.nscalar &&
         a.gammad == b.gammad && a.rgas == b.rgas && a.recon1_type == b.recon1_type &&
         a.recon1_shock == b.recon1_shock && a.recon1_scale == b.recon1_scale &&
         a.recon23_type == b.recon23_type && a.recon23_shock == b.recon23_shock &&
         a.recon23_scale == b.recon23_scale && a.scalar_recon_type == b.scalar_recon_type &&
         a.scalar_recon_scale == b.scalar_recon_scale && a.riemann == b.riemann &&
         a.implicit_scheme == b.implicit_scheme && a.grav1 == b.grav1 && a.grav2 == b.grav2 &&
         a.grav3 == b.grav3 && a.non_hydrostatic == b.non_hydrostatic &&
         a.nu_iso == b.nu_iso && a.kappa_iso == b.kappa_iso &&
         a.disable_flux[0] == b.disable_flux[0] && a.disable_flux[1] == b.disable_flux[1] &&
         a.disable_flux[2] == b.disable_flux[2] && (a.nx1 > 1) == (b.nx1 > 1) &&
         (a.nx2 > 1) == (b.nx2 > 1) && (a.nx3 > 1) == (b.nx3 > 1);
}

// tile counts and per-member tile shapes for the current tuning
int plan(snapb_ensemble* e) {
  const auto& t = e->tune;
  e->x1_smem = 0;
  for (auto& v : e->prefix) v.assign(e->M + 1, 0);
  for (int m = 0; m < e->M; ++m) {
    Member32& mb = e->mem[m];
    const Geo& g = mb.g;
    const int nvt = 5 + e->p.nscalar;
    // x1: columns per tile
    size_t per = x1_smem32_per_column(g, nvt);
    int C = t.x1_columns > 0 ? t.x1_columns : (int)std::min<size_t>(8, (96 * 1024) / per);
    C = x1_columns_pow2(std::max(1, std::min<int>(C, (int)((200 * 1024) / per))));
    mb.x1_cols = C;
    int64_t ncol1 = (int64_t)g.nc2 * g.nc3;
    // march: 128 lines per tile, segments of seglen faces
    int ni = g.iu - g.il + 1;
    int64_t lines2 = (int64_t)ni * (g.ku - g.kl + 1), lines3 = (int64_t)ni * (g.ju - g.jl + 1);
    int seg = t.march_segment > 0 ? t.march_segment : 32;
    mb.seglen2 = seg;
    mb.nseg2 = (g.nx2 + seg - 1) / seg;
    mb.seglen3 = seg;
    mb.nseg3 = (g.nx3 + seg - 1) / seg;
    int64_t ncolv = (int64_t)(g.ju - g.jl + 1) * (g.ku - g.kl + 1);
    mb.vic_cols = t.vic_block > 0 ? t.vic_block : 64;
    int64_t tiles[PH_COUNT] = {0};
    tiles[PH_X1] = e->a1 ? (ncol1 + C - 1) / C : 0;
    tiles[PH_X1REV] = e->a1 && e->p.grav1 != 0.
                          ? (ncol1 * 2 * g.ng + kRevisionItem - 1) / kRevisionItem : 0;
    tiles[PH_X2] = e->a2 ? ((lines2 + 127) / 128) * mb.nseg2 : 0;
    tiles[PH_X3] = e->a3 ? ((lines3 + 127) / 128) * mb.nseg3 : 0;
    tiles[PH_VCOL] = e->p.implicit_scheme ? (ncolv + mb.vic_cols - 1) / mb.vic_cols : 0;
    const int fl = vic_finish_layers32(e->p);
    tiles[PH_VFIN] = e->p.implicit_scheme
                         ? ((ncolv + kVicFinishCols - 1) / kVicFinishCols) * ((g.nx1 + fl - 1) / fl)
                         : 0;
    const int fc = vicf_tile_columns();
    tiles[PH_VFUSED] = e->p.implicit_scheme ? (ncolv + fc - 1) / fc : 0;
    tiles[PH_VCR] = e->p.implicit_scheme ? ncolv : 0;  // one column per tile
    // ghost-shell cells, kShellItem per tile (same count as bc_shell_slots)
    const int64_t nj = g.ju - g.jl + 1, nk = g.ku - g.kl + 1;
    const int64_t shell = (g.nc1 > 1 ? nj * nk * 2 * g.ng : 0) +
                          ((g.nc3 > 1 ? (int64_t)2 * g.ng * g.nc2 : 0) +
                           (g.nc2 > 1 ? nk * 2 * g.ng : 0)) * g.nc1;
    tiles[PH_BCU] = (shell + kShellItem - 1) / kShellItem;
    tiles[PH_BCS] = e->p.nscalar ? (shell + kShellItem - 1) / kShellItem : 0;
    int64_t ncell = (int64_t)(g.iu - g.il + 1) * (g.ju - g.jl + 1) * (g.ku - g.kl + 1);
    tiles[PH_CFL] = (ncell + kCflItem - 1) / kCflItem;
    for (int ph = 0; ph < PH_COUNT; ++ph) e->prefix[ph][m + 1] = e->prefix[ph][m] + tiles[ph];
  }
  // one x1 tile width for the ensemble (the CTA size of the x1 launch): the
  // smallest member choice, then the tile counts and shared memory from it
  e->x1_cols = 16;
  e->x1_nc1 = 1;
  for (const Member32& mb : e->mem) {
    e->x1_cols = std::min(e->x1_cols, mb.x1_cols);
    e->x1_nc1 = std::max(e->x1_nc1, mb.g.nc1);
  }
  for (int m = 0; m < e->M; ++m) {
    Member32& mb = e->mem[m];
    mb.x1_cols = e->x1_cols;
    const int64_t ncol1 = (int64_t)mb.g.nc2 * mb.g.nc3;
    const int64_t n1 = e->a1 ? (ncol1 + e->x1_cols - 1) / e->x1_cols : 0;
    e->prefix[PH_X1][m + 1] = e->prefix[PH_X1][m] + n1;
  }
  e->x1_smem = x1_smem32_bytes(e->x1_nc1, 5 + e->p.nscalar, e->x1_cols);
  if (e->x1_smem > 200 * 1024) return efail(SNAPB_ERR_ARG, "ensemble: x1 tile too large");
  // implicit solve: cyclic reduction only when every member is in its range
  e->max_layers = 0;
  bool cr_ok = true;
  for (const Member32& mb : e->mem) {
    e->max_layers = std::max(e->max_layers, mb.g.nx1);
    cr_ok = cr_ok && vic_cr_applies(mb.g, e->p);
  }
  if (t.vic_kernel < 0 || t.vic_kernel > kVicFused)
    return efail(SNAPB_ERR_ARG, "ensemble: vic_kernel in [0, 2]");
  e->vic_kernel = t.vic_kernel == kVicCyclic ? (cr_ok ? kVicCyclic : kVicColumn) : t.vic_kernel;
  size_t o = 0;
  e->o_mem = o;
  o = al(o + sizeof(Member32) * e->M);
  e->o_prefix = o;
  o = al(o + sizeof(int64_t) * (e->M + 1) * PH_COUNT);
  e->o_counter = o;
  o = al(o + sizeof(unsigned long long) * 32);
  e->o_dts = o;
  o = al(o + sizeof(double) * e->M);
  e->o_slots = o;
  o = al(o + sizeof(unsigned long long) * 3 * e->M);
  e->total = o;
  return SNAPB_OK;
}

int upload(snapb_ensemble* e, cudaStream_t st) {
  if (!e->ws) return efail(SNAPB_ERR_ARG, "ensemble: no workspace bound");
  // every member's dt points at its slot of the ensemble's dt array
  double* dts = reinterpret_cast<double*>(e->ws + e->o_dts);
  for (int m = 0; m < e->M; ++m) e->mem[m].b.dt = dts + m;
  std::vector<int64_t> pf((size_t)(e->M + 1) * PH_COUNT);
  for (int ph = 0; ph < PH_COUNT; ++ph)
    std::copy(e->prefix[ph].begin(), e->prefix[ph].end(), pf.begin() + (size_t)ph * (e->M + 1));
  cudaError_t c = cudaMemcpyAsync(e->ws + e->o_mem, e->mem.data(), sizeof(Member32) * e->M,
                                  cudaMemcpyHostToDevice, st);
  if (c == cudaSuccess)
    c = cudaMemcpyAsync(e->ws + e->o_prefix, pf.data(), sizeof(int64_t) * pf.size(),
                        cudaMemcpyHostToDevice, st);
  if (c == cudaSuccess) c = cudaStreamSynchronize(st);  // pageable sources
  return cuda_e(c, "ensemble upload");
}

WorkQueue queue(const snapb_ensemble* e, int ph) {
  WorkQueue q;
  q.prefix = reinterpret_cast<const int64_t*>(e->ws + e->o_prefix) + (size_t)ph * (e->M + 1);
  q.M = e->M;
  q.counter = reinterpret_cast<unsigned long long*>(e->ws + e->o_counter) + ph;
  return q;
}

PersistGrid pgrid(const snapb_ensemble* e, int ph) {
  PersistGrid g;
  g.sms = e->sms;
  g.cap = e->tune.ctas_per_sm;
  g.tiles = e->prefix[ph][e->M];
  return g;
}

}  // namespace

extern "C" {

int snapb_ensemble_create(const snapb_member_f32* members, int n,
                          const snapb_ensemble_tuning* tune, snapb_ensemble** out) {
  if (!out) return efail(SNAPB_ERR_ARG, "ensemble_create: null output");
  *out = nullptr;
  if (!members || n < 1) return efail(SNAPB_ERR_ARG, "ensemble_create: no members");
  auto* e = new snapb_ensemble();
  e->in.assign(members, members + n);
  e->M = n;
  e->cfg0 = members[0].cfg;
  std::memset(&e->tune, 0, sizeof(e->tune));
  if (tune) e->tune = *tune;
  for (int m = 0; m < n; ++m) {
    const snapb_member_f32& in = members[m];
    if (const char* er = internal_check_config(&in.cfg)) {
      delete e;
      return efail(SNAPB_ERR_ARG, "ensemble_create: member " + std::to_string(m) + ": " + er);
    }
    if (!same_physics(in.cfg, e->cfg0)) {
      delete e;
      return efail(SNAPB_ERR_ARG, "ensemble_create: member " + std::to_string(m) +
                                      " differs from member 0 in physics or active axes");
    }
    if (in.cfg.nu_iso > 0. || in.cfg.kappa_iso > 0. ||
        (in.cfg.non_hydrostatic != 1. && in.cfg.nx1 > 1)) {
      delete e;
      return efail(SNAPB_ERR_ARG, "ensemble_create: diffusion and non_hydrostatic < 1 are "
                                  "not batched");
    }
    if (!in.u || !in.u0 || !in.w || !in.workspace ||
        in.workspace_bytes < workspace_size_f32_of(in.cfg) ||
        (in.cfg.nscalar > 0 && (!in.s || !in.s0 || (in.cfg.implicit_scheme && !in.r)))) {
      delete e;
      return efail(SNAPB_ERR_ARG, "ensemble_create: member " + std::to_string(m) +
                                      " lacks a state pointer or an FP32 workspace");
    }
    Member32 mb;
    std::memset(&mb, 0, sizeof(mb));
    mb.g = make_geo(in.cfg);
    mb.b = bufs32_of(in.cfg, in.workspace);
    mb.b.u = in.u;
    mb.b.u0 = in.u0;
    mb.b.w = in.w;
    mb.b.s = in.s;
    mb.b.s0 = in.s0;
    mb.b.r = in.cfg.implicit_scheme ? in.r : nullptr;
    mb.b.write_du = in.cfg.implicit_scheme ? 1 : 0;
    mb.b.vic_du_only = 0;
    for (int k = 0; k < 6; ++k) mb.bc[k] = in.cfg.bc[k];
    e->mem.push_back(mb);
  }
  e->p = make_phys(e->cfg0);
  Geo g0 = make_geo(e->cfg0);
  e->a1 = g0.nc1 > 1;
  e->a2 = g0.nc2 > 1;
  e->a3 = g0.nc3 > 1;
  int scheme = e->p.implicit_scheme;
  e->use1 = e->a1, e->use2 = e->a2, e->use3 = e->a3;
  if (scheme != 0) {
    e->use1 = e->use1 && (!(scheme & 1) || (!e->a3 && !e->a2));
    e->use2 = e->use2 && !((scheme >> 1) & 1);
    e->use3 = e->use3 && !((scheme >> 2) & 1);
  }
  int dev = 0;
  cudaDeviceProp prop;
  if (cudaGetDevice(&dev) == cudaSuccess && cudaGetDeviceProperties(&prop, dev) == cudaSuccess)
    e->sms = prop.multiProcessorCount;
  int rc = plan(e);
  if (rc != SNAPB_OK) {
    delete e;
    return rc;
  }
  *out = e;
  return SNAPB_OK;
}

size_t snapb_ensemble_workspace_size(const snapb_ensemble* e) { return e ? e->total : 0; }

int snapb_ensemble_bind(snapb_ensemble* e, void* workspace, size_t workspace_bytes,
                        void* stream) {
  if (!e || !workspace) return efail(SNAPB_ERR_ARG, "ensemble_bind: null argument");
  if (workspace_bytes < e->total)
    return efail(SNAPB_ERR_WORKSPACE, "ensemble_bind: workspace smaller than " +
                                          std::to_string(e->total) + " bytes");
  e->ws = static_cast<char*>(workspace);
  return upload(e, (cudaStream_t)stream);
}

int snapb_ensemble_set_tuning(snapb_ensemble* e, const snapb_ensemble_tuning* tune,
                              void* stream) {
  if (!e || !tune) return efail(SNAPB_ERR_ARG, "ensemble_set_tuning: null argument");
  size_t old_total = e->total;
  snapb_ensemble_tuning keep = e->tune;
  e->tune = *tune;
  int rc = plan(e);
  if (rc == SNAPB_OK && e->total > old_total) rc = efail(SNAPB_ERR_WORKSPACE, "ensemble_set_tuning: plan outgrew the bound workspace");
  if (rc != SNAPB_OK) {
    e->tune = keep;
    plan(e);
    return rc;
  }
  return e->ws ? upload(e, (cudaStream_t)stream) : SNAPB_OK;
}

const double* snapb_ensemble_dt(const snapb_ensemble* e) {
  return (e && e->ws) ? reinterpret_cast<const double*>(e->ws + e->o_dts) : nullptr;
}

int snapb_ensemble_max_time_step_f32(snapb_ensemble* e, double factor, void* stream) {
  if (!e || !e->ws) return efail(SNAPB_ERR_ARG, "ensemble_max_time_step: not bound");
  cudaStream_t st = (cudaStream_t)stream;
  auto* slots = reinterpret_cast<unsigned long long*>(e->ws + e->o_slots);
  unsigned long long big = (unsigned long long)0x7FEFFFFFFFFFFFFFULL;  // DBL_MAX bits
  k_fill_u64<<<(3 * e->M + 255) / 256, 256, 0, st>>>(slots, 3 * e->M, big);
  cudaError_t c = cudaMemsetAsync(e->ws + e->o_counter + PH_CFL * sizeof(unsigned long long), 0,
                                  sizeof(unsigned long long), st);
  if (c != cudaSuccess) return cuda_e(c, "ensemble cfl");
  k_cfl32_batch<<<persistent_grid(k_cfl32_batch, 256, 0, pgrid(e, PH_CFL)), 256, 0, st>>>(
      reinterpret_cast<const Member32*>(e->ws + e->o_mem), e->p, queue(e, PH_CFL), slots, e->use1,
      e->use2, e->use3);
  k_cfl_batch_final<<<(e->M + 127) / 128, 128, 0, st>>>(
      slots, e->M, e->use1, e->use2, e->use3, factor,
      reinterpret_cast<double*>(e->ws + e->o_dts));
  return cuda_e(cudaGetLastError(), "ensemble cfl");
}

int snapb_ensemble_stage_f32(snapb_ensemble* e, int stage, void* stream) {
  if (!e || !e->ws) return efail(SNAPB_ERR_ARG, "ensemble_stage: not bound");
  if (stage < 0 || stage > 2) return efail(SNAPB_ERR_ARG, "ensemble_stage: stage in [0, 2]");
  cudaStream_t st = (cudaStream_t)stream;
  const Member32* mem = reinterpret_cast<const Member32*>(e->ws + e->o_mem);
  cudaError_t c = cudaMemsetAsync(e->ws + e->o_counter, 0, sizeof(unsigned long long) * PH_CFL,
                                  st);
  if (c != cudaSuccess) return cuda_e(c, "ensemble stage");
  const Phys& p = e->p;
  int last = e->a3 ? 3 : (e->a2 ? 2 : 1);
  if (e->a1) {
    ScopedTimer t(SNAPB_K_X1, st);
    if (p.grav1 != 0.)
      c = launch_x1_ghost_revision32_batch(mem, p, queue(e, PH_X1REV), pgrid(e, PH_X1REV), st);
    if (c == cudaSuccess)
      c = launch_x1_32_batch(mem, p, queue(e, PH_X1), stage, last == 1, pgrid(e, PH_X1),
                             e->x1_smem, e->x1_cols, e->x1_nc1, st);
    if (c != cudaSuccess) return cuda_e(c, "ensemble x1");
  }
  if (e->a2) {
    ScopedTimer t(SNAPB_K_X2, st);
    c = launch_march32_batch(2, mem, p, queue(e, PH_X2), stage, !e->a1, last == 2,
                             pgrid(e, PH_X2), st);
    if (c != cudaSuccess) return cuda_e(c, "ensemble x2");
  }
  if (e->a3) {
    ScopedTimer t(SNAPB_K_X3, st);
    c = launch_march32_batch(3, mem, p, queue(e, PH_X3), stage, !e->a1 && !e->a2, true,
                             pgrid(e, PH_X3), st);
    if (c != cudaSuccess) return cuda_e(c, "ensemble x3");
  }
  if (p.implicit_scheme) {
    ScopedTimer t(SNAPB_K_VIC, st);
    if (e->vic_kernel == kVicCyclic) {
      c = launch_vic_cr32_batch(mem, p, queue(e, PH_VCR), stage, pgrid(e, PH_VCR),
                                e->max_layers, st);
    } else if (e->vic_kernel == kVicFused) {
      c = launch_vicf_batch(mem, p, queue(e, PH_VFUSED), stage, pgrid(e, PH_VFUSED), st);
    } else {
      int blk = e->mem.empty() ? 64 : e->mem[0].vic_cols;
      c = launch_vic_column_batch(mem, p, queue(e, PH_VCOL), stage, pgrid(e, PH_VCOL), blk,
                                  e->tune.vic_regs, st);
      if (c == cudaSuccess)
        c = launch_vic_finish_batch(mem, p, queue(e, PH_VFIN), stage, pgrid(e, PH_VFIN), st);
    }
    if (c != cudaSuccess) return cuda_e(c, "ensemble implicit");
  }
  {
    ScopedTimer t(SNAPB_K_BC, st);
    double igm1 = 1.0 / (e->cfg0.gammad - 1.0);
    c = launch_bc32_batch(mem, p, queue(e, PH_BCU), SNAPB_CONSERVED, igm1, pgrid(e, PH_BCU),
                          st);
    if (c == cudaSuccess && p.nscalar)
      c = launch_bc32_batch(mem, p, queue(e, PH_BCS), SNAPB_SCALAR, igm1,
                            pgrid(e, PH_BCS), st);
    if (c != cudaSuccess) return cuda_e(c, "ensemble boundary");
  }
  return SNAPB_OK;
}

void snapb_ensemble_destroy(snapb_ensemble* e) { delete e; }

}  // extern "C"
