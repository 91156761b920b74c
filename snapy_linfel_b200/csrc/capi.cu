// capi.cu — the extern "C" boundary of libsnapb (declared in include/snapb.h).
//
// Validates arguments, carves the caller's workspace, and sequences the
// kernels of a stage on the caller's stream.  No allocation happens here: all
// device memory is owned by the caller.  Errors are returned as status codes
// and described by snapb_last_error(); nothing throws across the boundary.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "kernels.cuh"

using namespace snapb;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

int cuda_status(cudaError_t e, const char* where) {
  if (e == cudaSuccess) return SNAPB_OK;
  return fail(SNAPB_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

const char* check_config(const snapb_hydro_config* c) {
  if (!c) return "null config";
  if (c->nvar != 5) return "nvar must be 5 (ideal gas)";
  if (c->nscalar < 0 || c->nscalar > kMaxScalar) return "nscalar must be in [0, 3]";
  if (c->nghost < 3) return "nghost must be >= 3";
  if (c->nx1 < 1 || c->nx2 < 1 || c->nx3 < 1) return "nx must be >= 1";
  if ((c->nx1 > 1 && c->nx1 < c->nghost) || (c->nx2 > 1 && c->nx2 < c->nghost) ||
      (c->nx3 > 1 && c->nx3 < c->nghost))
    return "number of grids must be greater than the ghost zone size";
  for (int t : {c->recon1_type, c->recon23_type, c->scalar_recon_type})
    if (t < SNAPB_RECON_DC || t > SNAPB_RECON_WENO5) return "unknown reconstruction type";
  if (c->riemann < SNAPB_RIEMANN_ROE || c->riemann > SNAPB_RIEMANN_HLLC)
    return "hydro Riemann solver must be roe, lmars or hllc";
  if (c->implicit_scheme != 0 && c->implicit_scheme != 1 && c->implicit_scheme != 9)
    return "implicit scheme must be 0, 1 or 9";
  if (c->implicit_scheme != 0 && c->nx1 <= 1) return "the implicit scheme needs an active x1";
  if (c->gammad <= 1.0) return "gammad must exceed 1";
  for (int b = 0; b < 6; ++b)
    if (c->bc[b] < SNAPB_BC_CUSTOM || c->bc[b] > SNAPB_BC_OUTFLOW) return "unknown boundary type";
  if (c->nu_iso < 0. || c->kappa_iso < 0.) return "diffusion coefficients must be >= 0";
  if (c->non_hydrostatic < 0. || c->non_hydrostatic > 1.) return "non-hydrostatic outside [0,1]";
  Geo g = make_geo(*c);
  if ((int64_t)(c->nvar + c->nscalar) * g.sv >= ((int64_t)1 << 31))
    return "block too large: (nvar + nscalar) x cells (ghosts included) must stay below 2^31";
  if (g.nc1 > 1 && x1_smem_per_column(g, 5 + c->nscalar) > 200 * 1024)
    return "x1 column too long for one CTA's shared memory";
  return nullptr;
}

struct Layout {
  size_t D, RG, DD, R, M, VIC, VICT, SLOTS, DT, total;
};

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

Layout ws_layout(const snapb_hydro_config& c) {
  Geo g = make_geo(c);
  Phys p = make_phys(c);
  Layout L;
  size_t o = 0, sv = (size_t)g.sv * sizeof(double);
  L.D = o;
  o = align256(o + (size_t)(c.nvar + c.nscalar) * sv);
  L.RG = o;
  bool need_rg = c.grav1 != 0. && p.has_grav && c.non_hydrostatic < 1.;
  o = align256(o + (need_rg ? sv : 0));
  L.DD = o;
  bool diff = c.nu_iso > 0. || c.kappa_iso > 0.;
  o = align256(o + (diff ? (size_t)c.nvar * sv : 0));
  L.R = o;
  o = align256(o + (size_t)c.nscalar * sv);
  L.M = o;
  o = align256(o + (c.implicit_scheme ? sv : 0));
  L.VIC = o;
  o = align256(o + vic_scratch_bytes(g, p));
  L.VICT = o;
  o = align256(o + vic_blocks_bytes(g, p));
  L.SLOTS = o;
  o = align256(o + 8 * sizeof(double));
  L.DT = o;
  o = align256(o + sizeof(double));
  L.total = o;
  return L;
}

// ---- optional per-kernel event timing ----
struct TimedLaunch {
  int kind;
  cudaEvent_t a, b;
};
bool g_timing = false;
std::vector<TimedLaunch> g_launches;

using KernelTimer = snapb::ScopedTimer;

void clear_timings() {
  for (auto& l : g_launches) {
    cudaEventDestroy(l.a);
    cudaEventDestroy(l.b);
  }
  g_launches.clear();
}

template <class P>
P* at(void* ws, size_t off) {
  return reinterpret_cast<P*>(static_cast<char*>(ws) + off);
}

// Runs the sweeps of one stage.  mode 0: RK update of u (and s) in place;
// mode 1: du only (left in D), no scalars.
int run_stage(const snapb_hydro_config* c, int stage, const double* dt, double* u, double* u0,
              double* w, double* s, double* s0, double* r, void* ws, size_t ws_bytes,
              cudaStream_t st, int mode, const char* who) {
  if (const char* e = check_config(c)) return fail(SNAPB_ERR_ARG, std::string(who) + ": " + e);
  if (!dt || !u || !w) return fail(SNAPB_ERR_ARG, std::string(who) + ": null state pointer");
  if (stage < 0 || stage > 2) return fail(SNAPB_ERR_ARG, std::string(who) + ": stage in [0, 2]");
  Layout L = ws_layout(*c);
  if (!ws || ws_bytes < L.total)
    return fail(SNAPB_ERR_WORKSPACE, std::string(who) + ": workspace smaller than " +
                                         std::to_string(L.total) + " bytes");
  Geo g = make_geo(*c);
  Phys p = make_phys(*c);
  if (mode == 1) p.nscalar = 0;
  if (mode == 0 && !u0) return fail(SNAPB_ERR_ARG, std::string(who) + ": null u0");
  if (p.nscalar > 0 && (!s || !s0))
    return fail(SNAPB_ERR_ARG, std::string(who) + ": scalars need s and s0");
  if (p.nscalar > 0 && p.implicit_scheme != 0 && !r)
    return fail(SNAPB_ERR_ARG, std::string(who) + ": implicit scalar transport needs r");

  StageBufs b;
  std::memset(&b, 0, sizeof(b));
  b.dt = dt;
  b.u = u;
  b.u0 = u0;
  b.w = w;
  b.s = s;
  b.s0 = s0;
  b.r = p.implicit_scheme != 0 ? r : nullptr;
  b.D = at<double>(ws, L.D);
  b.RG = at<double>(ws, L.RG);
  b.DD = at<double>(ws, L.DD);
  b.R = at<double>(ws, L.R);
  b.M = p.implicit_scheme ? at<double>(ws, L.M) : nullptr;
  b.vic = at<double>(ws, L.VIC);
  b.vicT = vic_blocks_bytes(g, p) ? at<double>(ws, L.VICT) : nullptr;
  b.stage = stage;
  rk3_weights(stage, b.wgt0, b.wgt1, b.wgt2);
  b.write_du = (mode == 1 || p.implicit_scheme != 0) ? 1 : 0;
  b.vic_du_only = mode == 1 ? 1 : 0;

  const bool a1 = g.nc1 > 1, a2 = g.nc2 > 1, a3 = g.nc3 > 1;
  const bool diff = p.nu > 0. || p.kappa > 0.;
  if (!a1 && !a2 && !a3) return fail(SNAPB_ERR_ARG, std::string(who) + ": no active axis");
  // the sweep that finishes the cell: the last active axis, unless only x1 is
  // active and diffusion must be added after it
  int last_axis = a3 ? 3 : (a2 ? 2 : 1);
  bool separate_finalize = (last_axis == 1 && diff);
  cudaError_t e;
  {
    KernelTimer t(SNAPB_K_X1, st);
    if (a1)
      e = launch_x1(g, p, b, last_axis == 1 && !separate_finalize, st);
    else
      e = launch_c2p_only(g, p, b, st);
  }
  if (e != cudaSuccess) return cuda_status(e, "x1 sweep");
  if (diff) {
    KernelTimer t(SNAPB_K_DIFF, st);
    e = launch_diffusion(g, p, b, st);
    if (e != cudaSuccess) return cuda_status(e, "diffusion");
  }
  if (a2) {
    KernelTimer t(SNAPB_K_X2, st);
    e = launch_march(2, g, p, b, !a1, last_axis == 2, st);
    if (e != cudaSuccess) return cuda_status(e, "x2 sweep");
  }
  if (a3) {
    KernelTimer t(SNAPB_K_X3, st);
    e = launch_march(3, g, p, b, !a1 && !a2, true, st);
    if (e != cudaSuccess) return cuda_status(e, "x3 sweep");
  }
  if (separate_finalize) {
    KernelTimer t(SNAPB_K_FINAL, st);
    e = launch_finalize(g, p, b, st);
    if (e != cudaSuccess) return cuda_status(e, "finalize");
  }
  if (p.implicit_scheme != 0) {
    KernelTimer t(SNAPB_K_VIC, st);
    e = launch_vic(g, p, b, st);
    if (e != cudaSuccess) return cuda_status(e, "implicit solve");
  }
  if (mode == 0) {
    KernelTimer t(SNAPB_K_BC, st);
    e = launch_bc(g, *c, u, c->nvar, SNAPB_CONSERVED, st);
    if (e != cudaSuccess) return cuda_status(e, "hydro boundary");
    if (p.nscalar > 0) {
      e = launch_bc(g, *c, s, p.nscalar, SNAPB_SCALAR, st);
      if (e != cudaSuccess) return cuda_status(e, "scalar boundary");
    }
  }
  return SNAPB_OK;
}

}  // namespace

namespace snapb {
ScopedTimer::ScopedTimer(int k, cudaStream_t s) : kind(k), st(s) {
  if (!g_timing) return;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, st);
}
ScopedTimer::~ScopedTimer() {
  if (!g_timing || !a) return;
  cudaEventRecord(b, st);
  g_launches.push_back({kind, a, b});
}
const char* internal_check_config(const snapb_hydro_config* c) { return check_config(c); }
int internal_fail(int code, const std::string& msg) { return fail(code, msg); }
}  // namespace snapb

extern "C" {

int snapb_abi_version(void) { return SNAPB_ABI_VERSION; }

const char* snapb_last_error(void) { return g_err.c_str(); }

size_t snapb_workspace_size(const snapb_hydro_config* cfg) {
  if (check_config(cfg)) return 0;
  return ws_layout(*cfg).total;
}

int snapb_cons2prim(const snapb_hydro_config* cfg, const double* u, double* w, void* stream) {
  if (const char* e = check_config(cfg)) return fail(SNAPB_ERR_ARG, std::string("cons2prim: ") + e);
  if (!u || !w) return fail(SNAPB_ERR_ARG, "cons2prim: null pointer");
  return cuda_status(launch_cons2prim(make_geo(*cfg), make_phys(*cfg), u, w, (cudaStream_t)stream),
                     "cons2prim");
}

int snapb_prim2cons(const snapb_hydro_config* cfg, const double* w, double* u, void* stream) {
  if (const char* e = check_config(cfg)) return fail(SNAPB_ERR_ARG, std::string("prim2cons: ") + e);
  if (!u || !w) return fail(SNAPB_ERR_ARG, "prim2cons: null pointer");
  return cuda_status(launch_prim2cons(make_geo(*cfg), make_phys(*cfg), w, u, (cudaStream_t)stream),
                     "prim2cons");
}

int snapb_reconstruct(const snapb_hydro_config* cfg, int dim, int group, const double* w, int nv,
                      double* wlr, void* stream) {
  if (const char* e = check_config(cfg)) return fail(SNAPB_ERR_ARG, std::string("reconstruct: ") + e);
  if (dim < 1 || dim > 3 || group < 0 || group > 1 || nv < 1 || !w || !wlr)
    return fail(SNAPB_ERR_ARG, "reconstruct: bad arguments");
  Geo g = make_geo(*cfg);
  int n = dim == 3 ? g.nc1 : (dim == 2 ? g.nc2 : g.nc3);
  if (n < 7) return fail(SNAPB_ERR_ARG, "reconstruct: axis too short (il > iu)");
  return cuda_status(launch_reconstruct(g, make_phys(*cfg), dim, group, w, nv, wlr,
                                        (cudaStream_t)stream),
                     "reconstruct");
}

int snapb_riemann(const snapb_hydro_config* cfg, int solver, int dim, const double* wl,
                  const double* wr, int nv, double* flx, double* face_pressure, const double* vel,
                  void* stream) {
  if (const char* e = check_config(cfg)) return fail(SNAPB_ERR_ARG, std::string("riemann: ") + e);
  if (dim < 1 || dim > 3 || !wl || !wr || !flx) return fail(SNAPB_ERR_ARG, "riemann: bad arguments");
  if (solver == SNAPB_RIEMANN_UPWIND) {
    if (!vel) return fail(SNAPB_ERR_ARG, "riemann: upwind needs the face velocity");
    if (face_pressure)
      return fail(SNAPB_ERR_ARG,
                  "riemann: face-pressure output is not implemented for the upwind solver");
  } else if (solver < SNAPB_RIEMANN_ROE || solver > SNAPB_RIEMANN_HLLC || nv != 5) {
    return fail(SNAPB_ERR_ARG, "riemann: unknown solver or nv != 5");
  }
  return cuda_status(launch_riemann(make_geo(*cfg), make_phys(*cfg), solver, dim, wl, wr, nv, flx,
                                    face_pressure, vel, (cudaStream_t)stream),
                     "riemann");
}

int snapb_hydro_forward(const snapb_hydro_config* cfg, const double* dt, const double* u,
                        double* w, double* du, double* mass_corr, void* workspace,
                        size_t workspace_bytes, void* stream) {
  if (const char* e = check_config(cfg))
    return fail(SNAPB_ERR_ARG, std::string("hydro_forward: ") + e);
  if (!du) return fail(SNAPB_ERR_ARG, "hydro_forward: null du");
  cudaStream_t st = (cudaStream_t)stream;
  Geo g = make_geo(*cfg);
  size_t bytes = (size_t)cfg->nvar * g.sv * sizeof(double);
  Layout L = ws_layout(*cfg);
  if (!workspace || workspace_bytes < L.total)
    return fail(SNAPB_ERR_WORKSPACE, "hydro_forward: workspace too small");
  // du is defined on interior cells and zero elsewhere
  cudaError_t e = cudaMemsetAsync(at<double>(workspace, L.D), 0, bytes, st);
  if (e != cudaSuccess) return cuda_status(e, "hydro_forward clear");
  int rc = run_stage(cfg, 0, dt, const_cast<double*>(u), nullptr, w, nullptr, nullptr, nullptr,
                     workspace, workspace_bytes, st, 1, "hydro_forward");
  if (rc != SNAPB_OK) return rc;
  e = cudaMemcpyAsync(du, at<double>(workspace, L.D), bytes, cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) return cuda_status(e, "hydro_forward copy");
  if (mass_corr) {
    e = cudaMemsetAsync(mass_corr, 0, bytes, st);
    if (e == cudaSuccess && cfg->implicit_scheme)
      e = cudaMemcpyAsync(mass_corr, at<double>(workspace, L.M), (size_t)g.sv * sizeof(double),
                          cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return cuda_status(e, "hydro_forward mass copy");
  }
  return SNAPB_OK;
}

int snapb_implicit_correction(const snapb_hydro_config* cfg, const double* dt, double* du,
                              const double* w, double* mass_corr, void* workspace,
                              size_t workspace_bytes, void* stream) {
  if (const char* e = check_config(cfg))
    return fail(SNAPB_ERR_ARG, std::string("implicit_correction: ") + e);
  if (cfg->implicit_scheme == 0) return SNAPB_OK;  // null operation
  if (!dt || !du || !w) return fail(SNAPB_ERR_ARG, "implicit_correction: null pointer");
  Layout L = ws_layout(*cfg);
  if (!workspace || workspace_bytes < L.total)
    return fail(SNAPB_ERR_WORKSPACE, "implicit_correction: workspace smaller than " +
                                         std::to_string(L.total) + " bytes");
  Geo g = make_geo(*cfg);
  Phys p = make_phys(*cfg);
  p.nscalar = 0;
  StageBufs b;
  std::memset(&b, 0, sizeof(b));
  b.dt = dt;
  b.w = const_cast<double*>(w);
  b.D = du;
  b.M = mass_corr;
  b.vic = at<double>(workspace, L.VIC);
  b.vicT = vic_blocks_bytes(g, p) ? at<double>(workspace, L.VICT) : nullptr;
  b.vic_du_only = 1;
  cudaStream_t st = (cudaStream_t)stream;
  KernelTimer t(SNAPB_K_VIC, st);
  return cuda_status(launch_vic(g, p, b, st), "implicit_correction");
}

int snapb_stage(const snapb_hydro_config* cfg, int stage, const double* dt, double* u, double* u0,
                double* w, double* s, double* s0, double* r, void* workspace,
                size_t workspace_bytes, void* stream) {
  return run_stage(cfg, stage, dt, u, u0, w, s, s0, r, workspace, workspace_bytes,
                   (cudaStream_t)stream, 0, "stage");
}

int snapb_bc_apply(const snapb_hydro_config* cfg, double* var, int nv, int kind, void* stream) {
  if (const char* e = check_config(cfg)) return fail(SNAPB_ERR_ARG, std::string("bc_apply: ") + e);
  if (!var || nv < 1 || kind < SNAPB_PRIMITIVE || kind > SNAPB_SCALAR)
    return fail(SNAPB_ERR_ARG, "bc_apply: bad arguments");
  return cuda_status(launch_bc(make_geo(*cfg), *cfg, var, nv, kind, (cudaStream_t)stream),
                     "bc_apply");
}

int snapb_max_time_step(const snapb_hydro_config* cfg, const double* w, double* dt_out,
                        void* workspace, size_t workspace_bytes, void* stream) {
  if (const char* e = check_config(cfg))
    return fail(SNAPB_ERR_ARG, std::string("max_time_step: ") + e);
  Layout L = ws_layout(*cfg);
  if (!w || !dt_out) return fail(SNAPB_ERR_ARG, "max_time_step: null pointer");
  if (!workspace || workspace_bytes < L.total)
    return fail(SNAPB_ERR_WORKSPACE, "max_time_step: workspace too small");
  return cuda_status(launch_cfl(make_geo(*cfg), make_phys(*cfg), w, at<double>(workspace, L.SLOTS),
                                dt_out, (cudaStream_t)stream),
                     "max_time_step");
}

int snapb_scale_dt(const double* dt_in, double cfl, int redo, double* dt_out, void* stream) {
  if (!dt_in || !dt_out) return fail(SNAPB_ERR_ARG, "scale_dt: null pointer");
  return cuda_status(launch_scale_dt(dt_in, cfl, redo, dt_out, (cudaStream_t)stream), "scale_dt");
}

int snapb_check_positive(const snapb_hydro_config* cfg, const double* u, int* flags,
                         void* stream) {
  if (const char* e = check_config(cfg))
    return fail(SNAPB_ERR_ARG, std::string("check_positive: ") + e);
  if (!u || !flags) return fail(SNAPB_ERR_ARG, "check_positive: null pointer");
  return cuda_status(launch_check_positive(make_geo(*cfg), make_phys(*cfg), u, flags,
                                           (cudaStream_t)stream),
                     "check_positive");
}

int snapb_timing_enable(int on) {
  clear_timings();
  g_timing = on != 0;
  return SNAPB_OK;
}

int snapb_timing_query(int kernel, double* total_ms, int* launches) {
  if (kernel < 0 || kernel >= SNAPB_K_COUNT || !total_ms || !launches)
    return fail(SNAPB_ERR_ARG, "timing_query: bad arguments");
  double tot = 0.;
  int n = 0;
  for (auto& l : g_launches) {
    if (l.kind != kernel) continue;
    cudaError_t e = cudaEventSynchronize(l.b);
    if (e != cudaSuccess) return cuda_status(e, "timing_query");
    float ms = 0.f;
    e = cudaEventElapsedTime(&ms, l.a, l.b);
    if (e != cudaSuccess) return cuda_status(e, "timing_query");
    tot += ms;
    ++n;
  }
  *total_ms = tot;
  *launches = n;
  return SNAPB_OK;
}

}  // extern "C"
