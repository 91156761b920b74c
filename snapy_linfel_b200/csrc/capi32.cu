// capi32.cu — C ABI of the FP32 perturbation form (include/snapb.h, "FP32
// perturbation form" section).  Same conventions as capi.cu: caller-owned
// memory, status codes, dt in device memory.
#include <cstring>
#include <string>

#include "kernels.cuh"

namespace snapb {
cudaError_t launch_ref32(const Geo& g, const Phys& p, const double* rb, const double* pb,
                         double* rbw, double* pbw, const StageBufs32& b, cudaStream_t st);
cudaError_t launch_x1_32(const Geo& g, const Phys& p, const StageBufs32& b, bool last,
                         cudaStream_t st);
cudaError_t launch_march32(int axis, const Geo& g, const Phys& p, const StageBufs32& b,
                           bool first, bool last, cudaStream_t st);
cudaError_t launch_bc32(const Geo& g, const snapb_hydro_config& c, float* var, int nv, int kind,
                        const double* rb, const double* pb, cudaStream_t st);
cudaError_t launch_to_pert(const Geo& g, const Phys& p, int kind, const double* in,
                           const double* rb, const double* pb, float* out, cudaStream_t st);
cudaError_t launch_from_pert(const Geo& g, const Phys& p, int kind, const float* in,
                             const double* rb, const double* pb, double* out, cudaStream_t st);
cudaError_t launch_cfl32(const Geo& g, const Phys& p, const float* w, const float* rbf,
                         const float* pbf, unsigned long long* slots, cudaStream_t st);
size_t x1_smem32_per_column(const Geo& g, int nvt);
}  // namespace snapb

using namespace snapb;

namespace {

const char* check32(const snapb_hydro_config* c, bool has_ref_p) {
  if (const char* e = internal_check_config(c)) return e;
  if (c->nx1 <= 1) return "the FP32 perturbation form needs an active x1 axis";
  if (c->non_hydrostatic != 1.0) return "the FP32 perturbation form needs non-hydrostatic = 1";
  if (c->nu_iso > 0. || c->kappa_iso > 0.)
    return "the FP32 perturbation form does not carry diffusion";
  int pt = c->recon1_shock ? c->recon1_type : (c->recon1_type == SNAPB_RECON_WENO5
                                                   ? SNAPB_RECON_CP5
                                                   : (c->recon1_type == SNAPB_RECON_WENO3
                                                          ? SNAPB_RECON_CP3
                                                          : c->recon1_type));
  bool linear = pt == SNAPB_RECON_CP5 || pt == SNAPB_RECON_CP3 || pt == SNAPB_RECON_DC;
  if (has_ref_p && !linear)
    return "with a reference pressure the x1 pressure interpolation must be linear "
           "(cp5 / cp3 / dc, i.e. shock: false for weno5)";
  Geo g = make_geo(*c);
  if (x1_smem32_per_column(g, 5 + c->nscalar) > 200 * 1024)
    return "x1 column too long for one CTA's shared memory";
  return nullptr;
}

struct Layout32 {
  size_t D, R, M, VIC, PF, OFFL, OFFR, RBAR, RBF, PBF, RBW, PBW, SLOTS, total;
};

size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

Layout32 layout32(const snapb_hydro_config& c) {
  Geo g = make_geo(c);
  Phys p = make_phys(c);
  Layout32 L;
  size_t o = 0, svf = (size_t)g.sv * sizeof(float);
  size_t n1 = (size_t)g.nc1;
  L.D = o;
  o = a256(o + (size_t)(c.nvar + c.nscalar) * svf);
  L.R = o;
  o = a256(o + (size_t)c.nscalar * svf);
  L.M = o;  // the FP32 form has no mass-correction output (scalars use it in place)
  L.VIC = o;
  o = a256(o + vic_scratch_bytes(g, p));
  L.PF = o;
  o = a256(o + (n1 + 1) * sizeof(double));
  L.OFFL = o;
  o = a256(o + (n1 + 1) * sizeof(float));
  L.OFFR = o;
  o = a256(o + (n1 + 1) * sizeof(float));
  L.RBAR = o;
  o = a256(o + n1 * sizeof(float));
  L.RBF = o;
  o = a256(o + n1 * sizeof(float));
  L.PBF = o;
  o = a256(o + n1 * sizeof(float));
  L.RBW = o;
  o = a256(o + n1 * sizeof(double));
  L.PBW = o;
  o = a256(o + n1 * sizeof(double));
  L.SLOTS = o;
  o = a256(o + 8 * sizeof(double));
  L.total = o;
  return L;
}

template <class P>
P* at(void* ws, size_t off) {
  return reinterpret_cast<P*>(static_cast<char*>(ws) + off);
}

StageBufs32 bufs32(const snapb_hydro_config& c, void* ws) {
  Layout32 L = layout32(c);
  StageBufs32 b;
  std::memset(&b, 0, sizeof(b));
  b.D = at<float>(ws, L.D);
  b.R = at<float>(ws, L.R);
  b.M = nullptr;
  b.vic = at<double>(ws, L.VIC);
  b.pf = at<double>(ws, L.PF);
  b.offL = at<float>(ws, L.OFFL);
  b.offR = at<float>(ws, L.OFFR);
  b.rbar = at<float>(ws, L.RBAR);
  b.rbf = at<float>(ws, L.RBF);
  b.pbf = at<float>(ws, L.PBF);
  b.rb = at<double>(ws, L.RBW);
  b.pb = at<double>(ws, L.PBW);
  return b;
}

int cuda32(cudaError_t e, const char* where) {
  if (e == cudaSuccess) return SNAPB_OK;
  return internal_fail(SNAPB_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

}  // namespace

namespace snapb {
StageBufs32 bufs32_of(const snapb_hydro_config& c, void* ws) { return bufs32(c, ws); }
size_t workspace_size_f32_of(const snapb_hydro_config& c) { return layout32(c).total; }
}  // namespace snapb

extern "C" {

size_t snapb_workspace_size_f32(const snapb_hydro_config* cfg) {
  if (check32(cfg, false)) return 0;
  return layout32(*cfg).total;
}

int snapb_reference_f32(const snapb_hydro_config* cfg, const double* ref_rho, const double* ref_p,
                        void* workspace, size_t workspace_bytes, void* stream) {
  if (const char* e = check32(cfg, ref_p != nullptr))
    return internal_fail(SNAPB_ERR_ARG, std::string("reference_f32: ") + e);
  Layout32 L = layout32(*cfg);
  if (!workspace || workspace_bytes < L.total)
    return internal_fail(SNAPB_ERR_WORKSPACE, "reference_f32: workspace smaller than " +
                                                  std::to_string(L.total) + " bytes");
  StageBufs32 b = bufs32(*cfg, workspace);
  Geo g = make_geo(*cfg);
  Phys p = make_phys(*cfg);
  return cuda32(launch_ref32(g, p, ref_rho, ref_p, const_cast<double*>(b.rb),
                             const_cast<double*>(b.pb), b, (cudaStream_t)stream),
                "reference_f32");
}

int snapb_stage_f32(const snapb_hydro_config* cfg, int stage, const double* dt, float* u,
                    float* u0, float* w, float* s, float* s0, float* r, void* workspace,
                    size_t workspace_bytes, void* stream) {
  if (const char* e = check32(cfg, false))
    return internal_fail(SNAPB_ERR_ARG, std::string("stage_f32: ") + e);
  if (!dt || !u || !u0 || !w) return internal_fail(SNAPB_ERR_ARG, "stage_f32: null state pointer");
  if (stage < 0 || stage > 2) return internal_fail(SNAPB_ERR_ARG, "stage_f32: stage in [0, 2]");
  Layout32 L = layout32(*cfg);
  if (!workspace || workspace_bytes < L.total)
    return internal_fail(SNAPB_ERR_WORKSPACE, "stage_f32: workspace smaller than " +
                                                  std::to_string(L.total) + " bytes");
  Geo g = make_geo(*cfg);
  Phys p = make_phys(*cfg);
  if (p.nscalar > 0 && (!s || !s0))
    return internal_fail(SNAPB_ERR_ARG, "stage_f32: scalars need s and s0");
  if (p.nscalar > 0 && p.implicit_scheme && !r)
    return internal_fail(SNAPB_ERR_ARG, "stage_f32: implicit scalar transport needs r");
  StageBufs32 b = bufs32(*cfg, workspace);
  b.dt = dt;
  b.u = u;
  b.u0 = u0;
  b.w = w;
  b.s = s;
  b.s0 = s0;
  b.r = p.implicit_scheme ? r : nullptr;
  b.stage = stage;
  rk3_weights(stage, b.wgt0, b.wgt1, b.wgt2);
  b.write_du = p.implicit_scheme ? 1 : 0;
  b.vic_du_only = 0;
  cudaStream_t st = (cudaStream_t)stream;
  const bool a2 = g.nc2 > 1, a3 = g.nc3 > 1;
  int last = a3 ? 3 : (a2 ? 2 : 1);
  cudaError_t e;
  {
    ScopedTimer t(SNAPB_K_X1, st);
    e = launch_x1_32(g, p, b, last == 1, st);
  }
  if (e != cudaSuccess) return cuda32(e, "stage_f32 x1");
  if (a2) {
    ScopedTimer t(SNAPB_K_X2, st);
    e = launch_march32(2, g, p, b, false, last == 2, st);
    if (e != cudaSuccess) return cuda32(e, "stage_f32 x2");
  }
  if (a3) {
    ScopedTimer t(SNAPB_K_X3, st);
    e = launch_march32(3, g, p, b, false, true, st);
    if (e != cudaSuccess) return cuda32(e, "stage_f32 x3");
  }
  if (p.implicit_scheme) {
    ScopedTimer t(SNAPB_K_VIC, st);
    e = launch_vic32(g, p, b, st);
    if (e != cudaSuccess) return cuda32(e, "stage_f32 implicit");
  }
  ScopedTimer t(SNAPB_K_BC, st);
  e = launch_bc32(g, *cfg, u, cfg->nvar, SNAPB_CONSERVED, b.rb, b.pb, st);
  if (e == cudaSuccess && p.nscalar > 0)
    e = launch_bc32(g, *cfg, s, p.nscalar, SNAPB_SCALAR, b.rb, b.pb, st);
  return cuda32(e, "stage_f32 boundary");
}

int snapb_bc_apply_f32(const snapb_hydro_config* cfg, float* var, int nv, int kind,
                       void* workspace, size_t workspace_bytes, void* stream) {
  if (const char* e = check32(cfg, false))
    return internal_fail(SNAPB_ERR_ARG, std::string("bc_apply_f32: ") + e);
  Layout32 L = layout32(*cfg);
  if (!var || !workspace || workspace_bytes < L.total)
    return internal_fail(SNAPB_ERR_ARG, "bc_apply_f32: bad arguments");
  StageBufs32 b = bufs32(*cfg, workspace);
  return cuda32(launch_bc32(make_geo(*cfg), *cfg, var, nv, kind, b.rb, b.pb,
                            (cudaStream_t)stream),
                "bc_apply_f32");
}

int snapb_to_perturbation(const snapb_hydro_config* cfg, int kind, const double* in, float* out,
                          void* workspace, size_t workspace_bytes, void* stream) {
  if (const char* e = check32(cfg, false))
    return internal_fail(SNAPB_ERR_ARG, std::string("to_perturbation: ") + e);
  Layout32 L = layout32(*cfg);
  if (!in || !out || !workspace || workspace_bytes < L.total)
    return internal_fail(SNAPB_ERR_ARG, "to_perturbation: bad arguments");
  StageBufs32 b = bufs32(*cfg, workspace);
  return cuda32(launch_to_pert(make_geo(*cfg), make_phys(*cfg), kind, in, b.rb, b.pb, out,
                               (cudaStream_t)stream),
                "to_perturbation");
}

int snapb_from_perturbation(const snapb_hydro_config* cfg, int kind, const float* in, double* out,
                            void* workspace, size_t workspace_bytes, void* stream) {
  if (const char* e = check32(cfg, false))
    return internal_fail(SNAPB_ERR_ARG, std::string("from_perturbation: ") + e);
  Layout32 L = layout32(*cfg);
  if (!in || !out || !workspace || workspace_bytes < L.total)
    return internal_fail(SNAPB_ERR_ARG, "from_perturbation: bad arguments");
  StageBufs32 b = bufs32(*cfg, workspace);
  return cuda32(launch_from_pert(make_geo(*cfg), make_phys(*cfg), kind, in, b.rb, b.pb, out,
                                 (cudaStream_t)stream),
                "from_perturbation");
}

int snapb_max_time_step_f32(const snapb_hydro_config* cfg, const float* w, double* dt_out,
                            void* workspace, size_t workspace_bytes, void* stream) {
  if (const char* e = check32(cfg, false))
    return internal_fail(SNAPB_ERR_ARG, std::string("max_time_step_f32: ") + e);
  Layout32 L = layout32(*cfg);
  if (!w || !dt_out || !workspace || workspace_bytes < L.total)
    return internal_fail(SNAPB_ERR_ARG, "max_time_step_f32: bad arguments");
  StageBufs32 b = bufs32(*cfg, workspace);
  Geo g = make_geo(*cfg);
  Phys p = make_phys(*cfg);
  cudaStream_t st = (cudaStream_t)stream;
  auto* slots = at<unsigned long long>(workspace, L.SLOTS);
  cudaError_t e = cudaMemsetAsync(slots, 0x7f, 3 * sizeof(unsigned long long), st);
  if (e == cudaSuccess) e = launch_cfl32(g, p, w, b.rbf, b.pbf, slots, st);
  if (e == cudaSuccess) e = launch_cfl_final(g, p, slots, dt_out, st);
  return cuda32(e, "max_time_step_f32");
}

}  // extern "C"
