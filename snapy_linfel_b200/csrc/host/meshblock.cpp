// meshblock.cpp — C++ host modules over libtorch tensors that drive the snapb
// C ABI (include/snapb.h) on the current torch CUDA stream.
//
// Mirrors the module interface of the reference on this path:
//   snapb::Hydro::forward(dt, u, w) -> du        HydroImpl::forward
//                                                (src/hydro/hydro_forward.cpp:14-217)
//   snapb::Hydro::max_time_step(w) -> double     HydroImpl::max_time_step
//                                                (src/hydro/hydro.cpp:118-180)
//   snapb::MeshBlock::initialize / forward(dt, stage) / max_time_step /
//   check_redo                                   MeshBlockImpl (src/mesh/meshblock.cpp)
//   snapb::MeshBlockF32, snapb::Ensemble         the FP32 perturbation form and
//                                                batched ensembles (no reference
//                                                counterpart)
// Errors raise c10::Error through TORCH_CHECK, as the reference's modules do.
#include <ATen/cuda/CUDAContext.h>
#include <c10/cuda/CUDAGuard.h>
#include <torch/extension.h>

#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../../include/snapb.h"

namespace snapb_host {

namespace {

void check(int rc, const char* what) {
  TORCH_CHECK(rc == SNAPB_OK, what, " failed (", rc, "): ", snapb_last_error());
}

void* dptr(const torch::Tensor& t, torch::ScalarType ty, const char* name) {
  TORCH_CHECK(t.is_cuda(), name, " must be a CUDA tensor");
  TORCH_CHECK(t.is_contiguous(), name, " must be contiguous");
  TORCH_CHECK(t.scalar_type() == ty, name, " has the wrong dtype");
  return t.data_ptr();
}

void* stream() { return (void*)at::cuda::getCurrentCUDAStream().stream(); }

}  // namespace

// configuration mirror: built from a Python dict of snapb_hydro_config fields
snapb_hydro_config config_from_dict(const pybind11::dict& d) {
  snapb_hydro_config c{};
  auto geti = [&](const char* k, int def) {
    return d.contains(k) ? d[k].cast<int>() : def;
  };
  auto getd = [&](const char* k, double def) {
    return d.contains(k) ? d[k].cast<double>() : def;
  };
  c.nx1 = geti("nx1", 1);
  c.nx2 = geti("nx2", 1);
  c.nx3 = geti("nx3", 1);
  c.nghost = geti("nghost", 3);
  c.nvar = geti("nvar", 5);
  c.nscalar = geti("nscalar", 0);
  c.x1min = getd("x1min", 0.);
  c.x1max = getd("x1max", 1.);
  c.x2min = getd("x2min", 0.);
  c.x2max = getd("x2max", 1.);
  c.x3min = getd("x3min", 0.);
  c.x3max = getd("x3max", 1.);
  c.gammad = getd("gammad", 1.4);
  c.rgas = getd("rgas", 287.);
  c.recon1_type = geti("recon1_type", SNAPB_RECON_WENO5);
  c.recon1_shock = geti("recon1_shock", 0);
  c.recon1_scale = geti("recon1_scale", 0);
  c.recon23_type = geti("recon23_type", SNAPB_RECON_WENO5);
  c.recon23_shock = geti("recon23_shock", 0);
  c.recon23_scale = geti("recon23_scale", 0);
  c.scalar_recon_type = geti("scalar_recon_type", SNAPB_RECON_DC);
  c.scalar_recon_scale = geti("scalar_recon_scale", 0);
  c.riemann = geti("riemann", SNAPB_RIEMANN_HLLC);
  c.implicit_scheme = geti("implicit_scheme", 0);
  c.grav1 = getd("grav1", 0.);
  c.grav2 = getd("grav2", 0.);
  c.grav3 = getd("grav3", 0.);
  c.non_hydrostatic = getd("non_hydrostatic", 1.);
  c.nu_iso = getd("nu_iso", 0.);
  c.kappa_iso = getd("kappa_iso", 0.);
  if (d.contains("bc")) {
    auto b = d["bc"].cast<std::vector<int>>();
    TORCH_CHECK(b.size() == 6, "bc needs six entries");
    for (int i = 0; i < 6; ++i) c.bc[i] = b[i];
  } else {
    for (int i = 0; i < 6; ++i) c.bc[i] = SNAPB_BC_REFLECTING;
  }
  if (d.contains("disable_flux")) {
    auto b = d["disable_flux"].cast<std::vector<int>>();
    for (int i = 0; i < 3 && i < (int)b.size(); ++i) c.disable_flux[i] = b[i];
  }
  TORCH_CHECK(snapb_workspace_size(&c) > 0, "invalid hydro configuration: ", snapb_last_error());
  return c;
}

std::vector<int64_t> shape_of(const snapb_hydro_config& c, int nv) {
  auto nc = [&](int nx) { return nx > 1 ? nx + 2 * c.nghost : 1; };
  return {nv, nc(c.nx3), nc(c.nx2), nc(c.nx1)};
}

// The hydro forward module: du = forward(dt, u, w) with w written in place.
class Hydro {
 public:
  explicit Hydro(const pybind11::dict& d) : cfg_(config_from_dict(d)) {}

  torch::Tensor forward(double dt, torch::Tensor u, torch::Tensor w) {
    c10::cuda::CUDAGuard guard(u.device());
    ensure(u);
    auto du = torch::empty_like(u);
    dt_.fill_(dt);
    check(snapb_hydro_forward(&cfg_, (double*)dt_.data_ptr(),
                              (double*)dptr(u, torch::kFloat64, "u"),
                              (double*)dptr(w, torch::kFloat64, "w"), (double*)du.data_ptr(),
                              cfg_.implicit_scheme ? (double*)mass_.data_ptr() : nullptr,
                              ws_.data_ptr(), (size_t)ws_.numel(), stream()),
          "snapb_hydro_forward");
    return du;
  }

  double max_time_step(torch::Tensor w) {
    c10::cuda::CUDAGuard guard(w.device());
    ensure(w);
    check(snapb_max_time_step(&cfg_, (double*)dptr(w, torch::kFloat64, "w"),
                              (double*)dt_.data_ptr(), ws_.data_ptr(), (size_t)ws_.numel(),
                              stream()),
          "snapb_max_time_step");
    return dt_.item<double>();
  }

  torch::Tensor implicit_mass_correction() const { return mass_; }

 private:
  void ensure(const torch::Tensor& like) {
    if (ws_.defined() && ws_.device() == like.device()) return;
    auto opts = like.options();
    ws_ = torch::empty({(int64_t)snapb_workspace_size(&cfg_)}, opts.dtype(torch::kUInt8));
    dt_ = torch::zeros({1}, opts.dtype(torch::kFloat64));
    mass_ = torch::zeros(shape_of(cfg_, cfg_.nvar), opts.dtype(torch::kFloat64));
  }

  snapb_hydro_config cfg_;
  torch::Tensor ws_, dt_, mass_;
};

// One mesh block: state buffers + the RK3 stage loop.
class MeshBlock {
 public:
  MeshBlock(const pybind11::dict& d, double cfl, int64_t device)
      : cfg_(config_from_dict(d)), cfl_(cfl) {
    auto opts = torch::TensorOptions().dtype(torch::kFloat64).device(torch::kCUDA, device);
    hydro_u = torch::zeros(shape_of(cfg_, cfg_.nvar), opts);
    hydro_w = torch::zeros_like(hydro_u);
    hydro_u0 = torch::zeros_like(hydro_u);
    if (cfg_.nscalar > 0) {
      scalar_s = torch::zeros(shape_of(cfg_, cfg_.nscalar), opts);
      scalar_s0 = torch::zeros_like(scalar_s);
      scalar_r = torch::zeros_like(scalar_s);
    }
    ws_ = torch::empty({(int64_t)snapb_workspace_size(&cfg_)}, opts.dtype(torch::kUInt8));
    dt_raw_ = torch::zeros({1}, opts);
    dt = torch::zeros({1}, opts);
    flags_ = torch::zeros({4}, opts.dtype(torch::kInt32));
  }

  void initialize(torch::Tensor w, torch::optional<torch::Tensor> r) {
    c10::cuda::CUDAGuard guard(hydro_u.device());
    hydro_w.copy_(w);
    check(snapb_bc_apply(&cfg_, (double*)hydro_w.data_ptr(), cfg_.nvar, SNAPB_PRIMITIVE,
                         stream()),
          "snapb_bc_apply");
    if (cfg_.nscalar > 0) {
      TORCH_CHECK(r.has_value(), "initialize: scalar_r is required for scalar model.");
      scalar_r.copy_(*r);
      check(snapb_bc_apply(&cfg_, (double*)scalar_r.data_ptr(), cfg_.nscalar, SNAPB_SCALAR,
                           stream()),
            "snapb_bc_apply");
    }
    check(snapb_prim2cons(&cfg_, (double*)hydro_w.data_ptr(), (double*)hydro_u.data_ptr(),
                          stream()),
          "snapb_prim2cons");
    if (cfg_.nscalar > 0) scalar_s.copy_(hydro_w.narrow(0, 0, 1) * scalar_r);
    check(snapb_bc_apply(&cfg_, (double*)hydro_u.data_ptr(), cfg_.nvar, SNAPB_CONSERVED,
                         stream()),
          "snapb_bc_apply");
    if (cfg_.nscalar > 0)
      check(snapb_bc_apply(&cfg_, (double*)scalar_s.data_ptr(), cfg_.nscalar, SNAPB_SCALAR,
                           stream()),
            "snapb_bc_apply");
  }

  // dt = cfl * 2^-redo * CFL limit; stays on the device (returned as a tensor)
  torch::Tensor max_time_step() {
    c10::cuda::CUDAGuard guard(hydro_u.device());
    check(snapb_max_time_step(&cfg_, (double*)hydro_w.data_ptr(), (double*)dt_raw_.data_ptr(),
                              ws_.data_ptr(), (size_t)ws_.numel(), stream()),
          "snapb_max_time_step");
    check(snapb_scale_dt((double*)dt_raw_.data_ptr(), cfl_, current_redo,
                         (double*)dt.data_ptr(), stream()),
          "snapb_scale_dt");
    return dt;
  }

  void forward(int64_t stage) {
    c10::cuda::CUDAGuard guard(hydro_u.device());
    auto sp = [](torch::Tensor& t) { return t.defined() ? (double*)t.data_ptr() : nullptr; };
    check(snapb_stage(&cfg_, (int)stage, (double*)dt.data_ptr(), (double*)hydro_u.data_ptr(),
                      (double*)hydro_u0.data_ptr(), (double*)hydro_w.data_ptr(), sp(scalar_s),
                      sp(scalar_s0), sp(scalar_r), ws_.data_ptr(), (size_t)ws_.numel(),
                      stream()),
          "snapb_stage");
  }

  void step(torch::optional<double> dt_fixed) {
    if (dt_fixed.has_value())
      dt.fill_(*dt_fixed);
    else
      max_time_step();
    for (int s = 0; s < 3; ++s) forward(s);
    ++cycle;
  }

  int check_redo(int64_t max_redo) {
    c10::cuda::CUDAGuard guard(hydro_u.device());
    check(snapb_check_positive(&cfg_, (double*)hydro_u.data_ptr(), (int*)flags_.data_ptr(),
                               stream()),
          "snapb_check_positive");
    auto f = flags_.cpu();
    auto a = f.accessor<int, 1>();
    if (a[0] || (a[1] && a[2])) {
      ++current_redo;
      if (current_redo > max_redo) return -1;
      hydro_u.copy_(hydro_u0);
      check(snapb_bc_apply(&cfg_, (double*)hydro_u.data_ptr(), cfg_.nvar, SNAPB_CONSERVED,
                           stream()),
            "snapb_bc_apply");
      if (cfg_.nscalar > 0) {
        scalar_s.copy_(scalar_s0);
        check(snapb_bc_apply(&cfg_, (double*)scalar_s.data_ptr(), cfg_.nscalar, SNAPB_SCALAR,
                             stream()),
              "snapb_bc_apply");
      }
      --cycle;  // the rejected step does not count (step() counted it)
      return 1;
    }
    current_redo = 0;
    return 0;
  }

  torch::Tensor hydro_u, hydro_w, hydro_u0, scalar_s, scalar_s0, scalar_r, dt;
  int64_t cycle = 0;
  int current_redo = 0;

 private:
  snapb_hydro_config cfg_;
  double cfl_;
  torch::Tensor ws_, dt_raw_, flags_;
};

// The FP32 perturbation form of one mesh block: FP32 state about an FP64
// reference profile rho_bar(x1), p_bar(x1) (by default the horizontal mean
// of the initial state), driven through snapb_stage_f32.  state64() returns
// the FP64 conserved state.
class MeshBlockF32 {
 public:
  MeshBlockF32(const pybind11::dict& d, double cfl, int64_t device)
      : cfg_(config_from_dict(d)), cfl_(cfl) {
    const size_t nbytes = snapb_workspace_size_f32(&cfg_);
    TORCH_CHECK(nbytes > 0, "configuration not supported by the FP32 form: ",
                snapb_last_error());
    auto f32 = torch::TensorOptions().dtype(torch::kFloat32).device(torch::kCUDA, device);
    auto f64 = f32.dtype(torch::kFloat64);
    hydro_u = torch::zeros(shape_of(cfg_, cfg_.nvar), f32);
    hydro_u0 = torch::zeros_like(hydro_u);
    hydro_w = torch::zeros_like(hydro_u);
    if (cfg_.nscalar > 0) {
      scalar_s = torch::zeros(shape_of(cfg_, cfg_.nscalar), f32);
      scalar_s0 = torch::zeros_like(scalar_s);
      scalar_r = torch::zeros_like(scalar_s);
    }
    workspace = torch::empty({(int64_t)nbytes}, f32.dtype(torch::kUInt8));
    const int64_t nc1 = shape_of(cfg_, 1)[3];
    ref_rho = torch::zeros({nc1}, f64);
    ref_p = torch::zeros({nc1}, f64);
    dt_raw_ = torch::zeros({1}, f64);
    dt = torch::zeros({1}, f64);
  }

  // w, r: FP64 primitive state and mixing ratios [nv, nc3, nc2, nc1];
  // reference "mean" (horizontal mean at each x1 level) or "none"
  void initialize(torch::Tensor w, torch::optional<torch::Tensor> r, std::string reference) {
    c10::cuda::CUDAGuard guard(hydro_u.device());
    auto w64 = w.to(hydro_u.device(), torch::kFloat64).contiguous();
    check(snapb_bc_apply(&cfg_, (double*)w64.data_ptr(), cfg_.nvar, SNAPB_PRIMITIVE, stream()),
          "snapb_bc_apply");
    void* ws = workspace.data_ptr();
    const size_t nb = (size_t)workspace.numel();
    if (reference == "none") {
      ref_rho.zero_();
      ref_p.zero_();
      check(snapb_reference_f32(&cfg_, nullptr, nullptr, ws, nb, stream()),
            "snapb_reference_f32");
    } else {
      TORCH_CHECK(reference == "mean", "reference: 'mean' or 'none'");
      using torch::indexing::Slice;
      const int64_t g = cfg_.nghost;
      auto k = cfg_.nx3 > 1 ? Slice(g, g + cfg_.nx3) : Slice(0, 1);
      auto j = cfg_.nx2 > 1 ? Slice(g, g + cfg_.nx2) : Slice(0, 1);
      const std::vector<int64_t> dims{0, 1};
      ref_rho.copy_(w64[0].index({k, j, Slice()}).mean(dims));
      ref_p.copy_(w64[4].index({k, j, Slice()}).mean(dims));
      check(snapb_reference_f32(&cfg_, (double*)ref_rho.data_ptr(), (double*)ref_p.data_ptr(),
                                ws, nb, stream()),
            "snapb_reference_f32");
    }
    auto u64 = torch::empty_like(w64);
    check(snapb_prim2cons(&cfg_, (double*)w64.data_ptr(), (double*)u64.data_ptr(), stream()),
          "snapb_prim2cons");
    if (cfg_.nscalar > 0) {
      TORCH_CHECK(r.has_value(), "initialize: scalar_r is required for scalar model.");
      auto r64 = r->to(hydro_u.device(), torch::kFloat64).contiguous();
      check(snapb_bc_apply(&cfg_, (double*)r64.data_ptr(), cfg_.nscalar, SNAPB_SCALAR,
                           stream()),
            "snapb_bc_apply");
      auto s64 = (w64.narrow(0, 0, 1) * r64).contiguous();
      check(snapb_bc_apply(&cfg_, (double*)s64.data_ptr(), cfg_.nscalar, SNAPB_SCALAR,
                           stream()),
            "snapb_bc_apply");
      scalar_s.copy_(s64);
      scalar_r.copy_(r64);
    }
    check(snapb_bc_apply(&cfg_, (double*)u64.data_ptr(), cfg_.nvar, SNAPB_CONSERVED, stream()),
          "snapb_bc_apply");
    check(snapb_to_perturbation(&cfg_, SNAPB_CONSERVED, (double*)u64.data_ptr(),
                                (float*)hydro_u.data_ptr(), ws, nb, stream()),
          "snapb_to_perturbation");
    check(snapb_to_perturbation(&cfg_, SNAPB_PRIMITIVE, (double*)w64.data_ptr(),
                                (float*)hydro_w.data_ptr(), ws, nb, stream()),
          "snapb_to_perturbation");
  }

  torch::Tensor max_time_step() {
    c10::cuda::CUDAGuard guard(hydro_u.device());
    check(snapb_max_time_step_f32(&cfg_, (float*)hydro_w.data_ptr(),
                                  (double*)dt_raw_.data_ptr(), workspace.data_ptr(),
                                  (size_t)workspace.numel(), stream()),
          "snapb_max_time_step_f32");
    check(snapb_scale_dt((double*)dt_raw_.data_ptr(), cfl_, current_redo,
                         (double*)dt.data_ptr(), stream()),
          "snapb_scale_dt");
    return dt;
  }

  void forward(int64_t stage) {
    c10::cuda::CUDAGuard guard(hydro_u.device());
    auto sp = [](torch::Tensor& t) { return t.defined() ? (float*)t.data_ptr() : nullptr; };
    check(snapb_stage_f32(&cfg_, (int)stage, (double*)dt.data_ptr(), (float*)hydro_u.data_ptr(),
                          (float*)hydro_u0.data_ptr(), (float*)hydro_w.data_ptr(),
                          sp(scalar_s), sp(scalar_s0), sp(scalar_r), workspace.data_ptr(),
                          (size_t)workspace.numel(), stream()),
          "snapb_stage_f32");
  }

  void step(torch::optional<double> dt_fixed) {
    if (dt_fixed.has_value())
      dt.fill_(*dt_fixed);
    else
      max_time_step();
    for (int s = 0; s < 3; ++s) forward(s);
    ++cycle;
  }

  torch::Tensor state64() {
    c10::cuda::CUDAGuard guard(hydro_u.device());
    auto out = torch::empty(hydro_u.sizes(), hydro_u.options().dtype(torch::kFloat64));
    check(snapb_from_perturbation(&cfg_, SNAPB_CONSERVED, (float*)hydro_u.data_ptr(),
                                  (double*)out.data_ptr(), workspace.data_ptr(),
                                  (size_t)workspace.numel(), stream()),
          "snapb_from_perturbation");
    return out;
  }

  const snapb_hydro_config& config() const { return cfg_; }

  torch::Tensor hydro_u, hydro_u0, hydro_w, scalar_s, scalar_s0, scalar_r, workspace;
  torch::Tensor ref_rho, ref_p, dt;
  int64_t cycle = 0;
  int current_redo = 0;

 private:
  snapb_hydro_config cfg_;
  double cfl_;
  torch::Tensor dt_raw_;
};

// A batched ensemble of FP32 blocks of uneven sizes with the same physics:
// every stage is one persistent launch per sweep over all members
// (snapb_ensemble_*), dt per member on the device.
class Ensemble {
 public:
  Ensemble(std::vector<std::shared_ptr<MeshBlockF32>> blocks, double cfl,
           const std::vector<int>& tuning)
      : blocks_(std::move(blocks)), cfl_(cfl) {
    TORCH_CHECK(!blocks_.empty(), "ensemble: no members");
    std::memset(&tune_, 0, sizeof(tune_));
    if (tuning.size() > 0) tune_.x1_columns = tuning[0];
    if (tuning.size() > 1) tune_.march_segment = tuning[1];
    if (tuning.size() > 2) tune_.ctas_per_sm = tuning[2];
    if (tuning.size() > 3) tune_.vic_block = tuning[3];
    if (tuning.size() > 4) tune_.vic_regs = tuning[4];
    if (tuning.size() > 5) tune_.vic_kernel = tuning[5];
    std::vector<snapb_member_f32> mem(blocks_.size());
    auto fp = [](torch::Tensor& t) { return t.defined() ? (float*)t.data_ptr() : nullptr; };
    for (size_t k = 0; k < blocks_.size(); ++k) {
      auto& b = *blocks_[k];
      std::memset(&mem[k], 0, sizeof(mem[k]));
      mem[k].cfg = b.config();
      mem[k].u = fp(b.hydro_u);
      mem[k].u0 = fp(b.hydro_u0);
      mem[k].w = fp(b.hydro_w);
      mem[k].s = fp(b.scalar_s);
      mem[k].s0 = fp(b.scalar_s0);
      mem[k].r = fp(b.scalar_r);
      mem[k].workspace = b.workspace.data_ptr();
      mem[k].workspace_bytes = (size_t)b.workspace.numel();
    }
    check(snapb_ensemble_create(mem.data(), (int)mem.size(), &tune_, &handle_),
          "snapb_ensemble_create");
    c10::cuda::CUDAGuard guard(blocks_[0]->hydro_u.device());
    const size_t nbytes = snapb_ensemble_workspace_size(handle_);
    workspace_ = torch::zeros({(int64_t)nbytes},
                              blocks_[0]->hydro_u.options().dtype(torch::kUInt8));
    check(snapb_ensemble_bind(handle_, workspace_.data_ptr(), nbytes, stream()),
          "snapb_ensemble_bind");
  }
  ~Ensemble() {
    if (handle_) snapb_ensemble_destroy(handle_);
  }
  Ensemble(const Ensemble&) = delete;
  Ensemble& operator=(const Ensemble&) = delete;

  void max_time_step() {
    c10::cuda::CUDAGuard guard(workspace_.device());
    check(snapb_ensemble_max_time_step_f32(handle_, cfl_, stream()),
          "snapb_ensemble_max_time_step_f32");
  }
  void stage(int64_t k) {
    c10::cuda::CUDAGuard guard(workspace_.device());
    check(snapb_ensemble_stage_f32(handle_, (int)k, stream()), "snapb_ensemble_stage_f32");
  }
  // CFL of every member, then the three stages (capturable in a CUDA graph)
  void step() {
    max_time_step();
    for (int k = 0; k < 3; ++k) stage(k);
    ++cycle;
  }
  // the members' dt [n] (a view of the bound workspace)
  torch::Tensor dts() {
    const double* p = snapb_ensemble_dt(handle_);
    const int64_t off = (const char*)p - (const char*)workspace_.data_ptr();
    return workspace_.narrow(0, off, 8 * (int64_t)blocks_.size()).view(torch::kFloat64);
  }
  int64_t cells() const {
    int64_t n = 0;
    for (auto& b : blocks_) {
      const auto& c = b->config();
      n += (int64_t)c.nx1 * c.nx2 * c.nx3;
    }
    return n;
  }

  int64_t cycle = 0;

 private:
  std::vector<std::shared_ptr<MeshBlockF32>> blocks_;
  double cfl_;
  snapb_ensemble_tuning tune_;
  snapb_ensemble* handle_ = nullptr;
  torch::Tensor workspace_;
};

}  // namespace snapb_host

PYBIND11_MODULE(_snapb_host, m) {
  using namespace snapb_host;
  m.doc() = "C++ host modules (libtorch) over the snapb C ABI";
  pybind11::class_<Hydro>(m, "Hydro")
      .def(pybind11::init<const pybind11::dict&>())
      .def("forward", &Hydro::forward)
      .def("max_time_step", &Hydro::max_time_step)
      .def("implicit_mass_correction", &Hydro::implicit_mass_correction);
  pybind11::class_<MeshBlock>(m, "MeshBlock")
      .def(pybind11::init<const pybind11::dict&, double, int64_t>())
      .def("initialize", &MeshBlock::initialize, pybind11::arg("w"),
           pybind11::arg("r") = pybind11::none())
      .def("max_time_step", &MeshBlock::max_time_step)
      .def("forward", &MeshBlock::forward)
      .def("step", &MeshBlock::step, pybind11::arg("dt") = pybind11::none())
      .def("check_redo", &MeshBlock::check_redo, pybind11::arg("max_redo") = 5)
      .def_readonly("hydro_u", &MeshBlock::hydro_u)
      .def_readonly("hydro_w", &MeshBlock::hydro_w)
      .def_readonly("hydro_u0", &MeshBlock::hydro_u0)
      .def_readonly("current_redo", &MeshBlock::current_redo)
      .def_readonly("scalar_s", &MeshBlock::scalar_s)
      .def_readonly("scalar_r", &MeshBlock::scalar_r)
      .def_readonly("dt", &MeshBlock::dt)
      .def_readonly("cycle", &MeshBlock::cycle);
  pybind11::class_<MeshBlockF32, std::shared_ptr<MeshBlockF32>>(m, "MeshBlockF32")
      .def(pybind11::init<const pybind11::dict&, double, int64_t>())
      .def("initialize", &MeshBlockF32::initialize, pybind11::arg("w"),
           pybind11::arg("r") = pybind11::none(), pybind11::arg("reference") = "mean")
      .def("max_time_step", &MeshBlockF32::max_time_step)
      .def("forward", &MeshBlockF32::forward)
      .def("step", &MeshBlockF32::step, pybind11::arg("dt") = pybind11::none())
      .def("state64", &MeshBlockF32::state64)
      .def_readonly("hydro_u", &MeshBlockF32::hydro_u)
      .def_readonly("hydro_u0", &MeshBlockF32::hydro_u0)
      .def_readonly("hydro_w", &MeshBlockF32::hydro_w)
      .def_readonly("scalar_s", &MeshBlockF32::scalar_s)
      .def_readonly("scalar_r", &MeshBlockF32::scalar_r)
      .def_readonly("ref_rho", &MeshBlockF32::ref_rho)
      .def_readonly("ref_p", &MeshBlockF32::ref_p)
      .def_readonly("dt", &MeshBlockF32::dt)
      .def_readonly("cycle", &MeshBlockF32::cycle);
  pybind11::class_<Ensemble>(m, "Ensemble")
      .def(pybind11::init<std::vector<std::shared_ptr<MeshBlockF32>>, double,
                          const std::vector<int>&>(),
           pybind11::arg("blocks"), pybind11::arg("cfl"),
           pybind11::arg("tuning") = std::vector<int>{})
      .def("max_time_step", &Ensemble::max_time_step)
      .def("stage", &Ensemble::stage)
      .def("step", &Ensemble::step)
      .def("dts", &Ensemble::dts)
      .def("cells", &Ensemble::cells)
      .def_readonly("cycle", &Ensemble::cycle);
}
