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
// Errors raise c10::Error through TORCH_CHECK, as the reference's modules do.
#include <ATen/cuda/CUDAContext.h>
#include <c10/cuda/CUDAGuard.h>
#include <torch/extension.h>

#include <string>

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
}
