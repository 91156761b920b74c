// oracle_capi.cpp — C entry points of the CPU oracle (TEST INFRASTRUCTURE
// ONLY).  Host-pointer twins of the snapb_* entry points in include/snapb.h,
// loaded with ctypes by tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg.  The same source is built twice: liboracle.so (restated point
// kernels) and _ref/libsnapref.so (the reference's own *_impl.h kernels).
#include <cstdio>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>

#include "oracle.hpp"

namespace {
thread_local std::string g_err;

int guard(const char* what, const std::function<void()>& f) {
  try {
    f();
    return SNAPB_OK;
  } catch (std::exception& e) {
    g_err = std::string(what) + ": " + e.what();
    return SNAPB_ERR_ARG;
  }
}
}  // namespace

extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }

int orc_kernels_kind(void) {
#ifdef ORC_REFERENCE_KERNELS
  return 1;
#else
  return 0;
#endif
}

void orc_set_threads(int n) { orc::num_threads() = n > 0 ? n : 1; }
int orc_get_threads(void) { return orc::num_threads(); }

// one interpolated value from a window: side 1 = "left" (wlr[IRT]), 0 = "right"
double orc_interp_point(int type, int side, const double* window, int scale) {
  if (type == SNAPB_RECON_PLM) {
    // value at the left (side 1) or right (side 0) face of window[1]
    double dl = window[1] - window[0], dr = window[2] - window[1];
    double dw2 = dl * dr;
    double dwm = 2. * dw2 / (dl + dr + (double)std::numeric_limits<float>::min());
    dwm *= (dw2 >= 0) ? 1 : 0;
    return side ? window[1] - 0.5 * dwm : window[1] + 0.5 * dwm;
  }
  return orc::interp_value(type, side, window, 1, scale != 0);
}

int orc_cons2prim(const snapb_hydro_config* cfg, const double* u, double* w) {
  return guard("orc_cons2prim", [&] { orc::cons2prim(orc::Grid(*cfg), u, w); });
}

int orc_prim2cons(const snapb_hydro_config* cfg, const double* w, double* u) {
  return guard("orc_prim2cons", [&] { orc::prim2cons(orc::Grid(*cfg), w, u); });
}

int orc_reconstruct(const snapb_hydro_config* cfg, int dim, int group, const double* w,
                    int nv, double* wlr) {
  return guard("orc_reconstruct",
               [&] { orc::reconstruct(orc::Grid(*cfg), dim, group, w, nv, wlr); });
}

int orc_riemann(const snapb_hydro_config* cfg, int solver, int dim, const double* wl,
                const double* wr, int nv, double* flx, double* fp, const double* vel) {
  return guard("orc_riemann", [&] {
    orc::riemann(orc::Grid(*cfg), solver, dim, wl, wr, nv, flx, fp, vel);
  });
}

int orc_bc_apply(const snapb_hydro_config* cfg, double* var, int nv, int kind) {
  return guard("orc_bc_apply", [&] { orc::bc_apply(orc::Grid(*cfg), var, nv, kind); });
}

double orc_max_time_step(const snapb_hydro_config* cfg, const double* w) {
  return orc::max_time_step(orc::Grid(*cfg), w);
}

// a block keeps the module buffers (F1, F2, F3, mass_corr) between calls,
// as the reference's registered buffers do
void* orc_block_create(const snapb_hydro_config* cfg) {
  try {
    return new orc::Block(*cfg);
  } catch (std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}

void orc_block_destroy(void* b) { delete static_cast<orc::Block*>(b); }

int orc_hydro_forward(void* b, double dt, const double* u, double* w, double* du,
                      double* mass_corr) {
  return guard("orc_hydro_forward", [&] {
    static_cast<orc::Block*>(b)->hydro_forward(dt, u, w, du, mass_corr);
  });
}

int orc_stage(void* b, int stage, double dt, double* u, double* u0, double* w, double* s,
              double* s0, double* r) {
  return guard("orc_stage",
               [&] { static_cast<orc::Block*>(b)->stage(stage, dt, u, u0, w, s, s0, r); });
}

// the hydro mass fluxes of the last hydro_forward (x1, x2, x3 order; NULL if
// the axis is inactive)
const double* orc_block_flux(void* b, int axis) {
  auto* B = static_cast<orc::Block*>(b);
  auto& f = axis == 0 ? B->F1 : (axis == 1 ? B->F2 : B->F3);
  return f.empty() ? nullptr : f.data();
}

int orc_implicit_correction(const snapb_hydro_config* cfg, double dt, double* du,
                            const double* w, double* mass) {
  return guard("orc_implicit_correction", [&] {
    orc::implicit_correction(orc::Grid(*cfg), dt, du, w, mass);
  });
}

// MS-VIC column sums + redistribution on a [n_hydro][nlayer] column (the
// entry point behind the redistribution fixture test)
void orc_vic_redistribute(double* du, const double* w, double* mass, const double* delta,
                          const double* vol, int nlayer, int n_hydro, int ny, int nblock) {
  (void)n_hydro;
  orc::vic_reduce_redistribute(du, w, mass, delta, vol, 1, nlayer, nlayer, ny, nblock);
}

}  // extern "C"
