// oracle.hpp — CPU restatement of snapy's hydro forward step (FP64).
//
// TEST INFRASTRUCTURE ONLY.  This is the checker for the CUDA product path and
// the timed CPU baseline; nothing in the shipped library links or calls it.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
// it.
//
// It follows the reference's operation order statement by statement so that
// results can be compared to ~1 ulp:
//   reconstruction grouping + edge fill  src/recon/reconstruct.cpp:46-154
//   WENO5/cp5/WENO3/cp3 point kernels    src/recon/interp_impl.h:22-122
//   PLM                                  src/recon/plm.cpp:13-36
//   HLLC / LMARS / Roe                   src/riemann/{hllc,lmars,roe}_impl.h
//   ideal-gas EOS                        src/eos/ideal_gas.cpp:30-109,
//                                        src/eos/ideal_gas_impl.h:15-35
//   hydro forward                        src/hydro/hydro_forward.cpp:14-217
//   hydrostatic revisions                src/hydro/hydro.cpp:217-269
//   divergence                           src/coord/coordinate.cpp:352-396
//   gravity                              src/forcing/const_gravity.cpp:26-45
//   diffusion                            src/forcing/diffusion.cpp:152-265
//   VIC (implicit)                       src/implicit/*_impl.h,
//                                        src/math/{ludcmp,lubksb}.h
//   scalar transport                     src/scalar/scalar.cpp:50-132
//   BCs                                  src/bc/bc_func.cpp:7-63
//   CFL                                  src/hydro/hydro.cpp:118-180
//   RK stage                             src/mesh/meshblock.cpp:577-786
//
// Build with -DORC_REFERENCE_KERNELS and -I<reference root> to replace the
// restated point kernels by the reference's own *_impl.h functions (the
// oracle/_ref build); everything else is identical in both builds.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <thread>
#include <vector>

#include "../include/snapb.h"

#ifdef ORC_REFERENCE_KERNELS
// The reference's CPU build reaches these headers after the ATen/torch
// headers, which make the floating-point ::abs overloads visible (roe_impl.h
// calls unqualified abs on doubles).  <math.h>/<stdlib.h> do the same here;
// without them abs(double) would bind to abs(int).
#include <math.h>
#include <stdlib.h>
#include <snap/eos/ideal_gas_impl.h>
#include <snap/recon/interp_impl.h>
#include <snap/riemann/hllc_impl.h>
#include <snap/riemann/lmars_impl.h>
#include <snap/riemann/roe_impl.h>
// the implicit solve, compiled against the Eigen subset in ref_shim/Eigen
#include <snap/implicit/forward_sweep_impl.h>
#include <snap/implicit/vic_assemble_full_impl.h>
#include <snap/implicit/vic_assemble_partial_impl.h>
#include <snap/implicit/vic_redistribute_impl.h>
#endif

namespace orc {

// ---------------------------------------------------------------------------
// host threading: split [0, n) into contiguous chunks over std::threads.
// Results never depend on the thread count (no cross-chunk reductions).
// ---------------------------------------------------------------------------
inline int& num_threads() {
  static int n = (int)std::max(1u, std::thread::hardware_concurrency());
  return n;
}

template <class F>
inline void par_for(int64_t n, F&& f) {
  int64_t nt = std::min<int64_t>(num_threads(), n);
  if (nt <= 1) {
    for (int64_t t = 0; t < n; ++t) f(t);
    return;
  }
  std::vector<std::thread> pool;
  pool.reserve(nt);
  for (int64_t p = 0; p < nt; ++p) {
    int64_t lo = n * p / nt, hi = n * (p + 1) / nt;
    pool.emplace_back([lo, hi, &f] {
      for (int64_t t = lo; t < hi; ++t) f(t);
    });
  }
  for (auto& th : pool) th.join();
}

enum { IDN = 0, IVX = 1, IVY = 2, IVZ = 3, IPR = 4, ICY = 5 };
enum { ILT = 0, IRT = 1 };

inline double sqr(double x) { return x * x; }

// ---------------------------------------------------------------------------
// interpolation coefficient tables (src/recon/weno5.cpp:10-24, cp5.cpp:12-16,
// weno3.cpp:10-17, cp3.cpp:12-16).  "right" uses the column-flipped table.
// ---------------------------------------------------------------------------
struct Tables {
  double weno5_m[9][5], weno5_p[9][5];
  double cp5_m[5], cp5_p[5];
  double weno3_m[4][3], weno3_p[4][3];
  double cp3_m[3], cp3_p[3];
  Tables() {
    const double w5[9][5] = {{-1. / 6., 5. / 6., 1. / 3., 0., 0.},
                             {0., 1. / 3., 5. / 6., -1. / 6., 0.},
                             {0., 0., 11. / 6., -7. / 6., 1. / 3.},
                             {1., -2., 1., 0., 0.},
                             {1., -4., 3., 0., 0.},
                             {0., 1., -2., 1., 0.},
                             {0., -1., 0., 1., 0.},
                             {0., 0., 1., -2., 1.},
                             {0., 0., 3., -4., 1.}};
    for (int r = 0; r < 9; ++r)
      for (int c = 0; c < 5; ++c) {
        weno5_m[r][c] = w5[r][c];
        weno5_p[r][c] = w5[r][4 - c];
      }
    const double c5[5] = {-1. / 20., 9. / 20., 47. / 60., -13. / 60., 1. / 30.};
    for (int c = 0; c < 5; ++c) {
      cp5_m[c] = c5[c];
      cp5_p[c] = c5[4 - c];
    }
    const double w3[4][3] = {
        {1. / 2., 1. / 2., 0.}, {0., 3. / 2., -1. / 2.}, {1., -1., 0.}, {0., 1., -1.}};
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 3; ++c) {
        weno3_m[r][c] = w3[r][c];
        weno3_p[r][c] = w3[r][2 - c];
      }
    const double c3[3] = {1. / 3., 5. / 6., -1. / 6.};
    for (int c = 0; c < 3; ++c) {
      cp3_m[c] = c3[c];
      cp3_p[c] = c3[2 - c];
    }
  }
};

inline const Tables& tables() {
  static Tables t;
  return t;
}

// running dot product in index order, starting from 0 (the reference's
// _vvdot, src/recon/interp_impl.h:12-19)
template <int N>
inline double vdot(const double* v, const double* c) {
  double o = 0.;
  for (int i = 0; i < N; ++i) o += v[i] * c[i];
  return o;
}

// WENO5-JS value from a 5-point window phi[0..4] (src/recon/interp_impl.h:73-122)
inline double weno5_value(const double* inp, const double (*c)[5], bool scale) {
#ifdef ORC_REFERENCE_KERNELS
  double out;
  snap::interp_weno5_impl<double>(&out, const_cast<double*>(inp),
                                  const_cast<double*>(&c[0][0]), 1, 0, 0, 1,
                                  scale ? 1.0 : 0.0);
  return out;
#else
  double vs = 1.0;
  if (scale)
    vs = (std::fabs(inp[0]) + std::fabs(inp[1]) + std::fabs(inp[2]) +
          std::fabs(inp[3]) + std::fabs(inp[4])) /
         5.0;
  if (vs == 0.0) return 0.0;
  double phi[5];
  for (int k = 0; k < 5; ++k) phi[k] = inp[k] / vs;
  double p0 = vdot<5>(phi, c[0]);
  double p1 = vdot<5>(phi, c[1]);
  double p2 = vdot<5>(phi, c[2]);
  double b0 = 13. / 12. * sqr(vdot<5>(phi, c[3])) + .25 * sqr(vdot<5>(phi, c[4]));
  double b1 = 13. / 12. * sqr(vdot<5>(phi, c[5])) + .25 * sqr(vdot<5>(phi, c[6]));
  double b2 = 13. / 12. * sqr(vdot<5>(phi, c[7])) + .25 * sqr(vdot<5>(phi, c[8]));
  double a0 = .3 / sqr(b0 + 1e-6);
  double a1 = .6 / sqr(b1 + 1e-6);
  double a2 = .1 / sqr(b2 + 1e-6);
  return vs * (a0 * p0 + a1 * p1 + a2 * p2) / (a0 + a1 + a2);
#endif
}

// WENO3 value from a 3-point window (src/recon/interp_impl.h:34-70)
inline double weno3_value(const double* inp, const double (*c)[3], bool scale) {
#ifdef ORC_REFERENCE_KERNELS
  double out;
  snap::interp_weno3_impl<double>(&out, const_cast<double*>(inp),
                                  const_cast<double*>(&c[0][0]), 1, 0, 0, 1,
                                  scale ? 1.0 : 0.0);
  return out;
#else
  double vs = 1.0;
  if (scale) vs = (std::fabs(inp[0]) + std::fabs(inp[1]) + std::fabs(inp[2])) / 3.0;
  if (vs == 0.0) return 0.0;
  double phi[3] = {inp[0] / vs, inp[1] / vs, inp[2] / vs};
  double p0 = vdot<3>(phi, c[0]);
  double p1 = vdot<3>(phi, c[1]);
  double b0 = sqr(vdot<3>(phi, c[2]));
  double b1 = sqr(vdot<3>(phi, c[3]));
  double a0 = (2.0 / 3.0) / sqr(b0 + 1e-6);
  double a1 = (1.0 / 3.0) / sqr(b1 + 1e-6);
  return (a0 * p0 + a1 * p1) / (a0 + a1) * vs;
#endif
}

template <int N>
inline double poly_value(const double* inp, const double* c) {
#ifdef ORC_REFERENCE_KERNELS
  double out;
  snap::interp_poly_impl<double, N>(&out, const_cast<double*>(inp),
                                    const_cast<double*>(c), 1, 0, 0, 1);
  return out;
#else
  return vdot<N>(inp, c);
#endif
}

// stencil width of an interpolation type (InterpImpl::stencils())
inline int stencil_width(int type) {
  switch (type) {
    case SNAPB_RECON_DC: return 1;
    case SNAPB_RECON_PLM:
    case SNAPB_RECON_CP3:
    case SNAPB_RECON_WENO3: return 3;
    case SNAPB_RECON_CP5:
    case SNAPB_RECON_WENO5: return 5;
  }
  throw std::runtime_error("unknown interpolation type");
}

// interp1/interp2 of a Reconstruct module (src/recon/interpolation.cpp:11-39):
// weno5 -> (weno5, cp5), weno3 -> (weno3, cp3), others -> (type, type)
inline int interp2_of(int type) {
  if (type == SNAPB_RECON_WENO5) return SNAPB_RECON_CP5;
  if (type == SNAPB_RECON_WENO3) return SNAPB_RECON_CP3;
  return type;
}

// ---------------------------------------------------------------------------
// Grid: shape, strides, uniform Cartesian metrics
// (src/coord/cartesian.cpp:8-47, src/coord/coordinate.cpp:316-331)
// ---------------------------------------------------------------------------
struct Grid {
  snapb_hydro_config c;
  int nc1, nc2, nc3, ng;
  int64_t s1, s2, s3, sv;  // strides of x1, x2, x3, variable
  double dx1, dx2, dx3;
  int il, iu, jl, ju, kl, ku;  // interior bounds (inclusive), coordinate.hpp:125-141

  explicit Grid(const snapb_hydro_config& cfg) : c(cfg) {
    ng = c.nghost;
    nc1 = c.nx1 > 1 ? c.nx1 + 2 * ng : 1;
    nc2 = c.nx2 > 1 ? c.nx2 + 2 * ng : 1;
    nc3 = c.nx3 > 1 ? c.nx3 + 2 * ng : 1;
    s1 = 1;
    s2 = nc1;
    s3 = (int64_t)nc1 * nc2;
    sv = s3 * nc3;
    dx1 = (c.x1max - c.x1min) / c.nx1;
    dx2 = (c.x2max - c.x2min) / c.nx2;
    dx3 = (c.x3max - c.x3min) / c.nx3;
    il = c.nx1 > 1 ? ng : 0;
    iu = c.nx1 > 1 ? ng + c.nx1 - 1 : 0;
    jl = c.nx2 > 1 ? ng : 0;
    ju = c.nx2 > 1 ? ng + c.nx2 - 1 : 0;
    kl = c.nx3 > 1 ? ng : 0;
    ku = c.nx3 > 1 ? ng + c.nx3 - 1 : 0;
  }
  int64_t cells() const { return sv; }
  int64_t idx(int k, int j, int i) const { return k * s3 + j * s2 + i; }
  // size and stride along a tensor dim (3 = x1, 2 = x2, 1 = x3)
  int size(int dim) const { return dim == 3 ? nc1 : (dim == 2 ? nc2 : nc3); }
  int64_t stride(int dim) const { return dim == 3 ? s1 : (dim == 2 ? s2 : s3); }
  double area1() const { return dx3 * dx2; }
  double area2() const { return dx3 * dx1; }
  double area3() const { return dx2 * dx1; }
  double vol() const { return dx3 * (dx2 * dx1); }
};

// iterate over all lines along `dim`: calls f(base_offset)
template <class F>
inline void for_lines(const Grid& g, int dim, F&& f) {
  int n3 = g.nc3, n2 = g.nc2, n1 = g.nc1;
  if (dim == 3) n1 = 1;
  if (dim == 2) n2 = 1;
  if (dim == 1) n3 = 1;
  int64_t total = (int64_t)n3 * n2 * n1;
  par_for(total, [&](int64_t t) {
    int i = (int)(t % n1);
    int j = (int)((t / n1) % n2);
    int k = (int)(t / ((int64_t)n1 * n2));
    f(g.idx(k, j, i));
  });
}

// ---------------------------------------------------------------------------
// ideal-gas EOS (src/eos/ideal_gas.cpp, src/eos/ideal_gas_impl.h)
// ---------------------------------------------------------------------------
inline void cons2prim_cell(double* prim, const double* cons, double gammad,
                           int64_t sv) {
#ifdef ORC_REFERENCE_KERNELS
  double cth = 0.;
  snap::ideal_gas_cons2prim<double>(prim, const_cast<double*>(cons), &cth, gammad,
                                    (int)sv);
#else
  prim[IDN * sv] = cons[IDN * sv];
  prim[IVX * sv] = cons[IVX * sv] / prim[IDN * sv];
  prim[IVY * sv] = cons[IVY * sv] / prim[IDN * sv];
  prim[IVZ * sv] = cons[IVZ * sv] / prim[IDN * sv];
  // covariant -> contravariant with cos(theta) = 0 (Cartesian): v - w*0, w + (-v*0)
  double v = prim[IVY * sv], w = prim[IVZ * sv];
  prim[IVY * sv] = v / 1. - w * 0. / 1.;
  prim[IVZ * sv] = -v * 0. / 1. + w / 1.;
  double ke = 0.5 * (prim[IVX * sv] * cons[IVX * sv] + prim[IVY * sv] * cons[IVY * sv] +
                     prim[IVZ * sv] * cons[IVZ * sv]);
  double ie = cons[IPR * sv] - ke;
  prim[IPR * sv] = (gammad - 1.) * ie;
#endif
}

inline void cons2prim(const Grid& g, const double* u, double* w) {
  int64_t n = g.cells();
  double gd = g.c.gammad;
  par_for(n, [&](int64_t t) { cons2prim_cell(w + t, u + t, gd, g.sv); });
}

inline void prim2cons(const Grid& g, const double* w, double* u) {
  int64_t n = g.cells(), sv = g.sv;
  double gm1 = g.c.gammad - 1;
  par_for(n, [&](int64_t t) {
    const double* p = w + t;
    double* q = u + t;
    q[IDN * sv] = p[IDN * sv];
    double m1 = p[IVX * sv] * p[IDN * sv];
    double m2 = p[IVY * sv] * p[IDN * sv];
    double m3 = p[IVZ * sv] * p[IDN * sv];
    // lower index with cos(theta) = 0: v + w*0
    double l2 = m2 + m3 * 0.;
    double l3 = m3 + m2 * 0.;
    q[IVX * sv] = m1;
    q[IVY * sv] = l2;
    q[IVZ * sv] = l3;
    double ke = 0.5 * (p[IVX * sv] * m1 + p[IVY * sv] * l2 + p[IVZ * sv] * l3);
    q[IPR * sv] = p[IPR * sv] / gm1;
    q[IPR * sv] += ke;
  });
}

// ---------------------------------------------------------------------------
// Reconstruction along `dim` (src/recon/reconstruct.cpp:46-154)
// wlr layout: [2][nv][cells]
// ---------------------------------------------------------------------------
// value at the left face of window-centred cell (side IRT output) or the right
// face (side ILT output) from the window starting at `in` with stride `st`.
inline double interp_value(int type, int side, const double* in, int64_t st,
                           bool scale) {
  const Tables& T = tables();
  double win[5];
  int N = stencil_width(type);
  for (int k = 0; k < N; ++k) win[k] = in[k * st];
  bool left = (side == IRT);  // "left" interpolation fills wlr[IRT]
  switch (type) {
    case SNAPB_RECON_DC: return win[0];
    case SNAPB_RECON_CP3: return poly_value<3>(win, left ? T.cp3_m : T.cp3_p);
    case SNAPB_RECON_CP5: return poly_value<5>(win, left ? T.cp5_m : T.cp5_p);
    case SNAPB_RECON_WENO3: return weno3_value(win, left ? T.weno3_m : T.weno3_p, scale);
    case SNAPB_RECON_WENO5: return weno5_value(win, left ? T.weno5_m : T.weno5_p, scale);
  }
  throw std::runtime_error("interp_value: bad type");
}

// one variable line: fills wl (ILT) and wr (IRT) along the line, reference
// window conventions, then replicates the edges
inline void recon_line(int type, bool scale, const double* w, int64_t st, int n,
                       double* wl, double* wr) {
  int N = stencil_width(type);
  int r = N / 2;
  int il = r + 1, iu = n - (r + 1);
  if (il > iu) throw std::runtime_error("il > iu");
  if (type == SNAPB_RECON_PLM) {
    // src/recon/plm.cpp:13-36 on positions 1..n-2
    for (int o = 1; o <= n - 2; ++o) {
      double dl = w[o * st] - w[(o - 1) * st];
      double dr = w[(o + 1) * st] - w[o * st];
      double dw2 = dl * dr;
      double dwm = 2. * dw2 / (dl + dr + (double)std::numeric_limits<float>::min());
      dwm *= (dw2 >= 0) ? 1 : 0;
      wr[o * st] = w[o * st] - 0.5 * dwm;        // wlr[IRT] slot o
      wl[(o + 1) * st] = w[o * st] + 0.5 * dwm;  // wlr[ILT] slot o+1
    }
  } else {
    for (int o = il - 1; o <= iu; ++o)
      wr[o * st] = interp_value(type, IRT, w + (o - r) * st, st, scale);
    int ohi = std::min(iu + 1, n - 1);
    for (int o = il; o <= ohi; ++o)
      wl[o * st] = interp_value(type, ILT, w + (o - r - 1) * st, st, scale);
  }
  // populate dummy regions (reconstruct.cpp:56-60)
  double v;
  v = wr[il * st];
  for (int o = 0; o < il; ++o) wr[o * st] = v;
  v = wr[iu * st];
  for (int o = iu + 1; o < n; ++o) wr[o * st] = v;
  v = wl[il * st];
  for (int o = 0; o < il; ++o) wl[o * st] = v;
  v = wl[iu * st];
  for (int o = iu + 1; o < n; ++o) wl[o * st] = v;
}

// group 0 = hydro (uses recon1 for dim 3, recon23 otherwise), 1 = scalars
inline void reconstruct(const Grid& g, int dim, int group, const double* w, int nv,
                        double* wlr) {
  int type, shock, scale;
  if (group == 1) {
    type = g.c.scalar_recon_type;
    shock = 1;
    scale = g.c.scalar_recon_scale;
  } else if (dim == 3) {
    type = g.c.recon1_type;
    shock = g.c.recon1_shock;
    scale = g.c.recon1_scale;
  } else {
    type = g.c.recon23_type;
    shock = g.c.recon23_shock;
    scale = g.c.recon23_scale;
  }
  int n = g.size(dim);
  int64_t st = g.stride(dim), sv = g.sv;
  std::fill(wlr, wlr + 2 * (int64_t)nv * sv, 0.0);
  double* wl = wlr;
  double* wr = wlr + (int64_t)nv * sv;
  for_lines(g, dim, [&](int64_t base) {
    for (int v = 0; v < nv; ++v) {
      int t = type;
      if (!shock && v >= IVX && v <= IPR) t = interp2_of(type);
      recon_line(t, scale, w + v * sv + base, st, n, wl + v * sv + base,
                 wr + v * sv + base);
    }
  });
  if (group == 1) {  // no hydro parent: clamp_min(0) on the whole result
    int64_t tot = 2 * (int64_t)nv * sv;
    for (int64_t t = 0; t < tot; ++t)
      if (wlr[t] < 0.) wlr[t] = 0.;
  }
}

// ---------------------------------------------------------------------------
// Riemann solvers at one face; arrays with stride sv between variables
// ---------------------------------------------------------------------------
inline void hllc_face(double* flx, const double* wl, const double* wr, double el,
                      double er, double gl, double gr, double cl, double cr, int dim,
                      int ny, int64_t sw, int64_t sf, double* fp) {
#ifdef ORC_REFERENCE_KERNELS
  snap::hllc_impl<double>(flx, const_cast<double*>(wl), const_cast<double*>(wr), el,
                          er, gl, gr, cl, cr, dim, ny, (int)sw, (int)sf, fp);
#else
  const double TINY = 1.0e-10;
  int ivx = IPR - dim;
  int ivy = IVX + ((ivx - IVX) + 1) % 3;
  int ivz = IVX + ((ivx - IVX) + 2) % 3;
#define WL(n) wl[(n) * sw]
#define WR(n) wr[(n) * sw]
#define FX(n) flx[(n) * sf]
  el += 0.5 * WL(IDN) * (sqr(WL(IVX)) + sqr(WL(IVY)) + sqr(WL(IVZ)));
  er += 0.5 * WR(IDN) * (sqr(WR(IVX)) + sqr(WR(IVY)) + sqr(WR(IVZ)));
  double rhoa = .5 * (WL(IDN) + WR(IDN));
  double ca = .5 * (cl + cr);
  double pmid = .5 * (WL(IPR) + WR(IPR) + (WL(ivx) - WR(ivx)) * rhoa * ca);
  double ql = (pmid <= WL(IPR))
                  ? 1.0
                  : std::sqrt(1.0 + (gl + 1) / (2 * gl) * (pmid / WL(IPR) - 1.0));
  double qr = (pmid <= WR(IPR))
                  ? 1.0
                  : std::sqrt(1.0 + (gr + 1) / (2 * gr) * (pmid / WR(IPR) - 1.0));
  double al = WL(ivx) - cl * ql;
  double ar = WR(ivx) + cr * qr;
  double bp = ar > 0.0 ? ar : TINY;
  double bm = al < 0.0 ? al : -TINY;
  double vxl = WL(ivx) - al;
  double vxr = WR(ivx) - ar;
  double tl = WL(IPR) + vxl * WL(IDN) * WL(ivx);
  double tr = WR(IPR) + vxr * WR(IDN) * WR(ivx);
  double ml = WL(IDN) * vxl;
  double mr = -(WR(IDN) * vxr);
  double am = (tl - tr) / (ml + mr);
  double cp = (ml * tr + mr * tl) / (ml + mr);
  cp = cp > 0.0 ? cp : 0.0;
  if (fp) *fp = cp;
  vxl = WL(ivx) - bm;
  vxr = WR(ivx) - bp;
  double rdl = 1., rdr = 1.;
  for (int n = 0; n < ny; ++n) {
    rdl -= WL(ICY + n);
    rdr -= WR(ICY + n);
  }
  double fl[5], fr[5];
  fl[IDN] = WL(IDN) * vxl * rdl;
  fr[IDN] = WR(IDN) * vxr * rdr;
  fl[ivx] = WL(IDN) * WL(ivx) * vxl + WL(IPR);
  fr[ivx] = WR(IDN) * WR(ivx) * vxr + WR(IPR);
  fl[ivy] = WL(IDN) * WL(ivy) * vxl;
  fr[ivy] = WR(IDN) * WR(ivy) * vxr;
  fl[ivz] = WL(IDN) * WL(ivz) * vxl;
  fr[ivz] = WR(IDN) * WR(ivz) * vxr;
  fl[IPR] = el * vxl + WL(IPR) * WL(ivx);
  fr[IPR] = er * vxr + WR(IPR) * WR(ivx);
  double sl, sr, sm;
  if (am >= 0.0) {
    sl = am / (am - bm);
    sr = 0.0;
    sm = -bm / (am - bm);
  } else {
    sl = 0.0;
    sr = -am / (bp - am);
    sm = bp / (bp - am);
  }
  FX(IDN) = sl * fl[IDN] + sr * fr[IDN];
  FX(ivx) = sl * fl[ivx] + sr * fr[ivx] + sm * cp;
  FX(ivy) = sl * fl[ivy] + sr * fr[ivy];
  FX(ivz) = sl * fl[ivz] + sr * fr[ivz];
  FX(IPR) = sl * fl[IPR] + sr * fr[IPR] + sm * cp * am;
  for (int n = 0; n < ny; ++n) {
    double fln = WL(IDN) * WL(ICY + n) * vxl;
    double frn = WR(IDN) * WR(ICY + n) * vxr;
    FX(ICY + n) = sl * fln + sr * frn;
  }
#undef WL
#undef WR
#undef FX
#endif
}

inline void lmars_face(double* flx, const double* wl, const double* wr, double hl,
                       double hr, double gl, double gr, int dim, int ny, int64_t sw,
                       int64_t sf, double* fp) {
#ifdef ORC_REFERENCE_KERNELS
  snap::lmars_impl<double>(flx, const_cast<double*>(wl), const_cast<double*>(wr), hl,
                           hr, gl, gr, dim, ny, (int)sw, (int)sf, fp);
#else
  int ivx = IPR - dim;
  int ivy = IVX + ((ivx - IVX) + 1) % 3;
  int ivz = IVX + ((ivx - IVX) + 2) % 3;
#define WL(n) wl[(n) * sw]
#define WR(n) wr[(n) * sw]
#define FX(n) flx[(n) * sf]
  double wli[5] = {WL(IDN), WL(ivx), WL(ivy), WL(ivz), WL(IPR)};
  double wri[5] = {WR(IDN), WR(ivx), WR(ivy), WR(ivz), WR(IPR)};
  hl += 0.5 * (sqr(wli[IVX]) + sqr(wli[IVY]) + sqr(wli[IVZ])) + wli[IPR] / wli[IDN];
  hr += 0.5 * (sqr(wri[IVX]) + sqr(wri[IVY]) + sqr(wri[IVZ])) + wri[IPR] / wri[IDN];
  double rhobar = 0.5 * (wli[IDN] + wri[IDN]);
  double gbar = 0.5 * (gl + gr);
  double cbar = std::sqrt(0.5 * gbar * (wli[IPR] + wri[IPR]) / rhobar);
  double pbar = 0.5 * (wli[IPR] + wri[IPR]) + 0.5 * (rhobar * cbar) * (wli[IVX] - wri[IVX]);
  if (fp) *fp = pbar;
  double ubar = 0.5 * (wli[IVX] + wri[IVX]) + 0.5 / (rhobar * cbar) * (wli[IPR] - wri[IPR]);
  double rd = 1.0;
  if (ubar > 0.0) {
    for (int n = 0; n < ny; n++) rd -= WL(ICY + n);
    FX(IDN) = ubar * wli[IDN] * rd;
    for (int n = 0; n < ny; n++) FX(ICY + n) = ubar * wli[IDN] * WL(ICY + n);
    FX(ivx) = ubar * wli[IDN] * wli[IVX] + pbar;
    FX(ivy) = ubar * wli[IDN] * wli[IVY];
    FX(ivz) = ubar * wli[IDN] * wli[IVZ];
    FX(IPR) = ubar * wli[IDN] * hl;
  } else {
    for (int n = 0; n < ny; n++) rd -= WR(ICY + n);
    FX(IDN) = ubar * wri[IDN] * rd;
    for (int n = 0; n < ny; n++) FX(ICY + n) = ubar * wri[IDN] * WR(ICY + n);
    FX(ivx) = ubar * wri[IDN] * wri[IVX] + pbar;
    FX(ivy) = ubar * wri[IDN] * wri[IVY];
    FX(ivz) = ubar * wri[IDN] * wri[IVZ];
    FX(IPR) = ubar * wri[IDN] * hr;
  }
#undef WL
#undef WR
#undef FX
#endif
}

inline void roe_face(double* flx, const double* wl, const double* wr, double el,
                     double er, double gl, double gr, double cl, double cr, int dim,
                     int ny, int64_t sw, int64_t sf, double* fp) {
#ifdef ORC_REFERENCE_KERNELS
  snap::roe_impl<double>(flx, wl, wr, el, er, gl, gr, cl, cr, dim, ny, false, 0, 1.4,
                         nullptr, nullptr, nullptr, (int)sw, (int)sf, fp);
#else
  const double TINY = 1.0e-10;
  int ivx = IPR - dim;
  int ivy = IVX + ((ivx - IVX) + 1) % 3;
  int ivz = IVX + ((ivx - IVX) + 2) % 3;
#define WL(n) wl[(n) * sw]
#define WR(n) wr[(n) * sw]
#define FX(n) flx[(n) * sf]
  double etl = el + 0.5 * WL(IDN) * (sqr(WL(IVX)) + sqr(WL(IVY)) + sqr(WL(IVZ)));
  double etr = er + 0.5 * WR(IDN) * (sqr(WR(IVX)) + sqr(WR(IVY)) + sqr(WR(IVZ)));
  double sdl = std::sqrt(WL(IDN));
  double sdr = std::sqrt(WR(IDN));
  double isd = 1. / (sdl + sdr);
  double rhobar = sdl * sdr;
  double v1 = (sdl * WL(ivx) + sdr * WR(ivx)) * isd;
  double v2 = (sdl * WL(ivy) + sdr * WR(ivy)) * isd;
  double v3 = (sdl * WL(ivz) + sdr * WR(ivz)) * isd;
  double hl = (etl + WL(IPR)) / WL(IDN);
  double hr = (etr + WR(IPR)) / WR(IDN);
  double h = (hl * sdl + hr * sdr) * isd;
  double dryl = 1., dryr = 1.;
  for (int n = 0; n < ny; ++n) {
    dryl -= WL(ICY + n);
    dryr -= WR(ICY + n);
  }
  double rhol0 = WL(IDN) * dryl, rhor0 = WR(IDN) * dryr;
  double fl0 = rhol0 * WL(ivx), fr0 = rhor0 * WR(ivx);
  double fl1 = WL(IDN) * WL(ivx) * WL(ivx) + WL(IPR);
  double fr1 = WR(IDN) * WR(ivx) * WR(ivx) + WR(IPR);
  double fl2 = WL(IDN) * WL(ivx) * WL(ivy), fr2 = WR(IDN) * WR(ivx) * WR(ivy);
  double fl3 = WL(IDN) * WL(ivx) * WL(ivz), fr3 = WR(IDN) * WR(ivx) * WR(ivz);
  double fl4 = (etl + WL(IPR)) * WL(ivx), fr4 = (etr + WR(IPR)) * WR(ivx);
  double qbar[64];
  qbar[0] = (rhol0 / sdl + rhor0 / sdr) * isd;
  for (int n = 0; n < ny; ++n) {
    double rl = WL(IDN) * WL(ICY + n), rr = WR(IDN) * WR(ICY + n);
    qbar[1 + n] = (rl / sdl + rr / sdr) * isd;
  }
  double gamma_roe = 0.5 * (gl + gr);
  double offset = 0.;
  double du1 = WR(IDN) * WR(ivx) - WL(IDN) * WL(ivx);
  double du2 = WR(IDN) * WR(ivy) - WL(IDN) * WL(ivy);
  double du3 = WR(IDN) * WR(ivz) - WL(IDN) * WL(ivz);
  double du4 = etr - etl;
  FX(IDN) = 0.5 * (fl0 + fr0);
  FX(ivx) = 0.5 * (fl1 + fr1);
  FX(ivy) = 0.5 * (fl2 + fr2);
  FX(ivz) = 0.5 * (fl3 + fr3);
  FX(IPR) = 0.5 * (fl4 + fr4);
  for (int n = 0; n < ny; ++n) {
    double rl = WL(IDN) * WL(ICY + n), rr = WR(IDN) * WR(ICY + n);
    FX(ICY + n) = 0.5 * (rl * WL(ivx) + rr * WR(ivx));
  }
  double vsq = v1 * v1 + v2 * v2 + v3 * v3;
  double gm1 = gamma_roe - 1.;
  double q = h - 0.5 * vsq - offset;
  double cs_sq = std::max(gm1 * std::max(q, TINY), TINY);
  double cs = std::sqrt(cs_sq);
  if (fp) *fp = 0.5 * (WL(IPR) + WR(IPR) + rhobar * cs * (WL(ivx) - WR(ivx)));
  double lam_m = v1 - cs, lam_0 = v1, lam_p = v1 + cs;
  double spd_m = std::fabs(lam_m), spd_0 = std::fabs(lam_0), spd_p = std::fabs(lam_p);
  bool llf = false;
  double du = WR(ivx) - WL(ivx), dv = WR(ivy) - WL(ivy), dw = WR(ivz) - WL(ivz);
  double dp = WR(IPR) - WL(IPR);
  double alpha_m = -0.5 * rhobar / cs * du + 0.5 * dp / cs_sq;
  double alpha_p = +0.5 * rhobar / cs * du + 0.5 * dp / cs_sq;
  double alpha_v = rhobar * dv, alpha_w = rhobar * dw;
  double alpha0 = 0.;
  double ac0 = rhor0 - rhol0 - dp / cs_sq * qbar[0];
  double rho1 = rhol0 + alpha_m * qbar[0];
  if (rho1 < 0.) llf = true;
  double rho2 = rho1 + ac0;
  if (rho2 < 0.) llf = true;
  alpha0 += ac0;
  FX(IDN) -= 0.5 * (spd_m * alpha_m * qbar[0] + spd_0 * ac0 + spd_p * alpha_p * qbar[0]);
  for (int n = 0; n < ny; ++n) {
    double rl = WL(IDN) * WL(ICY + n), rr = WR(IDN) * WR(ICY + n);
    double an = rr - rl - dp / cs_sq * qbar[1 + n];
    double r1 = rl + alpha_m * qbar[1 + n];
    if (r1 < 0.) llf = true;
    double r2 = r1 + an;
    if (r2 < 0.) llf = true;
    alpha0 += an;
    FX(ICY + n) -= 0.5 * (spd_m * alpha_m * qbar[1 + n] + spd_0 * an +
                          spd_p * alpha_p * qbar[1 + n]);
  }
  FX(ivx) -= 0.5 * (spd_m * alpha_m * (v1 - cs) + spd_0 * (v1 * alpha0) +
                    spd_p * alpha_p * (v1 + cs));
  FX(ivy) -= 0.5 * (spd_m * alpha_m * v2 + spd_0 * (v2 * alpha0 + alpha_v) +
                    spd_p * alpha_p * v2);
  FX(ivz) -= 0.5 * (spd_m * alpha_m * v3 + spd_0 * (v3 * alpha0 + alpha_w) +
                    spd_p * alpha_p * v3);
  FX(IPR) -= 0.5 * (spd_m * alpha_m * (h - v1 * cs) +
                    spd_0 * (rhobar * (hr - hl - v1 * du) + alpha0 * h - dp) +
                    spd_p * alpha_p * (h + v1 * cs));
  if (lam_m > 0.) {
    FX(IDN) = fl0;
    FX(ivx) = fl1;
    FX(ivy) = fl2;
    FX(ivz) = fl3;
    FX(IPR) = fl4;
    for (int n = 0; n < ny; ++n) FX(ICY + n) = WL(IDN) * WL(ICY + n) * WL(ivx);
  }
  if (lam_p < 0.) {
    FX(IDN) = fr0;
    FX(ivx) = fr1;
    FX(ivy) = fr2;
    FX(ivz) = fr3;
    FX(IPR) = fr4;
    for (int n = 0; n < ny; ++n) FX(ICY + n) = WR(IDN) * WR(ICY + n) * WR(ivx);
  }
  if (llf) {
    double a = 0.5 * std::max(std::fabs(WL(ivx)) + cl, std::fabs(WR(ivx)) + cr);
    FX(IDN) = 0.5 * (fl0 + fr0) - a * (rhor0 - rhol0);
    FX(ivx) = 0.5 * (fl1 + fr1) - a * du1;
    FX(ivy) = 0.5 * (fl2 + fr2) - a * du2;
    FX(ivz) = 0.5 * (fl3 + fr3) - a * du3;
    FX(IPR) = 0.5 * (fl4 + fr4) - a * du4;
    for (int n = 0; n < ny; ++n) {
      double rl = WL(IDN) * WL(ICY + n), rr = WR(IDN) * WR(ICY + n);
      FX(ICY + n) = 0.5 * (rl * WL(ivx) + rr * WR(ivx)) - a * (rr - rl);
    }
  }
#undef WL
#undef WR
#undef FX
#endif
}

// Riemann solve at every position of the arrays (the reference iterates over
// the whole [nc3, nc2, nc1] index space).  EOS helpers as the modules compute
// them: W->I = p/(gammad-1), W->A = gammad, WA->L = sqrt(gamma*p/rho).
inline void riemann(const Grid& g, int solver, int dim, const double* wl,
                    const double* wr, int nv, double* flx, double* fp,
                    const double* vel) {
  int64_t n = g.cells(), sv = g.sv;
  double gd = g.c.gammad;
  int ny = nv - ICY;
  par_for(n, [&](int64_t t) {
    const double* L = wl + t;
    const double* R = wr + t;
    double* F = flx + t;
    double* P = fp ? fp + t : nullptr;
    if (solver == SNAPB_RIEMANN_UPWIND) {
      // src/riemann/riemann_solver.cpp:544-553
      double ve = vel[t];
      int ui = ve > 0 ? 1 : 0;
      for (int v = 0; v < nv; ++v)
        F[v * sv] = ve * (ui * L[v * sv] + (1 - ui) * R[v * sv]);
      return;
    }
    double el = L[IPR * sv] / (gd - 1);
    double er = R[IPR * sv] / (gd - 1);
    double gl = gd, gr = gd;
    if (solver == SNAPB_RIEMANN_LMARS) {
      lmars_face(F, L, R, el / L[IDN * sv], er / R[IDN * sv], gl, gr, dim, ny, sv, sv, P);
    } else {
      double cl = std::sqrt(gl * L[IPR * sv] / L[IDN * sv]);
      double cr = std::sqrt(gr * R[IPR * sv] / R[IDN * sv]);
      if (solver == SNAPB_RIEMANN_HLLC)
        hllc_face(F, L, R, el, er, gl, gr, cl, cr, dim, ny, sv, sv, P);
      else
        roe_face(F, L, R, el, er, gl, gr, cl, cr, dim, ny, sv, sv, P);
    }
  });
}

// ---------------------------------------------------------------------------
// Boundary conditions (src/bc/bc_func.cpp:7-63) applied in order x1-inner,
// x1-outer, x2-inner, x2-outer, x3-inner, x3-outer (meshblock.cpp:717-730)
// ---------------------------------------------------------------------------
inline void bc_apply(const Grid& g, double* var, int nv, int kind) {
  int ng = g.ng;
  for (int b = 0; b < 6; ++b) {
    int dim = 3 - b / 2;  // tensor dim of the var without its leading nv axis + 1
    int n = g.size(dim);
    if (n == 1) continue;
    int type = g.c.bc[b];
    bool inner = (b % 2) == 0;
    int64_t st = g.stride(dim);
    int normal = 4 - dim;  // var[4 - dim] is the normal velocity / momentum
    bool flip = (kind == SNAPB_CONSERVED || kind == SNAPB_PRIMITIVE);
    for (int v = 0; v < nv; ++v) {
      double* base = var + v * g.sv;
      for_lines(g, dim, [&](int64_t off) {
        double* L = base + off;
        for (int q = 0; q < ng; ++q) {
          int dst, src;
          double sgn = 1.0;
          if (type == SNAPB_BC_CUSTOM) return;
          if (type == SNAPB_BC_REFLECTING) {
            dst = inner ? q : n - ng + q;
            src = inner ? 2 * ng - 1 - q : n - ng - 1 - q;
            if (flip && v == normal) sgn = -1.0;
          } else if (type == SNAPB_BC_PERIODIC) {
            dst = inner ? q : n - ng + q;
            src = inner ? n - 2 * ng + q : ng + q;
          } else {  // outflow
            dst = inner ? q : n - ng + q;
            src = inner ? ng : n - ng - 1;
          }
          L[dst * st] = L[src * st] * sgn;
        }
      });
    }
  }
}

// ---------------------------------------------------------------------------
// Hydrostatic revisions (src/hydro/hydro.cpp:217-269)
// ---------------------------------------------------------------------------
inline void revise_x1_ghosts(const Grid& g, double* w) {
  double grav = -g.c.grav1;
  double gamma = g.c.gammad;
  double gm = gamma - 1.;
  double a = gm / gamma;
  double ig = 1. / gamma;
  double ia = 1. / a;
  int is = g.il, ie = g.iu;
  double dz = g.dx1;
  int64_t sv = g.sv;
  int64_t ncol = (int64_t)g.nc2 * g.nc3;
  par_for(ncol, [&](int64_t col) {
    double* p = w + IPR * sv + col * g.nc1;
    double* r = w + IDN * sv + col * g.nc1;
    double K = p[is] / std::pow(r[is], gamma);
    for (int n = 0; n < g.ng; ++n) {
      double h = std::pow(p[is - n], a) + a * grav * dz / std::pow(K, ig);
      p[is - n - 1] = std::pow(h, ia);
      r[is - n - 1] = std::pow(p[is - n - 1] / K, ig);
    }
    K = p[ie] / std::pow(r[ie], gamma);
    for (int n = 0; n < g.ng; ++n) {
      double h = std::pow(p[ie + n], a) - a * grav * dz / std::pow(K, ig);
      p[ie + n + 1] = std::pow(h, ia);
      r[ie + n + 1] = std::pow(p[ie + n + 1] / K, ig);
    }
  });
}

// ---------------------------------------------------------------------------
// VIC: vertically implicit correction (src/implicit/*)
// ---------------------------------------------------------------------------
template <int N>
struct Mat {
  double m[N][N];
};

template <int N>
inline void matmul(const Mat<N>& A, const Mat<N>& B, Mat<N>& C) {
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) {
      double s = A.m[i][0] * B.m[0][j];
      for (int k = 1; k < N; ++k) s += A.m[i][k] * B.m[k][j];
      C.m[i][j] = s;
    }
}

template <int N>
inline void matvec(const Mat<N>& A, const double* x, double* y) {
  for (int i = 0; i < N; ++i) {
    double s = A.m[i][0] * x[0];
    for (int k = 1; k < N; ++k) s += A.m[i][k] * x[k];
    y[i] = s;
  }
}

// 3x3 inverse by cofactors over the determinant (expansion along column 0)
inline void inv3(const Mat<3>& A, Mat<3>& R) {
  auto cof = [&](int i, int j) {
    int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
    return A.m[i1][j1] * A.m[i2][j2] - A.m[i1][j2] * A.m[i2][j1];
  };
  double c0 = cof(0, 0), c1 = cof(1, 0), c2 = cof(2, 0);
  double det = c0 * A.m[0][0] + c1 * A.m[1][0] + c2 * A.m[2][0];
  double id = 1. / det;
  // R(i, j) = cofactor(j, i) / det
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) R.m[i][j] = cof(j, i) * id;
}

// LU decomposition with implicit-scaling partial pivoting (Crout), the
// published Numerical Recipes ludcmp method used by src/math/ludcmp.h:24-76
template <int N>
inline int lu_decompose(Mat<N>& a, int* indx) {
  double vv[N];
  for (int i = 0; i < N; ++i) {
    double big = 0.0;
    for (int j = 0; j < N; ++j) big = std::max(big, std::fabs(a.m[i][j]));
    if (big == 0.0) return 1;
    vv[i] = 1.0 / big;
  }
  for (int j = 0; j < N; ++j) {
    for (int i = 0; i < j; ++i) {
      double s = a.m[i][j];
      for (int k = 0; k < i; ++k) s -= a.m[i][k] * a.m[k][j];
      a.m[i][j] = s;
    }
    double big = 0.0;
    int imax = 0;
    for (int i = j; i < N; ++i) {
      double s = a.m[i][j];
      for (int k = 0; k < j; ++k) s -= a.m[i][k] * a.m[k][j];
      a.m[i][j] = s;
      double d = vv[i] * std::fabs(s);
      if (d >= big) {
        big = d;
        imax = i;
      }
    }
    if (j != imax) {
      for (int k = 0; k < N; ++k) std::swap(a.m[imax][k], a.m[j][k]);
      vv[imax] = vv[j];
    }
    indx[j] = imax;
    if (j != N - 1) {
      double d = 1.0 / a.m[j][j];
      for (int i = j + 1; i < N; ++i) a.m[i][j] *= d;
    }
  }
  return 0;
}

// forward/back substitution of M right-hand-side columns stored row-wise in
// b[N][M] (row swaps applied as the decomposition recorded them;
// src/math/lubksb.h:124-147)
template <int N, int M>
inline void lu_solve(const Mat<N>& a, const int* indx, double (&b)[N][M]) {
  for (int i = 0; i < N; ++i) {
    int ip = indx[i];
    if (ip != i)
      for (int c = 0; c < M; ++c) std::swap(b[ip][c], b[i][c]);
    for (int j = 0; j < i; ++j)
      for (int c = 0; c < M; ++c) b[i][c] -= a.m[i][j] * b[j][c];
  }
  for (int i = N - 1; i >= 0; --i) {
    for (int j = i + 1; j < N; ++j)
      for (int c = 0; c < M; ++c) b[i][c] -= a.m[i][j] * b[j][c];
    for (int c = 0; c < M; ++c) b[i][c] /= a.m[i][i];
  }
}

// flux Jacobian dF/dU of the Euler flux along x1 at primitive state w
// (src/implicit/flux_decomposition_impl.h:224-245), 5x5
inline void flux_jacobian(Mat<5>& J, double gm1, const double* w) {
  double v1 = w[IVX], v2 = w[IVY], v3 = w[IVZ];
  double rho = w[IDN], pres = w[IPR];
  double s2 = v1 * v1 + v2 * v2 + v3 * v3;
  double c1 = ((gm1 - 1) * s2 / 2 - (gm1 + 1) / gm1 * pres / rho) * v1;
  double c2 = (gm1 + 1) / gm1 * pres / rho + s2 / 2 - gm1 * v1 * v1;
  double r[5][5] = {
      {0, 1., 0., 0., 0.},
      {gm1 * s2 / 2 - v1 * v1, (2. - gm1) * v1, -gm1 * v2, -gm1 * v3, gm1},
      {-v1 * v2, v2, v1, 0., 0.},
      {-v1 * v3, v3, 0., v1, 0.},
      {c1, c2, -gm1 * v2 * v1, -gm1 * v3 * v1, (gm1 + 1) * v1}};
  std::memcpy(J.m, r, sizeof(r));
}

// Roe-averaged state and |A| = R |Lambda| R^-1 at an interface
// (flux_decomposition_impl.h:133-222)
inline void roe_abs_jacobian(Mat<5>& A, double gm1, const double* wl, const double* wr) {
  double prim[5];
  double sdl = std::sqrt(wl[IDN]), sdr = std::sqrt(wr[IDN]);
  double isd = 1.0 / (sdl + sdr);
  prim[IDN] = sdl * sdr;
  prim[IVX] = (sdl * wl[IVX] + sdr * wr[IVX]) * isd;
  prim[IVY] = (sdl * wl[IVY] + sdr * wr[IVY]) * isd;
  prim[IVZ] = (sdl * wl[IVZ] + sdr * wr[IVZ]) * isd;
  double el = wl[IPR] / gm1 + 0.5 * wl[IDN] * (sqr(wl[IVX]) + sqr(wl[IVY]) + sqr(wl[IVZ]));
  double er = wr[IPR] / gm1 + 0.5 * wr[IDN] * (sqr(wr[IVX]) + sqr(wr[IVY]) + sqr(wr[IVZ]));
  double hbar = ((el + wl[IPR]) / sdl + (er + wr[IPR]) / sdr) * isd;
  prim[IPR] = (hbar - 0.5 * (sqr(prim[IVX]) + sqr(prim[IVY]) + sqr(prim[IVZ]))) * gm1 /
              (gm1 + 1.) * prim[IDN];
  double cs = std::sqrt(prim[IPR] * (gm1 + 1.) / prim[IDN]);
  double r = prim[IDN], u = prim[IVX], v = prim[IVY], w = prim[IVZ], p = prim[IPR];
  double lam[5] = {std::fabs(u - cs), std::fabs(u), std::fabs(u + cs), std::fabs(u),
                   std::fabs(u)};
  double ke = 0.5 * (u * u + v * v + w * w);
  double hp = (gm1 + 1.) / gm1 * p / r;
  double h = hp + ke;
  double R[5][5] = {{1., 1., 1., 0., 0.},
                    {u - cs, u, u + cs, 0., 0.},
                    {v, v, v, 1., 0.},
                    {w, w, w, 0., 1.},
                    {h - u * cs, ke, h + u * cs, v, w}};
  double Ri[5][5] = {{(cs * ke + u * hp) / (2. * cs * hp), (-hp - cs * u) / (2. * cs * hp),
                      -v / (2. * hp), -w / (2. * hp), 1. / (2. * hp)},
                     {(hp - ke) / hp, u / hp, v / hp, w / hp, -1. / hp},
                     {(cs * ke - u * hp) / (2. * cs * hp), (hp - cs * u) / (2. * cs * hp),
                      -v / (2. * hp), -w / (2. * hp), 1. / (2. * hp)},
                     {-v, 0., 1., 0., 0.},
                     {-w, 0., 0., 1., 0.}};
  // (R * diag(lam)) * Ri
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 5; ++j) {
      double s = (R[i][0] * lam[0]) * Ri[0][j];
      for (int k = 1; k < 5; ++k) s += (R[i][k] * lam[k]) * Ri[k][j];
      A.m[i][j] = s;
    }
}

// rows/cols kept by the partial (3x3) scheme: IDN, IVX, IPR
static const int kPart[3] = {IDN, IVX, IPR};

template <int N>
inline void sub_block(const Mat<5>& A, Mat<N>& B) {
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j)
      B.m[i][j] = (N == 3) ? A.m[kPart[i]][kPart[j]] : A.m[i][j];
}

// Column sums and per-cell MS-VIC redistribution after the back
// substitution (src/implicit/vic_redistribute_impl.h:26-106).  du, w and mass
// hold n-hydro variables with variable stride sv and layer stride 1; delta is
// [nlayer][N]; vol has layer stride vstride (0 = uniform); ny species follow
// IPR at ICY.
inline void vic_reduce_redistribute(double* du, const double* w, double* mass,
                                    const double* delta, const double* vol, int vstride,
                                    int nlayer, int64_t sv, int ny, int N) {
  double sum_a2 = 0, b_dry = 0;
  for (int i = 0; i < nlayer; ++i) {
    double V = vol[i * vstride];
    double et = du[IDN * sv + i];
    double dry = 1;
    for (int n = 0; n < ny; ++n) {
      et += du[(ICY + n) * sv + i];
      dry -= w[(ICY + n) * sv + i];
    }
    double ai = w[IDN * sv + i] * V;
    sum_a2 += ai * ai;
    b_dry += (et - delta[(size_t)i * N]) * dry * V;
  }
  for (int i = 0; i < nlayer; ++i) {
    double V = vol[i * vstride];
    double ai = w[IDN * sv + i] * V;
    double dry = 1;
    for (int n = 0; n < ny; ++n) dry -= w[(ICY + n) * sv + i];
    double et = du[IDN * sv + i];
    for (int n = 0; n < ny; ++n) et += du[(ICY + n) * sv + i];
    const double* d = delta + (size_t)i * N;
    double fix = d[0] - et;
    if (mass) mass[IDN * sv + i] = fix;
    double structural = w[IDN * sv + i] * ai * b_dry / sum_a2;
    du[IDN * sv + i] = du[IDN * sv + i] + fix * dry + structural;
    if (N == 3) {
      du[IVX * sv + i] = d[1];
      du[IPR * sv + i] = d[2];
    } else {
      for (int v = 1; v < 5; ++v) du[v * sv + i] = d[v];
    }
    for (int n = 0; n < ny; ++n)
      du[(ICY + n) * sv + i] = du[(ICY + n) * sv + i] + fix * w[(ICY + n) * sv + i];
  }
}

// One column.  du/w point at (var 0, interior cell il) of the column with
// variable stride sv and x1 stride 1; w[-1] and w[nlayer] are the ghost cells.
template <int N>
inline void vic_column(double* du, const double* w, double* mass, int nlayer, int64_t sv,
                       double area_lo, double area_hi_unused, double vol, double dt,
                       double grav, double gamma) {
  (void)area_hi_unused;
  std::vector<Mat<N>> a(nlayer), b(nlayer), c(nlayer);
  std::vector<std::array<double, N>> delta(nlayer);
  Mat<N> Phi{};
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) Phi.m[i][j] = 0.;
  if (N == 3) {
    Phi.m[1][0] = grav;
    Phi.m[2][1] = grav;
  } else {
    Phi.m[IVX][IDN] = grav;
    Phi.m[IPR][IVX] = grav;
  }
  double bnd[N];
  for (int i = 0; i < N; ++i) bnd[i] = 1.;
  bnd[1] = -1;  // normal momentum (IVX) is row 1 in both forms
  auto prim_at = [&](int i, double* p) {
    for (int v = 0; v < 5; ++v) p[v] = w[v * sv + i];
  };
  double gm1c = gamma - 1.;
  double gm1f = 0.5 * (gamma + gamma) - 1.;
  // --- assemble (vic_assemble_partial_impl / vic_assemble_full_impl) ---
  for (int i = 0; i < nlayer; ++i) {
    double wm[5], wc[5], wp[5];
    prim_at(i - 1, wm);
    prim_at(i, wc);
    prim_at(i + 1, wp);
    Mat<5> Jp5, Jc5, Jn5, Am5, Ap5;
    flux_jacobian(Jp5, gm1c, wm);
    flux_jacobian(Jc5, gm1c, wc);
    flux_jacobian(Jn5, gm1c, wp);
    roe_abs_jacobian(Am5, gm1f, wm, wc);
    roe_abs_jacobian(Ap5, gm1f, wc, wp);
    Mat<N> Jp, Jc, Jn, Am, Ap;
    sub_block<N>(Jp5, Jp);
    sub_block<N>(Jc5, Jc);
    sub_block<N>(Jn5, Jn);
    sub_block<N>(Am5, Am);
    sub_block<N>(Ap5, Ap);
    double ai = area_lo, aip = area_lo;  // uniform Cartesian face areas
    double hiv = 0.5 / vol;
    for (int r = 0; r < N; ++r)
      for (int q = 0; q < N; ++q) {
        a[i].m[r][q] = (Am.m[r][q] * ai + Ap.m[r][q] * aip + (aip - ai) * Jc.m[r][q]) * hiv -
                       Phi.m[r][q];
        b[i].m[r][q] = -(Am.m[r][q] + Jp.m[r][q]) * ai * hiv;
        c[i].m[r][q] = -(Ap.m[r][q] - Jn.m[r][q]) * aip * hiv;
      }
    for (int r = 0; r < N; ++r) a[i].m[r][r] += 1. / dt;
    if (i == 0)
      for (int r = 0; r < N; ++r)
        for (int q = 0; q < N; ++q) a[i].m[r][q] += b[i].m[r][q] * bnd[q];
    if (i == nlayer - 1)
      for (int r = 0; r < N; ++r)
        for (int q = 0; q < N; ++q) a[i].m[r][q] += c[i].m[r][q] * bnd[q];
  }
  // --- forward sweep (forward_sweep_impl.h:20-109) ---
  for (int i = 0; i < nlayer; ++i) {
    double rhs[N];
    if (N == 3) {
      rhs[0] = du[IDN * sv + i] / dt;
      rhs[1] = du[IVX * sv + i] / dt;
      rhs[2] = du[IPR * sv + i] / dt;
    } else {
      for (int v = 0; v < 5; ++v) rhs[v] = du[v * sv + i] / dt;
    }
    if (i > 0) {
      Mat<N> t;
      matmul<N>(b[i], a[i - 1], t);
      for (int r = 0; r < N; ++r)
        for (int q = 0; q < N; ++q) a[i].m[r][q] -= t.m[r][q];
      double bd[N];
      matvec<N>(b[i], delta[i - 1].data(), bd);
      for (int r = 0; r < N; ++r) rhs[r] = rhs[r] - bd[r];
    }
    if constexpr (N > 4) {
      Mat<N> A = a[i];
      int indx[N];
      for (int n = 0; n < N; ++n) indx[n] = n;
      lu_decompose<N>(A, indx);
      double sol[N][N + 1];
      for (int r = 0; r < N; ++r) {
        for (int q = 0; q < N; ++q) sol[r][q] = c[i].m[r][q];
        sol[r][N] = rhs[r];
      }
      lu_solve<N, N + 1>(A, indx, sol);
      for (int r = 0; r < N; ++r) {
        for (int q = 0; q < N; ++q) a[i].m[r][q] = sol[r][q];
        delta[i][r] = sol[r][N];
      }
    } else {
      Mat<3> inv;
      inv3(a[i], inv);
      matvec<3>(inv, rhs, delta[i].data());
      matmul<3>(inv, c[i], a[i]);
    }
  }
  // --- backward substitution + column sums (vic_redistribute_impl.h:26-62) ---
  for (int i = nlayer - 2; i >= 0; --i) {
    double t[N];
    matvec<N>(a[i], delta[i + 1].data(), t);
    for (int r = 0; r < N; ++r) delta[i][r] -= t[r];
  }
  std::vector<double> dflat((size_t)nlayer * N);
  for (int i = 0; i < nlayer; ++i)
    for (int r = 0; r < N; ++r) dflat[(size_t)i * N + r] = delta[i][r];
  vic_reduce_redistribute(du, w, mass, dflat.data(), &vol, 0, nlayer, sv, 0, N);
}

#ifdef ORC_REFERENCE_KERNELS
// One column through the reference's own implicit code, called the way
// vic_{assemble,solve,redistribute}_{partial,full}_cpu call it
// (src/implicit/implicit_dispatch.cpp:22-180): du/w/mass point at the
// column's first interior cell with variable stride sv and layer stride 1, so
// index -1 and nlayer reach the x1 ghost cells as the interior views do in
// ImplicitHydroImpl::forward (src/implicit/implicit_hydro.cpp:141-176).
template <int N>
inline void vic_column_reference(double* du, const double* w, double* mass, int nlayer,
                                 int64_t sv, double area, double vol, double dt, double grav,
                                 double gamma) {
  using Mat = Eigen::Matrix<double, N, N>;
  using Vec = Eigen::Matrix<double, N, 1>;
  std::vector<Mat> a(nlayer), b(nlayer), c(nlayer);
  std::vector<Vec> delta(nlayer);
  std::vector<double> gam(nlayer + 2, gamma), ar(nlayer + 1, area), vl(nlayer, vol);
  std::vector<double> mfix;
  if (!mass) {
    mfix.assign((size_t)(IDN + 1) * sv, 0.0);
    mass = mfix.data();
  }
  double* wp = const_cast<double*>(w);
  const int il = 0, iu = nlayer - 1, dir = 0, ny = 0, nvapor = 0;
  const int stride1 = (int)sv, stride2 = 1;
  if (N == 5) {
    snap::vic_assemble_full_impl<double>(du, wp, gam.data() + 1, ar.data(), vl.data(), dt, grav,
                                         il, iu, dir, ny, stride1, stride2, true, true, false,
                                         reinterpret_cast<Eigen::Matrix<double, 5, 5>*>(a.data()),
                                         reinterpret_cast<Eigen::Matrix<double, 5, 5>*>(b.data()),
                                         reinterpret_cast<Eigen::Matrix<double, 5, 5>*>(c.data()));
  } else {
    for (int i = 0; i < nlayer; ++i)
      snap::vic_assemble_partial_impl<double>(
          reinterpret_cast<Eigen::Matrix<double, 3, 3>*>(a.data()),
          reinterpret_cast<Eigen::Matrix<double, 3, 3>*>(b.data()),
          reinterpret_cast<Eigen::Matrix<double, 3, 3>*>(c.data()), wp, gam.data() + 1,
          ar.data(), vl.data(), i, il, iu, dt, grav, dir, ny, stride1, stride2, true, true);
  }
  snap::ForwardSweep<double, N>(a.data(), b.data(), c.data(), delta.data(), du, dt, il, iu, dir,
                                ny, stride1, stride2, true, true);
  snap::vic_backward_reduce<double, N>(du, wp, a.data(), delta.data(), vl.data(), c[0].data(),
                                       il, iu, dir, ny, stride1, stride2);
  for (int i = il; i <= iu; ++i)
    snap::vic_redistribute_cell<double, N>(du, wp, mass, delta.data(), vl.data(), c[0].data(), i,
                                           dir, ny, nvapor, stride1, stride2);
}
#endif

inline void implicit_correction(const Grid& g, double dt, double* du, const double* w,
                                double* mass) {
  int scheme = g.c.implicit_scheme;
  if (scheme == 0) return;
  int nlayer = g.c.nx1;
  int64_t sv = g.sv;
  int nj = g.ju - g.jl + 1, nk = g.ku - g.kl + 1;
  if (mass) std::fill(mass, mass + (int64_t)g.c.nvar * sv, 0.0);
  bool full = (scheme >> 3) & 1;
  par_for((int64_t)nj * nk, [&](int64_t col) {
    int j = g.jl + (int)(col % nj);
    int k = g.kl + (int)(col / nj);
    int64_t off = g.idx(k, j, g.il);
#ifdef ORC_REFERENCE_KERNELS
    if (full)
      vic_column_reference<5>(du + off, w + off, mass ? mass + off : nullptr, nlayer, sv,
                              g.area1(), g.vol(), dt, g.c.grav1, g.c.gammad);
    else
      vic_column_reference<3>(du + off, w + off, mass ? mass + off : nullptr, nlayer, sv,
                              g.area1(), g.vol(), dt, g.c.grav1, g.c.gammad);
#else
    if (full)
      vic_column<5>(du + off, w + off, mass ? mass + off : nullptr, nlayer, sv, g.area1(),
                    g.area1(), g.vol(), dt, g.c.grav1, g.c.gammad);
    else
      vic_column<3>(du + off, w + off, mass ? mass + off : nullptr, nlayer, sv, g.area1(),
                    g.area1(), g.vol(), dt, g.c.grav1, g.c.gammad);
#endif
  });
}

// ---------------------------------------------------------------------------
// Block state and the stage / forward drivers
// ---------------------------------------------------------------------------
struct Block {
  Grid g;
  std::vector<double> F1, F2, F3, P1, rho_grav, wlr, mass;
  std::vector<double> sF1, sF2, sF3, rlr;

  explicit Block(const snapb_hydro_config& c) : g(c) {
    int nv = c.nvar;
    int64_t sv = g.sv;
    if (g.nc1 > 1) F1.assign(nv * sv, 0.), P1.assign(sv, 0.);
    if (g.nc2 > 1) F2.assign(nv * sv, 0.);
    if (g.nc3 > 1) F3.assign(nv * sv, 0.);
    rho_grav.assign(sv, 0.);
    wlr.assign(2 * (int64_t)nv * sv, 0.);
    mass.assign(nv * sv, 0.);
    int ns = c.nscalar;
    if (ns > 0) {
      if (g.nc1 > 1) sF1.assign(ns * sv, 0.);
      if (g.nc2 > 1) sF2.assign(ns * sv, 0.);
      if (g.nc3 > 1) sF3.assign(ns * sv, 0.);
      rlr.assign(2 * (int64_t)ns * sv, 0.);
    }
  }

  // flux divergence over the interior: d = sum_dim (A F_{+} - A F_{-}), / vol
  void divergence(const std::vector<double>& f1, const std::vector<double>& f2,
                  const std::vector<double>& f3, int nv, double dt, double* du) {
    int64_t sv = g.sv;
    double A1 = g.area1(), A2 = g.area2(), A3 = g.area3(), V = g.vol();
    std::fill(du, du + (int64_t)nv * sv, 0.0);
    int ni = g.iu - g.il + 1, nj = g.ju - g.jl + 1, nk = g.ku - g.kl + 1;
    par_for((int64_t)ni * nj * nk, [&](int64_t t) {
      int i = g.il + (int)(t % ni);
      int j = g.jl + (int)((t / ni) % nj);
      int k = g.kl + (int)(t / ((int64_t)ni * nj));
      int64_t c0 = g.idx(k, j, i);
      for (int v = 0; v < nv; ++v) {
        int64_t c = v * sv + c0;
        double d = 0.;
        if (!f1.empty()) d += A1 * f1[c + g.s1] - A1 * f1[c];
        if (!f2.empty()) d += A2 * f2[c + g.s2] - A2 * f2[c];
        if (!f3.empty()) d += A3 * f3[c + g.s3] - A3 * f3[c];
        du[c] = -dt * (d / V);
      }
    });
  }

  // HydroImpl::forward (src/hydro/hydro_forward.cpp:14-217)
  void hydro_forward(double dt, const double* u, double* w, double* du, double* mass_out) {
    const auto& c = g.c;
    int nv = c.nvar;
    int64_t sv = g.sv;
    cons2prim(g, u, w);
    std::fill(rho_grav.begin(), rho_grav.end(), 0.0);
    bool grav1 = c.grav1 != 0.;
    if (g.nc1 > 1) {
      if (grav1) revise_x1_ghosts(g, w);
      reconstruct(g, 3, 0, w, nv, wlr.data());
      double* wl = wlr.data();
      double* wr = wlr.data() + (int64_t)nv * sv;
      if (grav1) {
        // _revise_x1inner_lr / _revise_x1outer_lr
        int64_t ncol = (int64_t)g.nc2 * g.nc3;
        for (int64_t col = 0; col < ncol; ++col) {
          int64_t o = col * g.nc1;
          wl[IPR * sv + o + g.il] = wr[IPR * sv + o + g.il];
          wl[IDN * sv + o + g.il] = wr[IDN * sv + o + g.il];
          wr[IPR * sv + o + g.iu + 1] = wl[IPR * sv + o + g.iu + 1];
          wr[IDN * sv + o + g.iu + 1] = wl[IDN * sv + o + g.iu + 1];
        }
        for (int64_t col = 0; col < ncol; ++col) {
          int64_t o = col * g.nc1;
          for (int i = g.il; i <= g.iu; ++i)
            rho_grav[o + i] = (wl[IPR * sv + o + i + 1] - wr[IPR * sv + o + i]) / g.dx1;
        }
      }
      if (!c.disable_flux[0]) riemann(g, c.riemann, 3, wl, wr, nv, F1.data(), P1.data(), nullptr);
    }
    if (g.nc2 > 1) {
      reconstruct(g, 2, 0, w, nv, wlr.data());
      if (!c.disable_flux[1])
        riemann(g, c.riemann, 2, wlr.data(), wlr.data() + (int64_t)nv * sv, nv, F2.data(),
                nullptr, nullptr);
    }
    if (g.nc3 > 1) {
      reconstruct(g, 1, 0, w, nv, wlr.data());
      if (!c.disable_flux[2])
        riemann(g, c.riemann, 1, wlr.data(), wlr.data() + (int64_t)nv * sv, nv, F3.data(),
                nullptr, nullptr);
    }
    divergence(F1, F2, F3, nv, dt, du);
    // const gravity (full array)
    double nh = c.non_hydrostatic;
    int64_t n = g.cells();
    for (int64_t t = 0; t < n; ++t) {
      double rho = w[IDN * sv + t];
      if (c.grav1 != 0.) {
        du[IVX * sv + t] += dt * rho * c.grav1 * nh;
        du[IPR * sv + t] += dt * rho * w[IVX * sv + t] * c.grav1 * nh;
      }
      if (c.grav2 != 0.) {
        du[IVY * sv + t] += dt * rho * c.grav2;
        du[IPR * sv + t] += dt * rho * w[IVY * sv + t] * c.grav2;
      }
      if (c.grav3 != 0.) {
        du[IVZ * sv + t] += dt * rho * c.grav3;
        du[IPR * sv + t] += dt * rho * w[IVZ * sv + t] * c.grav3;
      }
    }
    if (c.nu_iso > 0. || c.kappa_iso > 0.) diffusion(dt, w, du);
    if (has_gravity() && nh < 1.) {
      for (int64_t t = 0; t < n; ++t) {
        du[IVX * sv + t] += dt * rho_grav[t] * (1. - nh);
        du[IPR * sv + t] += dt * w[IVX * sv + t] * rho_grav[t] * (1. - nh);
      }
    }
    if (c.implicit_scheme != 0) {
      implicit_correction(g, dt, du, w, mass.data());
      if (mass_out) std::copy(mass.begin(), mass.end(), mass_out);
    }
  }

  bool has_gravity() const {
    return g.c.grav1 != 0. || g.c.grav2 != 0. || g.c.grav3 != 0. ||
           g.c.non_hydrostatic != 1.;
  }

  void diffusion(double dt, const double* w, double* du);

  // ScalarImpl::forward (src/scalar/scalar.cpp:50-132)
  void scalar_forward(double dt, const double* s, const double* u, double* ds,
                      std::vector<double>& r) {
    int ns = g.c.nscalar;
    int64_t sv = g.sv;
    for (int v = 0; v < ns; ++v)
      for (int64_t t = 0; t < sv; ++t) r[v * sv + t] = s[v * sv + t] / u[IDN * sv + t];
    if (g.nc1 > 1) {
      reconstruct(g, 3, 1, r.data(), ns, rlr.data());
      riemann(g, SNAPB_RIEMANN_UPWIND, 3, rlr.data(), rlr.data() + (int64_t)ns * sv, ns,
              sF1.data(), nullptr, F1.data());
    }
    if (g.nc2 > 1) {
      reconstruct(g, 2, 1, r.data(), ns, rlr.data());
      riemann(g, SNAPB_RIEMANN_UPWIND, 2, rlr.data(), rlr.data() + (int64_t)ns * sv, ns,
              sF2.data(), nullptr, F2.data());
    }
    if (g.nc3 > 1) {
      reconstruct(g, 1, 1, r.data(), ns, rlr.data());
      riemann(g, SNAPB_RIEMANN_UPWIND, 1, rlr.data(), rlr.data() + (int64_t)ns * sv, ns,
              sF3.data(), nullptr, F3.data());
    }
    divergence(sF1, sF2, sF3, ns, dt, ds);
  }

  // MeshBlockImpl::advance_local (src/mesh/meshblock.cpp:577-786) with the
  // Shu-Osher RK3 weights
  void stage(int st, double dt, double* u, double* u0, double* w, double* s, double* s0,
             double* r) {
    static const double wgt[3][3] = {{1., 0., 1.}, {3. / 4., 1. / 4., 1. / 4.},
                                     {1. / 3., 2. / 3., 2. / 3.}};
    int nv = g.c.nvar, ns = g.c.nscalar;
    int64_t sv = g.sv, nu = (int64_t)nv * sv, nsv = (int64_t)ns * sv;
    if (st == 0) {
      std::copy(u, u + nu, u0);
      if (ns > 0) std::copy(s, s + nsv, s0);
    }
    std::vector<double> du(nu), ds(nsv), rtmp(nsv);
    hydro_forward(dt, u, w, du.data(), nullptr);
    if (ns > 0) {
      scalar_forward(dt, s, u, ds.data(), rtmp);
      if (g.c.implicit_scheme != 0 && r)
        for (int v = 0; v < ns; ++v)
          for (int64_t t = 0; t < sv; ++t) ds[v * sv + t] += mass[IDN * sv + t] * r[v * sv + t];
    }
    const double* W = wgt[st];
    for (int64_t t = 0; t < nu; ++t) u[t] = W[0] * u0[t] + W[1] * u[t] + W[2] * du[t];
    if (ns > 0) {
      for (int64_t t = 0; t < nsv; ++t) s[t] = W[0] * s0[t] + W[1] * s[t] + W[2] * ds[t];
      if (r)
        for (int v = 0; v < ns; ++v)
          for (int64_t t = 0; t < sv; ++t) r[v * sv + t] = s[v * sv + t] / u[IDN * sv + t];
    }
    bc_apply(g, u, nv, SNAPB_CONSERVED);
    if (ns > 0) bc_apply(g, s, ns, SNAPB_SCALAR);
  }
};

// ---------------------------------------------------------------------------
// CFL limit (src/hydro/hydro.cpp:118-180, src/forcing/diffusion.cpp:242-265)
// ---------------------------------------------------------------------------
inline double max_time_step(const Grid& g, const double* w) {
  const auto& c = g.c;
  int64_t sv = g.sv;
  double dtm[3] = {1.e9, 1.e9, 1.e9};
  int scheme = c.implicit_scheme;
  bool use1 = g.nc1 > 1, use2 = g.nc2 > 1, use3 = g.nc3 > 1;
  if (scheme != 0) {
    use1 = use1 && (!(scheme & 1) || (g.nc3 == 1 && g.nc2 == 1));
    use2 = use2 && !((scheme >> 1) & 1);
    use3 = use3 && !((scheme >> 2) & 1);
  }
  double m1 = std::numeric_limits<double>::infinity(), m2 = m1, m3 = m1;
  for (int k = g.kl; k <= g.ku; ++k)
    for (int j = g.jl; j <= g.ju; ++j)
      for (int i = g.il; i <= g.iu; ++i) {
        int64_t t = g.idx(k, j, i);
        double cs = std::sqrt(c.gammad * w[IPR * sv + t] / w[IDN * sv + t]);
        if (use1) m1 = std::min(m1, g.dx1 / (std::fabs(w[IVX * sv + t]) + cs));
        if (use2) m2 = std::min(m2, g.dx2 / (std::fabs(w[IVY * sv + t]) + cs));
        if (use3) m3 = std::min(m3, g.dx3 / (std::fabs(w[IVZ * sv + t]) + cs));
      }
  if (use1) dtm[0] = m1;
  if (use2) dtm[1] = m2;
  if (use3) dtm[2] = m3;
  double dt = std::min(dtm[0], std::min(dtm[1], dtm[2]));
  double coeff = std::max(c.nu_iso, c.kappa_iso);
  if (coeff > 0.) {
    int ndim = 0;
    double dxmin = std::numeric_limits<double>::max();
    if (g.nc1 > 1) ++ndim, dxmin = std::min(dxmin, g.dx1);
    if (g.nc2 > 1) ++ndim, dxmin = std::min(dxmin, g.dx2);
    if (g.nc3 > 1) ++ndim, dxmin = std::min(dxmin, g.dx3);
    if (ndim > 0) dt = std::min(dt, dxmin * dxmin / (2. * ndim * coeff));
  }
  return dt;
}

}  // namespace orc

#include "oracle_diffusion.hpp"
