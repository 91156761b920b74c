// common.cuh — shared device code of the B200 hydro step: geometry, the
// reconstruction and Riemann point kernels, error plumbing.
//
// Layout: [nvar, nc3, nc2, nc1], x1 contiguous (reference src/hydro/hydro.cpp:87-115).
// Variable order IDN, IVX, IVY, IVZ, IPR (src/snap.h:34-46).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/snapb.h"

namespace snapb {

enum { IDN = 0, IVX = 1, IVY = 2, IVZ = 3, IPR = 4, ICY = 5 };

constexpr int kMaxScalar = 3;  // passive scalars carried through the fused sweeps

// Geometry of one block, by value in kernel parameters.
struct Geo {
  int nx1, nx2, nx3, ng;
  int nc1, nc2, nc3;
  int64_t s2, s3, sv;  // strides of x2, x3, variable (x1 stride is 1)
  int il, iu, jl, ju, kl, ku;
  double dx1, dx2, dx3;
  double A1, A2, A3, vol;  // uniform Cartesian face areas and cell volume
};

inline Geo make_geo(const snapb_hydro_config& c) {
  Geo g;
  g.nx1 = c.nx1;
  g.nx2 = c.nx2;
  g.nx3 = c.nx3;
  g.ng = c.nghost;
  g.nc1 = c.nx1 > 1 ? c.nx1 + 2 * c.nghost : 1;
  g.nc2 = c.nx2 > 1 ? c.nx2 + 2 * c.nghost : 1;
  g.nc3 = c.nx3 > 1 ? c.nx3 + 2 * c.nghost : 1;
  g.s2 = g.nc1;
  g.s3 = (int64_t)g.nc1 * g.nc2;
  g.sv = g.s3 * g.nc3;
  g.il = c.nx1 > 1 ? c.nghost : 0;
  g.iu = c.nx1 > 1 ? c.nghost + c.nx1 - 1 : 0;
  g.jl = c.nx2 > 1 ? c.nghost : 0;
  g.ju = c.nx2 > 1 ? c.nghost + c.nx2 - 1 : 0;
  g.kl = c.nx3 > 1 ? c.nghost : 0;
  g.ku = c.nx3 > 1 ? c.nghost + c.nx3 - 1 : 0;
  g.dx1 = (c.x1max - c.x1min) / c.nx1;
  g.dx2 = (c.x2max - c.x2min) / c.nx2;
  g.dx3 = (c.x3max - c.x3min) / c.nx3;
  // face_area1 = dx3 (x) dx2, face_area2 = dx3 (x) dx1, face_area3 = dx2 (x) dx1,
  // volume = dx3 * (dx2 * dx1)  (src/coord/coordinate.cpp:316-331)
  g.A1 = g.dx3 * g.dx2;
  g.A2 = g.dx3 * g.dx1;
  g.A3 = g.dx2 * g.dx1;
  g.vol = g.dx3 * (g.dx2 * g.dx1);
  return g;
}

// Physics parameters, by value in kernel parameters.
struct Phys {
  double gammad, rgas;
  double grav1, grav2, grav3, nh;
  double nu, kappa;
  int riemann;
  int r1_type, r1_shock, r1_scale;
  int r23_type, r23_shock, r23_scale;
  int rs_type, rs_scale;
  int nvar, nscalar;
  int implicit_scheme;
  int disable1, disable2, disable3;
  bool has_grav;  // a const-gravity section exists (any g != 0 or nh != 1)
};

inline Phys make_phys(const snapb_hydro_config& c) {
  Phys p;
  p.gammad = c.gammad;
  p.rgas = c.rgas;
  p.grav1 = c.grav1;
  p.grav2 = c.grav2;
  p.grav3 = c.grav3;
  p.nh = c.non_hydrostatic;
  p.nu = c.nu_iso;
  p.kappa = c.kappa_iso;
  p.riemann = c.riemann;
  p.r1_type = c.recon1_type;
  p.r1_shock = c.recon1_shock;
  p.r1_scale = c.recon1_scale;
  p.r23_type = c.recon23_type;
  p.r23_shock = c.recon23_shock;
  p.r23_scale = c.recon23_scale;
  p.rs_type = c.scalar_recon_type;
  p.rs_scale = c.scalar_recon_scale;
  p.nvar = c.nvar;
  p.nscalar = c.nscalar;
  p.implicit_scheme = c.implicit_scheme;
  p.disable1 = c.disable_flux[0];
  p.disable2 = c.disable_flux[1];
  p.disable3 = c.disable_flux[2];
  p.has_grav = c.grav1 != 0. || c.grav2 != 0. || c.grav3 != 0. || c.non_hydrostatic != 1.;
  return p;
}

// Index arithmetic.  Every element, cell, column, line and slot index of a
// block is below 2^31 (check_config rejects larger blocks), so quotients and
// remainders by run-time divisors are taken in 32 bits: a 64-bit division is
// a long instruction sequence, and the sweeps take several per face.
__host__ __device__ __forceinline__ int udiv(int64_t a, int64_t b) {
  return (int)((uint32_t)a / (uint32_t)b);
}
__host__ __device__ __forceinline__ int umod(int64_t a, int64_t b) {
  return (int)((uint32_t)a % (uint32_t)b);
}

// The ghost shell of a block, one slot per ghost cell:
// slots [0, A) are the x1 ghosts of rows inside the x2/x3 interior
// (2 ng per row), slots [A, A + B) the cells of the ghost rows (x3-ghost slabs
// first, then the x2-ghost strips of interior x3 planes)
__host__ __device__ __forceinline__ int64_t bc_shell_slots(const Geo& g) {
  const int64_t nj = g.ju - g.jl + 1, nk = g.ku - g.kl + 1;
  const int64_t A = g.nc1 > 1 ? nj * nk * 2 * g.ng : 0;
  const int64_t c1 = g.nc3 > 1 ? (int64_t)2 * g.ng * g.nc2 : 0;
  const int64_t c2 = g.nc2 > 1 ? nk * 2 * g.ng : 0;
  return A + (c1 + c2) * g.nc1;
}

// flat index of ghost slot s, with its (i, j, k)
__host__ __device__ __forceinline__ int64_t bc_shell_cell(const Geo& g, int64_t s, int& i, int& j,
                                                          int& k) {
  const int64_t nj = g.ju - g.jl + 1, nk = g.ku - g.kl + 1;
  const int ng2 = 2 * g.ng;
  const int64_t A = g.nc1 > 1 ? nj * nk * ng2 : 0;
  if (s < A) {
    const int c = umod(s, ng2);
    const int row = udiv(s, ng2);
    i = c < g.ng ? c : g.nc1 - ng2 + c;
    j = g.jl + umod(row, nj);
    k = g.kl + udiv(row, nj);
  } else {
    s -= A;
    i = umod(s, g.nc1);
    int row = udiv(s, g.nc1);
    const int c1 = g.nc3 > 1 ? ng2 * g.nc2 : 0;
    if (row < c1) {
      j = umod(row, g.nc2);
      const int kk = udiv(row, g.nc2);
      k = kk < g.ng ? kk : g.nc3 - ng2 + kk;
    } else {
      row -= c1;
      const int jj = umod(row, ng2);
      j = jj < g.ng ? jj : g.nc2 - ng2 + jj;
      k = g.kl + udiv(row, ng2);
    }
  }
  return ((int64_t)k * g.nc2 + j) * g.nc1 + i;
}

inline int64_t bc_shell_slots_host(const Geo& g) { return bc_shell_slots(g); }

template <class T>
__host__ __device__ __forceinline__ T sqr(T x) {
  return x * x;
}

// Quotient of the face and block formulas: the correctly rounded division for
// FP64 (and the adjoint's dual numbers); for the FP32 perturbation form the
// fast single-precision division (__fdividef: within 2 ulp for divisors of
// magnitude below 2^126), since its FP32 face states and blocks are FP32
// approximations in any case and the correctly rounded quotient costs several
// times the instructions.
template <class T>
__device__ __forceinline__ T fdiv(T a, T b) {
  return a / b;
}
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }

// ---------------------------------------------------------------------------
// Reconstruction point kernels.  A face f (between cells f-1 and f) sees the
// six cells q[0..5] = w[f-3 .. f+2].  The left state wl is the value at the
// right face of cell f-1 (= q[2]); the right state wr is the value at the left
// face of cell f (= q[3]).  Formulas: src/recon/interp_impl.h:22-122,
// src/recon/plm.cpp:13-36, coefficient tables src/recon/{weno5,cp5,weno3,cp3}.cpp.
// ---------------------------------------------------------------------------

// WENO5-JS value at the face on the a-side of the window centre c:
// window (a, b, c, d, e) ordered away from that face.  Weights 0.3/0.6/0.1,
// epsilon 1e-6, optional mean-|phi| scaling.
template <class T>
__device__ __forceinline__ T weno5_face(T a, T b, T c, T d, T e, bool scale) {
  T vs = T(1);
  if (scale) {
    vs = fdiv(fabs(a) + fabs(b) + fabs(c) + fabs(d) + fabs(e), T(5));
    if (vs == T(0)) return T(0);
    T iv = fdiv(T(1), vs);
    a *= iv;
    b *= iv;
    c *= iv;
    d *= iv;
    e *= iv;
  }
  const T c16 = T(1. / 6.), c56 = T(5. / 6.), c13 = T(1. / 3.);
  const T c116 = T(11. / 6.), c76 = T(7. / 6.), c1312 = T(13. / 12.);
  T p0 = -c16 * a + c56 * b + c13 * c;
  T p1 = c13 * b + c56 * c - c16 * d;
  T p2 = c116 * c - c76 * d + c13 * e;
  T b0 = c1312 * sqr(a - T(2) * b + c) + T(0.25) * sqr(a - T(4) * b + T(3) * c);
  T b1 = c1312 * sqr(b - T(2) * c + d) + T(0.25) * sqr(d - b);
  T b2 = c1312 * sqr(c - T(2) * d + e) + T(0.25) * sqr(T(3) * c - T(4) * d + e);
  T s0 = sqr(b0 + T(1e-6)), s1 = sqr(b1 + T(1e-6)), s2 = sqr(b2 + T(1e-6));
  T out;
  if constexpr (sizeof(T) == 8) {
    // one division: alpha_k = d_k / s_k
    T s12 = s1 * s2, s02 = s0 * s2, s01 = s0 * s1;
    T n0 = T(0.3) * s12, n1 = T(0.6) * s02, n2 = T(0.1) * s01;
    out = (n0 * p0 + n1 * p1 + n2 * p2) / (n0 + n1 + n2);
  } else {
    T a0 = fdiv(T(0.3), s0), a1 = fdiv(T(0.6), s1), a2 = fdiv(T(0.1), s2);
    out = fdiv(a0 * p0 + a1 * p1 + a2 * p2, a0 + a1 + a2);
  }
  return vs * out;
}

// WENO3 value at the face between a and b, window (a, b, c) ordered away
// from that face (src/recon/interp_impl.h:34-70).
template <class T>
__device__ __forceinline__ T weno3_face(T a, T b, T c, bool scale) {
  T vs = T(1);
  if (scale) {
    vs = fdiv(fabs(a) + fabs(b) + fabs(c), T(3));
    if (vs == T(0)) return T(0);
    a = fdiv(a, vs);
    b = fdiv(b, vs);
    c = fdiv(c, vs);
  }
  T p0 = T(0.5) * a + T(0.5) * b;
  T p1 = T(1.5) * b - T(0.5) * c;
  T b0 = sqr(a - b);
  T b1 = sqr(b - c);
  T a0 = fdiv(T(2.0 / 3.0), sqr(b0 + T(1e-6)));
  T a1 = fdiv(T(1.0 / 3.0), sqr(b1 + T(1e-6)));
  return fdiv(a0 * p0 + a1 * p1, a0 + a1) * vs;
}

// face states from a six-cell window for one variable
template <class T>
__device__ __forceinline__ void face_states(int type, bool scale, const T* q, T& wl, T& wr) {
  switch (type) {
    case SNAPB_RECON_WENO5:
      wl = weno5_face(q[4], q[3], q[2], q[1], q[0], scale);  // right face of q[2]
      wr = weno5_face(q[1], q[2], q[3], q[4], q[5], scale);  // left face of q[3]
      break;
    case SNAPB_RECON_CP5: {
      const T a = T(-1. / 20.), b = T(9. / 20.), c = T(47. / 60.), d = T(-13. / 60.),
              e = T(1. / 30.);
      wl = a * q[4] + b * q[3] + c * q[2] + d * q[1] + e * q[0];
      wr = a * q[1] + b * q[2] + c * q[3] + d * q[4] + e * q[5];
      break;
    }
    case SNAPB_RECON_WENO3:
      wl = weno3_face(q[3], q[2], q[1], scale);
      wr = weno3_face(q[2], q[3], q[4], scale);
      break;
    case SNAPB_RECON_CP3: {
      const T a = T(1. / 3.), b = T(5. / 6.), c = T(-1. / 6.);
      wl = a * q[3] + b * q[2] + c * q[1];
      wr = a * q[2] + b * q[3] + c * q[4];
      break;
    }
    case SNAPB_RECON_PLM: {
      // harmonic-mean slope with FLT_MIN guard, zeroed across extrema
      const T tiny = T(1.1754943508222875e-38);
      T dl = q[2] - q[1], dr = q[3] - q[2];
      T d2 = dl * dr;
      T m = fdiv(T(2) * d2, dl + dr + tiny);
      m = d2 >= T(0) ? m : T(0);
      wl = q[2] + T(0.5) * m;
      dl = q[3] - q[2];
      dr = q[4] - q[3];
      d2 = dl * dr;
      m = fdiv(T(2) * d2, dl + dr + tiny);
      m = d2 >= T(0) ? m : T(0);
      wr = q[3] - T(0.5) * m;
      break;
    }
    default:  // donor cell
      wl = q[2];
      wr = q[3];
  }
}

// interp1 / interp2 of a Reconstruct module: weno5 -> cp5, weno3 -> cp3
__host__ __device__ __forceinline__ int interp2_of(int t) {
  return t == SNAPB_RECON_WENO5 ? SNAPB_RECON_CP5 : (t == SNAPB_RECON_WENO3 ? SNAPB_RECON_CP3 : t);
}

// ---------------------------------------------------------------------------
// Riemann solvers on primitive states in registers.  ivx is the normal
// velocity slot (1, 2, 3 for x1, x2, x3).  Formulas:
// src/riemann/hllc_impl.h:16-130, lmars_impl.h:16-78, roe_impl.h:23-211.
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ void hllc_flux(const T* L, const T* R, int ivx, T gamma, T* F,
                                          T* fp = nullptr) {
  const T TINY = T(1.0e-10);
  int ivy = IVX + (ivx - IVX + 1) % 3;
  int ivz = IVX + (ivx - IVX + 2) % 3;
  T igm1 = T(1) / (gamma - T(1));
  T cl = sqrt(gamma * L[IPR] / L[IDN]);
  T cr = sqrt(gamma * R[IPR] / R[IDN]);
  T el = L[IPR] * igm1 + T(0.5) * L[IDN] * (sqr(L[IVX]) + sqr(L[IVY]) + sqr(L[IVZ]));
  T er = R[IPR] * igm1 + T(0.5) * R[IDN] * (sqr(R[IVX]) + sqr(R[IVY]) + sqr(R[IVZ]));
  T rhoa = T(0.5) * (L[IDN] + R[IDN]);
  T ca = T(0.5) * (cl + cr);
  T pmid = T(0.5) * (L[IPR] + R[IPR] + (L[ivx] - R[ivx]) * rhoa * ca);
  T gf = (gamma + T(1)) / (T(2) * gamma);
  T ql = pmid <= L[IPR] ? T(1) : sqrt(T(1) + gf * (pmid / L[IPR] - T(1)));
  T qr = pmid <= R[IPR] ? T(1) : sqrt(T(1) + gf * (pmid / R[IPR] - T(1)));
  T al = L[ivx] - cl * ql;
  T ar = R[ivx] + cr * qr;
  T bp = ar > T(0) ? ar : TINY;
  T bm = al < T(0) ? al : -TINY;
  T vxl = L[ivx] - al;
  T vxr = R[ivx] - ar;
  T tl = L[IPR] + vxl * L[IDN] * L[ivx];
  T tr = R[IPR] + vxr * R[IDN] * R[ivx];
  T ml = L[IDN] * vxl;
  T mr = -(R[IDN] * vxr);
  T ims = T(1) / (ml + mr);
  T am = (tl - tr) * ims;
  T cp = (ml * tr + mr * tl) * ims;
  cp = cp > T(0) ? cp : T(0);
  if (fp) *fp = cp;
  vxl = L[ivx] - bm;
  vxr = R[ivx] - bp;
  T sl, sr, sm;
  if (am >= T(0)) {
    T id = T(1) / (am - bm);
    sl = am * id;
    sr = T(0);
    sm = -bm * id;
  } else {
    T id = T(1) / (bp - am);
    sl = T(0);
    sr = -am * id;
    sm = bp * id;
  }
  T fl, fr;
  fl = L[IDN] * vxl;
  fr = R[IDN] * vxr;
  F[IDN] = sl * fl + sr * fr;
  fl = L[IDN] * L[ivx] * vxl + L[IPR];
  fr = R[IDN] * R[ivx] * vxr + R[IPR];
  F[ivx] = sl * fl + sr * fr + sm * cp;
  fl = L[IDN] * L[ivy] * vxl;
  fr = R[IDN] * R[ivy] * vxr;
  F[ivy] = sl * fl + sr * fr;
  fl = L[IDN] * L[ivz] * vxl;
  fr = R[IDN] * R[ivz] * vxr;
  F[ivz] = sl * fl + sr * fr;
  fl = el * vxl + L[IPR] * L[ivx];
  fr = er * vxr + R[IPR] * R[ivx];
  F[IPR] = sl * fl + sr * fr + sm * cp * am;
}

template <class T>
__device__ __forceinline__ void lmars_flux(const T* L, const T* R, int ivx, T gamma, T* F,
                                           T* fp = nullptr) {
  int ivy = IVX + (ivx - IVX + 1) % 3;
  int ivz = IVX + (ivx - IVX + 2) % 3;
  T igm1 = T(1) / (gamma - T(1));
  T irl = T(1) / L[IDN], irr = T(1) / R[IDN];
  T ke_l = T(0.5) * (sqr(L[ivx]) + sqr(L[ivy]) + sqr(L[ivz]));
  T ke_r = T(0.5) * (sqr(R[ivx]) + sqr(R[ivy]) + sqr(R[ivz]));
  T hl = L[IPR] * igm1 * irl + ke_l + L[IPR] * irl;
  T hr = R[IPR] * igm1 * irr + ke_r + R[IPR] * irr;
  T rhobar = T(0.5) * (L[IDN] + R[IDN]);
  T cbar = sqrt(T(0.5) * gamma * (L[IPR] + R[IPR]) / rhobar);
  T pbar = T(0.5) * (L[IPR] + R[IPR]) + T(0.5) * (rhobar * cbar) * (L[ivx] - R[ivx]);
  if (fp) *fp = pbar;
  T ubar = T(0.5) * (L[ivx] + R[ivx]) + T(0.5) / (rhobar * cbar) * (L[IPR] - R[IPR]);
  const T* S = ubar > T(0) ? L : R;
  T h = ubar > T(0) ? hl : hr;
  T m = ubar * S[IDN];
  F[IDN] = m;
  F[ivx] = m * S[ivx] + pbar;
  F[ivy] = m * S[ivy];
  F[ivz] = m * S[ivz];
  F[IPR] = m * h;
}

template <class T>
__device__ __forceinline__ void roe_flux(const T* L, const T* R, int ivx, T gamma, T* F,
                                         T* fp = nullptr) {
  const T TINY = T(1.0e-10);
  int ivy = IVX + (ivx - IVX + 1) % 3;
  int ivz = IVX + (ivx - IVX + 2) % 3;
  T igm1 = T(1) / (gamma - T(1));
  T etl = L[IPR] * igm1 + T(0.5) * L[IDN] * (sqr(L[IVX]) + sqr(L[IVY]) + sqr(L[IVZ]));
  T etr = R[IPR] * igm1 + T(0.5) * R[IDN] * (sqr(R[IVX]) + sqr(R[IVY]) + sqr(R[IVZ]));
  T sdl = sqrt(L[IDN]), sdr = sqrt(R[IDN]);
  T isd = T(1) / (sdl + sdr);
  T rhobar = sdl * sdr;
  T v1 = (sdl * L[ivx] + sdr * R[ivx]) * isd;
  T v2 = (sdl * L[ivy] + sdr * R[ivy]) * isd;
  T v3 = (sdl * L[ivz] + sdr * R[ivz]) * isd;
  T hl = (etl + L[IPR]) / L[IDN];
  T hr = (etr + R[IPR]) / R[IDN];
  T h = (hl * sdl + hr * sdr) * isd;
  T rhol0 = L[IDN], rhor0 = R[IDN];
  T fl0 = rhol0 * L[ivx], fr0 = rhor0 * R[ivx];
  T fl1 = L[IDN] * L[ivx] * L[ivx] + L[IPR], fr1 = R[IDN] * R[ivx] * R[ivx] + R[IPR];
  T fl2 = L[IDN] * L[ivx] * L[ivy], fr2 = R[IDN] * R[ivx] * R[ivy];
  T fl3 = L[IDN] * L[ivx] * L[ivz], fr3 = R[IDN] * R[ivx] * R[ivz];
  T fl4 = (etl + L[IPR]) * L[ivx], fr4 = (etr + R[IPR]) * R[ivx];
  T qbar = (rhol0 / sdl + rhor0 / sdr) * isd;
  T vsq = v1 * v1 + v2 * v2 + v3 * v3;
  T gm1 = gamma - T(1);
  T q = h - T(0.5) * vsq;
  T qq = q > TINY ? q : TINY;
  T cs_sq = gm1 * qq;
  cs_sq = cs_sq > TINY ? cs_sq : TINY;
  T cs = sqrt(cs_sq);
  if (fp) *fp = T(0.5) * (L[IPR] + R[IPR] + rhobar * cs * (L[ivx] - R[ivx]));
  T lam_m = v1 - cs, lam_0 = v1, lam_p = v1 + cs;
  T spd_m = fabs(lam_m), spd_0 = fabs(lam_0), spd_p = fabs(lam_p);
  T du = R[ivx] - L[ivx], dv = R[ivy] - L[ivy], dw = R[ivz] - L[ivz];
  T dp = R[IPR] - L[IPR];
  T ics = T(1) / cs, ics2 = T(1) / cs_sq;
  T alpha_m = -T(0.5) * rhobar * ics * du + T(0.5) * dp * ics2;
  T alpha_p = T(0.5) * rhobar * ics * du + T(0.5) * dp * ics2;
  T alpha_v = rhobar * dv, alpha_w = rhobar * dw;
  T ac0 = rhor0 - rhol0 - dp * ics2 * qbar;
  T rho1 = rhol0 + alpha_m * qbar;
  T rho2 = rho1 + ac0;
  bool llf = (rho1 < T(0)) || (rho2 < T(0));
  T alpha0 = ac0;
  if (llf) {
    T cl = sqrt(gamma * L[IPR] / L[IDN]);
    T cr = sqrt(gamma * R[IPR] / R[IDN]);
    T al = fabs(L[ivx]) + cl, ar = fabs(R[ivx]) + cr;
    T a = T(0.5) * (al > ar ? al : ar);
    F[IDN] = T(0.5) * (fl0 + fr0) - a * (rhor0 - rhol0);
    F[ivx] = T(0.5) * (fl1 + fr1) - a * (R[IDN] * R[ivx] - L[IDN] * L[ivx]);
    F[ivy] = T(0.5) * (fl2 + fr2) - a * (R[IDN] * R[ivy] - L[IDN] * L[ivy]);
    F[ivz] = T(0.5) * (fl3 + fr3) - a * (R[IDN] * R[ivz] - L[IDN] * L[ivz]);
    F[IPR] = T(0.5) * (fl4 + fr4) - a * (etr - etl);
    return;
  }
  if (lam_m > T(0)) {
    F[IDN] = fl0;
    F[ivx] = fl1;
    F[ivy] = fl2;
    F[ivz] = fl3;
    F[IPR] = fl4;
    return;
  }
  if (lam_p < T(0)) {
    F[IDN] = fr0;
    F[ivx] = fr1;
    F[ivy] = fr2;
    F[ivz] = fr3;
    F[IPR] = fr4;
    return;
  }
  F[IDN] = T(0.5) * (fl0 + fr0) -
           T(0.5) * (spd_m * alpha_m * qbar + spd_0 * ac0 + spd_p * alpha_p * qbar);
  F[ivx] = T(0.5) * (fl1 + fr1) - T(0.5) * (spd_m * alpha_m * (v1 - cs) + spd_0 * (v1 * alpha0) +
                                            spd_p * alpha_p * (v1 + cs));
  F[ivy] = T(0.5) * (fl2 + fr2) - T(0.5) * (spd_m * alpha_m * v2 +
                                            spd_0 * (v2 * alpha0 + alpha_v) +
                                            spd_p * alpha_p * v2);
  F[ivz] = T(0.5) * (fl3 + fr3) - T(0.5) * (spd_m * alpha_m * v3 +
                                            spd_0 * (v3 * alpha0 + alpha_w) +
                                            spd_p * alpha_p * v3);
  F[IPR] = T(0.5) * (fl4 + fr4) -
           T(0.5) * (spd_m * alpha_m * (h - v1 * cs) +
                     spd_0 * (rhobar * (hr - hl - v1 * du) + alpha0 * h - dp) +
                     spd_p * alpha_p * (h + v1 * cs));
}

template <class T>
__device__ __forceinline__ void riemann_flux(int solver, const T* L, const T* R, int ivx, T gamma,
                                             T* F, T* fp = nullptr) {
  if (solver == SNAPB_RIEMANN_HLLC)
    hllc_flux(L, R, ivx, gamma, F, fp);
  else if (solver == SNAPB_RIEMANN_LMARS)
    lmars_flux(L, R, ivx, gamma, F, fp);
  else
    roe_flux(L, R, ivx, gamma, F, fp);
}

// ideal-gas cons2prim of one cell (src/eos/ideal_gas_impl.h:15-35)
template <class T>
__device__ __forceinline__ void cons2prim_cell(const T* u, T* w, T gm1) {
  T rho = u[IDN];
  T ir = T(1) / rho;
  w[IDN] = rho;
  w[IVX] = u[IVX] * ir;
  w[IVY] = u[IVY] * ir;
  w[IVZ] = u[IVZ] * ir;
  T ke = T(0.5) * (w[IVX] * u[IVX] + w[IVY] * u[IVY] + w[IVZ] * u[IVZ]);
  w[IPR] = gm1 * (u[IPR] - ke);
}

}  // namespace snapb
