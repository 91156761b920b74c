// adjoint.cu — hand-written reverse (adjoint) kernels of one FP64 RK stage.
//
// Given the cotangent of a stage's output state, produce the cotangents of
// its inputs: the stage-start state (full array, ghosts included) and the
// step-start state of the RK combination.  The stage is the composition
//
//   w = U->W(u) (+ isentropic x1 ghost revision), r = s / rho
//   du_e = -dt div F(recon(w)) + gravity          (explicit tendency)
//   du   = VIC(du_e; w)                           (vertically implicit solve)
//   u'   = BC(wgt0 u0 + wgt1 u + wgt2 du)         (RK combination, boundaries)
//
// and the kernels run its pieces backwards:
//   k_adj_combine   BC^T (a gather over each interior cell's ghost images)
//                   and the RK weights;
//   VIC adjoint     k_vadj_assemble / k_vadj_sweep / k_vadj_contract: the
//                   forward elimination is repeated, the transposed
//                   block-tridiagonal system T^T t = g_delta is solved with the
//                   same factors, and the dependence of the blocks on w is
//                   contracted exactly: with y = t_{k-1} - t_k and
//                   x = delta_k - delta_{k-1}, interface k contributes
//                   A hiv * d(y^T |A|(w_{k-1}, w_k) x) and cell m contributes
//                   A hiv * d((t_{m+1} - t_{m-1})^T J(w_m) delta_m);
//   k_march_adj     x2 / x3 faces: Riemann + reconstruction VJPs, a six-cell
//                   register window of cotangent accumulators per thread;
//   k_x1_adj        x1 faces of a column in shared memory, gravity, the
//                   ghost-revision VJP and the U->W VJP into g_u, g_s.
//
// Local derivatives: the Riemann solvers and WENO5 have hand-written reverses
// (riemann_adj.cuh, weno5_face_vjp); |A|, J, the other reconstructions and the
// ghost revision are differentiated with forward-mode dual numbers (dual.cuh)
// through the very templates the forward kernels use.  Every switch (HLLC wave
// selection, Roe entropy / LLF branches, LMARS upwinding, the pressure clamp)
// is taken on the branch the forward pass took.  dt is a
// constant of the adjoint (the CFL choice is not differentiated).
//
// Reference forward path: HydroImpl::forward (src/hydro/hydro_forward.cpp:14-217),
// ImplicitHydroImpl::forward (src/implicit/implicit_hydro.cpp:99-189),
// MeshBlockImpl::forward (src/mesh/meshblock.cpp:577-786), bc_func (src/bc/bc_func.cpp:7-63).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>

#include "dual.cuh"
#include "kernels.cuh"
#include "ring.cuh"
#include "riemann_adj.cuh"
#include "bilinear_adj.cuh"
#include "block_cr.cuh"
#include "vic_blocks.cuh"

namespace snapb {

constexpr int kMaxGhost = 8;

// ---------------------------------------------------------------------------
// Boundary transpose: interior cell x of an axis and the ghost cells whose
// fill copies it (reflecting / periodic / outflow), with their sign flips.
// Mirrors the composite map of k_bc in aux.cu.
// ---------------------------------------------------------------------------
struct AxisAdj {
  int n, ng, lo_type, hi_type;
};

__device__ __forceinline__ int axis_src(const AxisAdj& a, int i, bool& flip) {
  flip = false;
  if (a.n == 1) return i;
  if (i < a.ng) {
    switch (a.lo_type) {
      case SNAPB_BC_REFLECTING: flip = true; return 2 * a.ng - 1 - i;
      case SNAPB_BC_PERIODIC: return a.n - 2 * a.ng + i;
      case SNAPB_BC_OUTFLOW: return a.ng;
      default: return i;
    }
  }
  if (i >= a.n - a.ng) {
    switch (a.hi_type) {
      case SNAPB_BC_REFLECTING: flip = true; return 2 * (a.n - a.ng) - 1 - i;
      case SNAPB_BC_PERIODIC: return i - a.n + 2 * a.ng;
      case SNAPB_BC_OUTFLOW: return a.n - a.ng - 1;
      default: return i;
    }
  }
  return i;
}

// images of interior index x: itself plus the ghosts mapped onto it
__device__ __forceinline__ int axis_images(const AxisAdj& a, int x, int* ys, bool* fl) {
  int n = 0;
  ys[n] = x;
  fl[n++] = false;
  if (a.n == 1) return n;
  for (int y = 0; y < a.ng; ++y) {
    bool f;
    if (axis_src(a, y, f) == x) {
      ys[n] = y;
      fl[n++] = f;
    }
    int z = a.n - 1 - y;
    if (axis_src(a, z, f) == x) {
      ys[n] = z;
      fl[n++] = f;
    }
  }
  return n;
}

AxisAdj make_axis(int nc, int ng, int lo, int hi) { return AxisAdj{nc, ng, lo, hi}; }

// gather of the cotangent of a boundary-filled array onto interior cell (k,j,i)
__device__ __forceinline__ double bc_gather(const double* g, int64_t sv, int nc1, int nc2, int v,
                                            bool normals, const AxisAdj& a1, const AxisAdj& a2,
                                            const AxisAdj& a3, int i, int j, int k) {
  int y1[2 * kMaxGhost + 1], y2[2 * kMaxGhost + 1], y3[2 * kMaxGhost + 1];
  bool f1[2 * kMaxGhost + 1], f2[2 * kMaxGhost + 1], f3[2 * kMaxGhost + 1];
  int n1 = axis_images(a1, i, y1, f1);
  int n2 = axis_images(a2, j, y2, f2);
  int n3 = axis_images(a3, k, y3, f3);
  double acc = 0.;
  for (int c = 0; c < n3; ++c)
    for (int b = 0; b < n2; ++b)
      for (int a = 0; a < n1; ++a) {
        double x = g[v * sv + ((int64_t)y3[c] * nc2 + y2[b]) * nc1 + y1[a]];
        bool neg = false;
        if (normals) {
          if (v == IVX && f1[a]) neg = !neg;
          if (v == IVY && f2[b]) neg = !neg;
          if (v == IVZ && f3[c]) neg = !neg;
        }
        acc += neg ? -x : x;
      }
  return acc;
}

// ---------------------------------------------------------------------------
// (A) BC^T and the RK weights.  Every cell: interior cells gather their
// images; ghost entries of g_u (and of the stage cotangent GD) are zero.
// ---------------------------------------------------------------------------
struct CombineArgs {
  const double* gu_out;  // [nvar][sv] cotangent of the stage output (after BC)
  const double* gs_out;  // [ns][sv]
  double* gu;            // [nvar][sv] out: wgt1 * BC^T(gu_out) (interior), 0 (ghosts)
  double* gs;
  double* gu0;           // [nvar][sv] in/out: += wgt0 * BC^T(gu_out) on the interior
  double* gs0;
  double* GD;            // [nvar+ns][sv] out: wgt2 * BC^T(g_out): cotangent of du, ds
  double w0, w1, w2;
  int ns;
  AxisAdj a1, a2, a3;
};

__global__ void k_adj_combine(Geo g, CombineArgs A) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.sv) return;
  const int i = umod(t, g.nc1);
  const int j = umod(udiv(t, g.nc1), g.nc2);
  const int k = udiv(t, (int64_t)g.nc1 * g.nc2);
  const bool inner = i >= g.il && i <= g.iu && j >= g.jl && j <= g.ju && k >= g.kl && k <= g.ku;
  const int64_t sv = g.sv;
  for (int v = 0; v < 5; ++v) {
    double x = inner ? bc_gather(A.gu_out, sv, g.nc1, g.nc2, v, true, A.a1, A.a2, A.a3, i, j, k)
                     : 0.;
    A.gu[v * sv + t] = A.w1 * x;
    if (inner) A.gu0[v * sv + t] += A.w0 * x;
    A.GD[v * sv + t] = A.w2 * x;
  }
  for (int n = 0; n < A.ns; ++n) {
    double x = inner ? bc_gather(A.gs_out, sv, g.nc1, g.nc2, n, false, A.a1, A.a2, A.a3, i, j, k)
                     : 0.;
    A.gs[n * sv + t] = A.w1 * x;
    if (inner) A.gs0[n * sv + t] += A.w0 * x;
    A.GD[(5 + n) * sv + t] = A.w2 * x;
  }
}

// in-place BC^T: interior cells gather their images, ghosts become zero
// (two passes through a scratch copy so that the gather reads the input)
__global__ void k_bc_adjoint(Geo g, const double* gin, double* gout, int nv, int normals,
                             AxisAdj a1, AxisAdj a2, AxisAdj a3) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.sv) return;
  const int i = umod(t, g.nc1);
  const int j = umod(udiv(t, g.nc1), g.nc2);
  const int k = udiv(t, (int64_t)g.nc1 * g.nc2);
  const bool inner = i >= g.il && i <= g.iu && j >= g.jl && j <= g.ju && k >= g.kl && k <= g.ku;
  for (int v = 0; v < nv; ++v)
    gout[v * g.sv + t] =
        inner ? bc_gather(gin, g.sv, g.nc1, g.nc2, v, normals != 0, a1, a2, a3, i, j, k) : 0.;
}

// interior-masked copy of a du cotangent (ghost entries must read as zero)
__global__ void k_mask_interior(Geo g, const double* src, double* dst, int nv) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.sv) return;
  const int i = umod(t, g.nc1);
  const int j = umod(udiv(t, g.nc1), g.nc2);
  const int k = udiv(t, (int64_t)g.nc1 * g.nc2);
  const bool inner = i >= g.il && i <= g.iu && j >= g.jl && j <= g.ju && k >= g.kl && k <= g.ku;
  for (int v = 0; v < nv; ++v) dst[v * g.sv + t] = inner ? src[v * g.sv + t] : 0.;
}

// ---------------------------------------------------------------------------
// Local reverse maps
// ---------------------------------------------------------------------------

// WENO5-JS face value (weno5_face) reversed by hand: g * d out / d (a..e),
// accumulated into gx[0..4].  With omega_k = alpha_k / sum(alpha):
//   d out / d p_k = omega_k,  d out / d beta_k = -2 omega_k (p_k - out) / (beta_k + eps);
// the mean-|phi| scaling adds sign(x_i)/5 * (W - sum_j y_j dW/dy_j).
__device__ __forceinline__ void weno5_face_vjp(double a, double b, double c, double d, double e,
                                               bool scale, double g, double* gx) {
  double x[5] = {a, b, c, d, e};
  double vs = 1.;
  if (scale) {
    vs = (fabs(a) + fabs(b) + fabs(c) + fabs(d) + fabs(e)) / 5.;
    if (vs == 0.) return;  // the forward returns the constant 0
    double iv = 1. / vs;
#pragma unroll
    for (int q = 0; q < 5; ++q) x[q] *= iv;
  }
  const double c16 = 1. / 6., c56 = 5. / 6., c13 = 1. / 3.;
  const double c116 = 11. / 6., c76 = 7. / 6., c1312 = 13. / 12.;
  double y0 = x[0], y1 = x[1], y2 = x[2], y3 = x[3], y4 = x[4];
  double p0 = -c16 * y0 + c56 * y1 + c13 * y2;
  double p1 = c13 * y1 + c56 * y2 - c16 * y3;
  double p2 = c116 * y2 - c76 * y3 + c13 * y4;
  double u0 = y0 - 2. * y1 + y2, v0 = y0 - 4. * y1 + 3. * y2;
  double u1 = y1 - 2. * y2 + y3, v1 = y3 - y1;
  double u2 = y2 - 2. * y3 + y4, v2 = 3. * y2 - 4. * y3 + y4;
  double b0 = c1312 * u0 * u0 + 0.25 * v0 * v0;
  double b1 = c1312 * u1 * u1 + 0.25 * v1 * v1;
  double b2 = c1312 * u2 * u2 + 0.25 * v2 * v2;
  double e0 = b0 + 1e-6, e1 = b1 + 1e-6, e2 = b2 + 1e-6;
  double a0 = 0.3 / (e0 * e0), a1 = 0.6 / (e1 * e1), a2 = 0.1 / (e2 * e2);
  double is = 1. / (a0 + a1 + a2);
  double o0 = a0 * is, o1 = a1 * is, o2 = a2 * is;
  double W = o0 * p0 + o1 * p1 + o2 * p2;
  double gb0 = -2. * o0 * (p0 - W) / e0;
  double gb1 = -2. * o1 * (p1 - W) / e1;
  double gb2 = -2. * o2 * (p2 - W) / e2;
  const double k13 = 13. / 6.;
  double gy[5];
  gy[0] = -c16 * o0 + gb0 * (k13 * u0 + 0.5 * v0);
  gy[1] = c56 * o0 + c13 * o1 + gb0 * (-2. * k13 * u0 - 2. * v0) + gb1 * (k13 * u1 - 0.5 * v1);
  gy[2] = c13 * o0 + c56 * o1 + c116 * o2 + gb0 * (k13 * u0 + 1.5 * v0) +
          gb1 * (-2. * k13 * u1) + gb2 * (k13 * u2 + 1.5 * v2);
  gy[3] = -c16 * o1 - c76 * o2 + gb1 * (k13 * u1 + 0.5 * v1) + gb2 * (-2. * k13 * u2 - 2. * v2);
  gy[4] = c13 * o2 + gb2 * (k13 * u2 + 0.5 * v2);
  if (!scale) {
#pragma unroll
    for (int q = 0; q < 5; ++q) gx[q] += g * gy[q];
    return;
  }
  double ydw = 0.;
#pragma unroll
  for (int q = 0; q < 5; ++q) ydw += x[q] * gy[q];
  double corr = (W - ydw) / 5.;
  double raw[5] = {a, b, c, d, e};
#pragma unroll
  for (int q = 0; q < 5; ++q) gx[q] += g * (gy[q] + (raw[q] < 0. ? -corr : corr));
}

// g_L * dL/dq + g_R * dR/dq of face_states over the six-cell window
__device__ __forceinline__ void face_states_vjp(int type, bool scale, const double* q, double gl,
                                                double gr, double* gq) {
  switch (type) {
    case SNAPB_RECON_WENO5: {
      double t[5] = {0., 0., 0., 0., 0.};
      weno5_face_vjp(q[4], q[3], q[2], q[1], q[0], scale, gl, t);
      gq[4] += t[0];
      gq[3] += t[1];
      gq[2] += t[2];
      gq[1] += t[3];
      gq[0] += t[4];
      double s[5] = {0., 0., 0., 0., 0.};
      weno5_face_vjp(q[1], q[2], q[3], q[4], q[5], scale, gr, s);
#pragma unroll
      for (int k = 0; k < 5; ++k) gq[1 + k] += s[k];
      return;
    }
    case SNAPB_RECON_CP5: {
      const double a = -1. / 20., b = 9. / 20., c = 47. / 60., d = -13. / 60., e = 1. / 30.;
      gq[4] += a * gl;
      gq[3] += b * gl;
      gq[2] += c * gl;
      gq[1] += d * gl;
      gq[0] += e * gl;
      gq[1] += a * gr;
      gq[2] += b * gr;
      gq[3] += c * gr;
      gq[4] += d * gr;
      gq[5] += e * gr;
      return;
    }
    case SNAPB_RECON_CP3: {
      const double a = 1. / 3., b = 5. / 6., c = -1. / 6.;
      gq[3] += a * gl;
      gq[2] += b * gl;
      gq[1] += c * gl;
      gq[2] += a * gr;
      gq[3] += b * gr;
      gq[4] += c * gr;
      return;
    }
    case SNAPB_RECON_DC:
      gq[2] += gl;
      gq[3] += gr;
      return;
    default: {
      // WENO3 and PLM: one dual pass per window slot
      for (int s = 1; s < 5; ++s) {
        Dual qd[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) qd[k] = Dual(q[k], k == s ? 1. : 0.);
        Dual l, r;
        face_states<Dual>(type, scale, qd, l, r);
        gq[s] += gl * l.d + gr * r.d;
      }
    }
  }
}

// Reverse of one face: window q (cells f-3 .. f+2) of the nvar primitives and
// the ns mixing ratios, the cotangent gFin of its nvar + ns fluxes; adds the
// window cotangents into gq.  rev_l / rev_r: the x1 hydrostatic face
// revisions (left state takes the right state's p, rho at the lower boundary
// face, and the converse at the upper one).
template <int NS>
__device__ __forceinline__ void face_vjp(const Phys& p, int rtype, int rshock, int rscale, int ivx,
                                         bool disabled, bool rev_l, bool rev_r,
                                         const double (&q)[5 + NS][6],
                                         const double (&gFin)[5 + NS], double (&gq)[5 + NS][6]) {
  constexpr int NV = 5 + NS;
  double L[NV], R[NV], Lraw[NV > 5 ? NV : 6], Rraw[NV > 5 ? NV : 6];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    if (v < 5) {
      int typ = (rshock || v == IDN) ? rtype : interp2_of(rtype);
      face_states(typ, rscale != 0, q[v], L[v], R[v]);
    } else {
      face_states(p.rs_type, p.rs_scale != 0, q[v], Lraw[v], Rraw[v]);
      L[v] = Lraw[v] < 0. ? 0. : Lraw[v];
      R[v] = Rraw[v] < 0. ? 0. : Rraw[v];
    }
  }
  if (rev_l) {
    L[IPR] = R[IPR];
    L[IDN] = R[IDN];
  }
  if (rev_r) {
    R[IPR] = L[IPR];
    R[IDN] = L[IDN];
  }
  double gL[NV], gR[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) gL[v] = gR[v] = 0.;
  if (!disabled) {
    double F[5];
    riemann_flux(p.riemann, L, R, ivx, p.gammad, F);
    double gF[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) gF[v] = gFin[v];
    // scalar upwind flux F_s = F[IDN] * (F[IDN] > 0 ? r_L : r_R)
#pragma unroll
    for (int n = 0; n < NS; ++n) {
      double gs = gFin[5 + n];
      if (F[IDN] > 0.) {
        gF[IDN] += gs * L[5 + n];
        gL[5 + n] = gs * F[IDN];
      } else {
        gF[IDN] += gs * R[5 + n];
        gR[5 + n] = gs * F[IDN];
      }
    }
    riemann_vjp_rev(p.riemann, L, R, ivx, p.gammad, gF, gL, gR);
  }
  if (rev_l) {
    gR[IPR] += gL[IPR];
    gL[IPR] = 0.;
    gR[IDN] += gL[IDN];
    gL[IDN] = 0.;
  }
  if (rev_r) {
    gL[IPR] += gR[IPR];
    gR[IPR] = 0.;
    gL[IDN] += gR[IDN];
    gR[IDN] = 0.;
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    if (v < 5) {
      int typ = (rshock || v == IDN) ? rtype : interp2_of(rtype);
      face_states_vjp(typ, rscale != 0, q[v], gL[v], gR[v], gq[v]);
    } else {
      double gl = Lraw[v] < 0. ? 0. : gL[v];
      double gr = Rraw[v] < 0. ? 0. : gR[v];
      face_states_vjp(p.rs_type, p.rs_scale != 0, q[v], gl, gr, gq[v]);
    }
  }
}

// The same reverse for an x1 face whose window lives in shared memory (wb:
// the column's NV rows of nc1 cells); the window cotangents are added into the
// column's shared accumulator gb with shared-memory atomics, so no per-face
// array of contributions is held in registers.
template <int NS>
__device__ __forceinline__ void face_vjp_smem(const Phys& p, int rtype, int rshock, int rscale,
                                              bool disabled, bool rev_l, bool rev_r,
                                              const double* wb, int nc1, int f,
                                              const double (&gFin)[5 + NS], double* gb) {
  constexpr int NV = 5 + NS;
  double L[NV], R[NV], Lraw[NV > 5 ? NV : 6], Rraw[NV > 5 ? NV : 6];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double q[6];
#pragma unroll
    for (int t = 0; t < 6; ++t) q[t] = wb[v * nc1 + f - 3 + t];
    if (v < 5) {
      int typ = (rshock || v == IDN) ? rtype : interp2_of(rtype);
      face_states(typ, rscale != 0, q, L[v], R[v]);
    } else {
      face_states(p.rs_type, p.rs_scale != 0, q, Lraw[v], Rraw[v]);
      L[v] = Lraw[v] < 0. ? 0. : Lraw[v];
      R[v] = Rraw[v] < 0. ? 0. : Rraw[v];
    }
  }
  if (rev_l) {
    L[IPR] = R[IPR];
    L[IDN] = R[IDN];
  }
  if (rev_r) {
    R[IPR] = L[IPR];
    R[IDN] = L[IDN];
  }
  double gL[NV], gR[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) gL[v] = gR[v] = 0.;
  if (!disabled) {
    double F[5];
    riemann_flux(p.riemann, L, R, IVX, p.gammad, F);
    double gF[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) gF[v] = gFin[v];
#pragma unroll
    for (int n = 0; n < NS; ++n) {
      double gs = gFin[5 + n];
      if (F[IDN] > 0.) {
        gF[IDN] += gs * L[5 + n];
        gL[5 + n] = gs * F[IDN];
      } else {
        gF[IDN] += gs * R[5 + n];
        gR[5 + n] = gs * F[IDN];
      }
    }
    riemann_vjp_rev(p.riemann, L, R, IVX, p.gammad, gF, gL, gR);
  }
  if (rev_l) {
    gR[IPR] += gL[IPR];
    gL[IPR] = 0.;
    gR[IDN] += gL[IDN];
    gL[IDN] = 0.;
  }
  if (rev_r) {
    gL[IPR] += gR[IPR];
    gR[IPR] = 0.;
    gL[IDN] += gR[IDN];
    gR[IDN] = 0.;
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double q[6], t6[6] = {0., 0., 0., 0., 0., 0.};
#pragma unroll
    for (int t = 0; t < 6; ++t) q[t] = wb[v * nc1 + f - 3 + t];
    if (v < 5) {
      int typ = (rshock || v == IDN) ? rtype : interp2_of(rtype);
      face_states_vjp(typ, rscale != 0, q, gL[v], gR[v], t6);
    } else {
      double gl = Lraw[v] < 0. ? 0. : gL[v];
      double gr = Rraw[v] < 0. ? 0. : gR[v];
      face_states_vjp(p.rs_type, p.rs_scale != 0, q, gl, gr, t6);
    }
#pragma unroll
    for (int t = 0; t < 6; ++t)
      if (t6[t] != 0.) atomicAdd(gb + v * nc1 + f - 3 + t, t6[t]);
  }
}

// Buffers of the stage adjoint (all [var][sv], FP64)
struct AdjBufs {
  const double* dt;
  const double* u;   // stage-start state (ghosts filled)
  const double* s;
  const double* W;   // primitives of u with the x1 ghost revision (recomputed)
  const double* R;   // mixing ratios s / rho (recomputed)
  const double* D;   // explicit du (recomputed; implicit solve only)
  double* GD;        // cotangent of du (nvar + ns); rows replaced by the VIC adjoint
  double* GW;        // cotangent of w (nvar) and r (ns), accumulated
  double* gu;        // out: += cotangent of u
  double* gs;        // out: += cotangent of s
  double* vic;       // VIC adjoint scratch
};

// ---------------------------------------------------------------------------
// x2 / x3 faces: one thread per (x1 cell, other index) and segment of faces
// ---------------------------------------------------------------------------
template <int NS, int AX>
__global__ void __launch_bounds__(128) k_march_adj(Geo g, Phys p, AdjBufs b, int seglen) {
  constexpr int NV = 5 + NS;
  const int ni = g.iu - g.il + 1;
  int lo, hi, olo, ohi;
  int64_t st, ost;
  if (AX == 2) {
    lo = g.jl, hi = g.ju, st = g.s2, olo = g.kl, ohi = g.ku, ost = g.s3;
  } else {
    lo = g.kl, hi = g.ku, st = g.s3, olo = g.jl, ohi = g.ju, ost = g.s2;
  }
  const int no = ohi - olo + 1;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (int64_t)ni * no) return;
  const int i = g.il + umod(tid, ni);
  const int o = olo + udiv(tid, ni);
  const int f0 = lo + blockIdx.y * seglen;
  if (f0 > hi + 1) return;
  const int f1 = min(f0 + seglen - 1, hi + 1);
  const int64_t base = i + o * ost;
  const int64_t sv = g.sv;
  const int ivx = AX == 2 ? IVY : IVZ;
  const double A = AX == 2 ? g.A2 : g.A3;
  const int disabled = AX == 2 ? p.disable2 : p.disable3;
  const double cf = *b.dt * A / g.vol;

  double q[NV][6], acc[NV][6];
  auto load = [&](int cell, int slot) {
    int64_t off = base + (int64_t)cell * st;
#pragma unroll
    for (int v = 0; v < 5; ++v) q[v][slot] = b.W[v * sv + off];
#pragma unroll
    for (int n = 0; n < NS; ++n) q[5 + n][slot] = b.R[n * sv + off];
  };
  auto gd = [&](int cell, double* out) {
    bool in = cell >= lo && cell <= hi;
    int64_t off = base + (int64_t)cell * st;
#pragma unroll
    for (int v = 0; v < NV; ++v) out[v] = in ? b.GD[v * sv + off] : 0.;
  };
  auto flush = [&](int cell, int slot) {
    int64_t off = base + (int64_t)cell * st;
#pragma unroll
    for (int v = 0; v < NV; ++v)
      if (acc[v][slot] != 0.) atomicAdd(&b.GW[v * sv + off], acc[v][slot]);
  };
#pragma unroll
  for (int t = 0; t < 5; ++t) load(f0 - 3 + t, t);
#pragma unroll
  for (int v = 0; v < NV; ++v)
#pragma unroll
    for (int t = 0; t < 6; ++t) acc[v][t] = 0.;
  double gm[NV], gp[NV];
  gd(f0 - 1, gm);
  for (int f = f0; f <= f1; ++f) {
    load(f + 2, 5);
    gd(f, gp);
    double gF[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) gF[v] = cf * (gp[v] - gm[v]);
    face_vjp<NS>(p, p.r23_type, p.r23_shock, p.r23_scale, ivx, disabled != 0, false, false, q, gF,
                 acc);
    // cell f-3 is complete
    flush(f - 3, 0);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
#pragma unroll
      for (int t = 0; t < 5; ++t) {
        q[v][t] = q[v][t + 1];
        acc[v][t] = acc[v][t + 1];
      }
      acc[v][5] = 0.;
      gm[v] = gp[v];
    }
  }
  // after the shift, slot t holds cell f1 - 2 + t
#pragma unroll
  for (int t = 0; t < 5; ++t) flush(f1 - 2 + t, t);
}

// ---------------------------------------------------------------------------
// x1: one CTA per group of columns (every column: the U->W reverse covers the
// ghost columns too)
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ void revise_end(T P, T Rr, double gamma, double a, double ia, double ig,
                                           double gdz, int ng, T* pout, T* rout) {
  T K = P / pow(Rr, gamma);
  T kg = pow(K, ig);
  T pc = P;
  for (int n = 0; n < ng; ++n) {
    T h = pow(pc, a) + T(gdz) / kg;
    T pn = pow(h, ia);
    pout[n] = pn;
    rout[n] = pow(pn / K, ig);
    pc = pn;
  }
}

template <int NS>
__global__ void __launch_bounds__(256, 2) k_x1_adj(Geo g, Phys p, AdjBufs b, int C) {
  constexpr int NV = 5 + NS;
  extern __shared__ double sm[];
  const int nc1 = g.nc1;
  double* sw = sm;                              // [C][NV][nc1] w, r
  double* sg = sw + (size_t)C * NV * nc1;       // [C][NV][nc1] cotangents of w, r
  const int64_t ncol = (int64_t)g.nc2 * g.nc3;
  const int64_t col0 = (int64_t)blockIdx.x * C;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int64_t sv = g.sv;
  const double dt = *b.dt;

  for (int idx = tid; idx < C * nc1; idx += nt) {
    int c = idx / nc1, i = idx - c * nc1;
    int64_t col = col0 + c;
    if (col >= ncol) continue;
    int64_t off = col * nc1 + i;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      sw[(c * NV + v) * nc1 + i] = b.W[v * sv + off];
      sg[(c * NV + v) * nc1 + i] = b.GW[v * sv + off];
    }
#pragma unroll
    for (int n = 0; n < NS; ++n) {
      sw[(c * NV + 5 + n) * nc1 + i] = b.R[n * sv + off];
      sg[(c * NV + 5 + n) * nc1 + i] = b.GW[(5 + n) * sv + off];
    }
  }
  __syncthreads();

  // x1 faces il .. iu+1 of interior columns; window cotangents accumulate in
  // shared memory through atomics
  const int nf = g.nx1 + 1;
  const double cf = dt * g.A1 / g.vol;
  const bool grav = p.grav1 != 0.;
  for (int idx = tid; idx < C * nf; idx += nt) {
    int c = idx / nf, f = g.il + (idx - c * nf);
    int64_t col = col0 + c;
    if (col >= ncol) continue;
    int j = umod(col, g.nc2), k = udiv(col, g.nc2);
    if (j < g.jl || j > g.ju || k < g.kl || k > g.ku) continue;
    int64_t off = col * nc1 + f;
    double gF[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) gF[v] = cf * (b.GD[v * sv + off] - b.GD[v * sv + off - 1]);
    face_vjp_smem<NS>(p, p.r1_type, p.r1_shock, p.r1_scale, p.disable1 != 0, grav && f == g.il,
                      grav && f == g.iu + 1, sw + (size_t)c * NV * nc1, nc1, f, gF,
                      sg + (size_t)c * NV * nc1);
  }
  __syncthreads();

  // gravity forcing of interior cells: du[IVX] += dt rho g1 nh,
  // du[IPR] += dt rho v1 g1 nh (and the x2 / x3 analogues)
  for (int idx = tid; idx < C * g.nx1; idx += nt) {
    int c = idx / g.nx1, i = g.il + (idx - c * g.nx1);
    int64_t col = col0 + c;
    if (col >= ncol) continue;
    int j = umod(col, g.nc2), k = udiv(col, g.nc2);
    if (j < g.jl || j > g.ju || k < g.kl || k > g.ku) continue;
    int64_t off = col * nc1 + i;
    const double* wb = sw + (size_t)c * NV * nc1 + i;
    double* gb = sg + (size_t)c * NV * nc1 + i;
    double rho = wb[IDN * nc1];
    double gdp = b.GD[IPR * sv + off];
    if (p.grav1 != 0.) {
      double k1 = dt * p.grav1 * p.nh;
      gb[IDN * nc1] += k1 * (b.GD[IVX * sv + off] + wb[IVX * nc1] * gdp);
      gb[IVX * nc1] += k1 * rho * gdp;
    }
    if (p.grav2 != 0.) {
      double k2 = dt * p.grav2;
      gb[IDN * nc1] += k2 * (b.GD[IVY * sv + off] + wb[IVY * nc1] * gdp);
      gb[IVY * nc1] += k2 * rho * gdp;
    }
    if (p.grav3 != 0.) {
      double k3 = dt * p.grav3;
      gb[IDN * nc1] += k3 * (b.GD[IVZ * sv + off] + wb[IVZ * nc1] * gdp);
      gb[IVZ * nc1] += k3 * rho * gdp;
    }
  }
  __syncthreads();

  // reverse of the isentropic ghost revision (every column, like the forward)
  if (p.grav1 != 0. && tid < 2 * C) {
    int c = tid >> 1, top = tid & 1;
    if (col0 + c < ncol) {
      const double gamma = p.gammad;
      const double a = (gamma - 1.) / gamma, ig = 1. / gamma, ia = 1. / a;
      const double grav = -p.grav1, dz = g.dx1;
      const int ng = g.ng;
      const int edge = top ? g.iu : g.il;
      const double gdz = top ? -a * grav * dz : a * grav * dz;
      double* gpp = sg + (size_t)(c * NV + IPR) * nc1;
      double* grr = sg + (size_t)(c * NV + IDN) * nc1;
      const double* wpp = sw + (size_t)(c * NV + IPR) * nc1;
      const double* wrr = sw + (size_t)(c * NV + IDN) * nc1;
      double gP = 0., gR = 0.;
      for (int dir = 0; dir < 2; ++dir) {
        Dual P(wpp[edge], dir == 0 ? 1. : 0.), Rr(wrr[edge], dir == 1 ? 1. : 0.);
        Dual po[kMaxGhost], ro[kMaxGhost];
        revise_end<Dual>(P, Rr, gamma, a, ia, ig, gdz, ng, po, ro);
        double s = 0.;
        for (int n = 0; n < ng; ++n) {
          int cell = top ? edge + n + 1 : edge - n - 1;
          s += gpp[cell] * po[n].d + grr[cell] * ro[n].d;
        }
        if (dir == 0)
          gP = s;
        else
          gR = s;
      }
      for (int n = 0; n < ng; ++n) {
        int cell = top ? edge + n + 1 : edge - n - 1;
        gpp[cell] = 0.;
        grr[cell] = 0.;
      }
      gpp[edge] += gP;
      grr[edge] += gR;
    }
  }
  __syncthreads();

  // U -> W reverse (and r = s / rho) for every cell of the columns
  const double gm1 = p.gammad - 1.;
  for (int idx = tid; idx < C * nc1; idx += nt) {
    int c = idx / nc1, i = idx - c * nc1;
    int64_t col = col0 + c;
    if (col >= ncol) continue;
    int64_t off = col * nc1 + i;
    const double* gb = sg + (size_t)c * NV * nc1 + i;
    double rho = b.u[IDN * sv + off];
    double ir = 1. / rho;
    double vel[3], ke2 = 0.;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      vel[k] = b.u[(IVX + k) * sv + off] * ir;
      ke2 += vel[k] * vel[k];
    }
    double gp = gb[IPR * nc1];
    double gr = gb[IDN * nc1] + gp * gm1 * 0.5 * ke2;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double gv = gb[(IVX + k) * nc1];
      gr -= gv * vel[k] * ir;
      b.gu[(IVX + k) * sv + off] += gv * ir - gp * gm1 * vel[k];
    }
    b.gu[IPR * sv + off] += gp * gm1;
#pragma unroll
    for (int n = 0; n < NS; ++n) {
      double grn = gb[(5 + n) * nc1];
      double rn = b.s[n * sv + off] * ir;
      gr -= grn * rn * ir;
      b.gs[n * sv + off] += grn * ir;
    }
    b.gu[IDN * sv + off] += gr;
  }
}

// U -> W reverse and gravity when x1 is inactive (one thread per cell)
template <int NS>
__global__ void k_cell_adj(Geo g, Phys p, AdjBufs b) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.sv) return;
  const int64_t sv = g.sv;
  const double dt = *b.dt;
  const int i = umod(t, g.nc1);
  const int j = umod(udiv(t, g.nc1), g.nc2);
  const int k = udiv(t, (int64_t)g.nc1 * g.nc2);
  const bool inner = i >= g.il && i <= g.iu && j >= g.jl && j <= g.ju && k >= g.kl && k <= g.ku;
  double gw[5 + NS];
#pragma unroll
  for (int v = 0; v < 5 + NS; ++v) gw[v] = b.GW[v * sv + t];
  if (inner) {
    double rho = b.W[IDN * sv + t];
    double gdp = b.GD[IPR * sv + t];
    if (p.grav2 != 0.) {
      gw[IDN] += dt * p.grav2 * (b.GD[IVY * sv + t] + b.W[IVY * sv + t] * gdp);
      gw[IVY] += dt * p.grav2 * rho * gdp;
    }
    if (p.grav3 != 0.) {
      gw[IDN] += dt * p.grav3 * (b.GD[IVZ * sv + t] + b.W[IVZ * sv + t] * gdp);
      gw[IVZ] += dt * p.grav3 * rho * gdp;
    }
  }
  const double gm1 = p.gammad - 1.;
  double rho = b.u[IDN * sv + t];
  double ir = 1. / rho;
  double vel[3], ke2 = 0.;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    vel[q] = b.u[(IVX + q) * sv + t] * ir;
    ke2 += vel[q] * vel[q];
  }
  double gp = gw[IPR];
  double gr = gw[IDN] + gp * gm1 * 0.5 * ke2;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    gr -= gw[IVX + q] * vel[q] * ir;
    b.gu[(IVX + q) * sv + t] += gw[IVX + q] * ir - gp * gm1 * vel[q];
  }
  b.gu[IPR * sv + t] += gp * gm1;
#pragma unroll
  for (int n = 0; n < NS; ++n) {
    double rn = b.s[n * sv + t] * ir;
    gr -= gw[5 + n] * rn * ir;
    b.gs[n * sv + t] += gw[5 + n] * ir;
  }
  b.gu[IDN * sv + t] += gr;
}

// ---------------------------------------------------------------------------
// VIC adjoint.  Scratch (doubles, column index fastest):
//   T [nl+2][E1][ncol]  per t: |A| at face t (N*N), J of cell t-1 (N*N),
//                       explicit du rows of cell t (N), rho of cell t, the
//                       output cotangent rows of cell t (N), g_fix of cell t
//   S [nl][ES][ncol]    per layer: a~_i = ahat_i^-1 c_i (N*N), ahat_i (N*N),
//                       delta_i (N), t_i (N)
//   Z [3][ncol]         B_dry / sum (rho V)^2, g_S, g_B
// ---------------------------------------------------------------------------
template <int N>
struct VadjDims {
  static constexpr int E1 = 2 * N * N + 2 * N + 2;
  static constexpr int ES = 2 * N * N + 3 * N;
};

static inline int vic_n_adj(const Phys& p) { return ((p.implicit_scheme >> 3) & 1) ? 5 : 3; }

size_t vic_adj_scratch_bytes(const Geo& g, const Phys& p) {
  if (p.implicit_scheme == 0) return 0;
  int N = vic_n_adj(p);
  int64_t ncol = (int64_t)(g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  int64_t nl = g.nx1;
  int64_t e1 = 2 * N * N + 2 * N + 2, es = 2 * N * N + 3 * N;
  return (size_t)((nl + 2) * e1 * ncol + nl * es * ncol + 3 * ncol) * sizeof(double);
}

constexpr int kATC = 32;   // columns per tile (assembly)
template <int N>
constexpr int kATL = N == 5 ? 8 : 12;  // layers per tile (assembly; static smem <= 48 KB)
constexpr int kCTC = 16;   // columns per tile (contraction)
constexpr int kCTL = 32;   // cells per tile (contraction)

__device__ __forceinline__ int64_t adj_column_base(const Geo& g, int64_t col) {
  const int nj = g.ju - g.jl + 1;
  const int j = g.jl + umod(col, nj), k = g.kl + udiv(col, nj);
  return (int64_t)k * g.s3 + (int64_t)j * g.s2 + g.il;
}

template <int N, int NS>
__global__ void __launch_bounds__(256) k_vadj_assemble(Geo g, Phys p, AdjBufs b) {
  constexpr int E1 = VadjDims<N>::E1;
  const int nl = g.nx1;
  const int64_t ncol = (int64_t)(g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  const int64_t col0 = (int64_t)blockIdx.x * kATC;
  constexpr int TL = kATL<N>;
  const int t0 = blockIdx.y * TL;
  const int64_t sv = g.sv;
  __shared__ double ws[5][kATC][TL + 2];          // cells t0-1 .. t0+TL
  __shared__ double ds[2 * N + 1][kATC][TL + 1];  // du rows, g rows, g_fix of cells t0..
  const int tid = threadIdx.x;
  for (int idx = tid; idx < 5 * kATC * (TL + 1); idx += blockDim.x) {
    int s = idx % (TL + 1), rest = idx / (TL + 1);
    int c = rest % kATC, v = rest / kATC;
    int cell = t0 - 1 + s;
    int64_t col = col0 + c;
    double x = 0.;
    if (col < ncol && cell >= -1 && cell <= nl) x = b.W[v * sv + adj_column_base(g, col) + cell];
    ws[v][c][s] = x;
  }
  for (int idx = tid; idx < (2 * N + 1) * kATC * TL; idx += blockDim.x) {
    int s = idx % TL, rest = idx / TL;
    int c = rest % kATC, r = rest / kATC;
    int cell = t0 + s;
    int64_t col = col0 + c;
    double x = 0.;
    if (col < ncol && cell < nl) {
      int64_t off = adj_column_base(g, col) + cell;
      if (r < N)
        x = b.D[sel<N>(r) * sv + off];
      else if (r < 2 * N)
        x = b.GD[sel<N>(r - N) * sv + off];
      else {
#pragma unroll
        for (int n = 0; n < NS; ++n) x += b.GD[(5 + n) * sv + off] * b.R[n * sv + off];
      }
    }
    ds[r][c][s] = x;
  }
  __syncthreads();
  const double gm1c = p.gammad - 1.;
  const double gm1f = 0.5 * (p.gammad + p.gammad) - 1.;
  double* T = b.vic;
  for (int idx = tid; idx < kATC * TL; idx += blockDim.x) {
    int c = idx % kATC, s = idx / kATC;
    int t = t0 + s;
    int64_t col = col0 + c;
    if (col >= ncol || t > nl + 1) continue;
    double wl[5], wr[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      wl[v] = ws[v][c][s];
      wr[v] = ws[v][c][s + 1];
    }
    double* out = T + (int64_t)t * E1 * ncol + col;
    double A[N][N], J[N][N];
    if (t <= nl) {
      absA_block<N>(gm1f, wl, wr, A);
    } else {
#pragma unroll
      for (int r = 0; r < N; ++r)
#pragma unroll
        for (int q = 0; q < N; ++q) A[r][q] = 0.;
    }
    jac_block<N>(gm1c, wl, J);
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
      for (int q = 0; q < N; ++q) {
        out[(r * N + q) * ncol] = A[r][q];
        out[(N * N + r * N + q) * ncol] = J[r][q];
      }
#pragma unroll
    for (int r = 0; r < N; ++r) {
      out[(2 * N * N + r) * ncol] = t < nl ? ds[r][c][s] : 0.;
      out[(2 * N * N + N + 1 + r) * ncol] = t < nl ? ds[N + r][c][s] : 0.;
    }
    out[(2 * N * N + N) * ncol] = t < nl ? wr[IDN] : 0.;
    out[(2 * N * N + 2 * N + 1) * ncol] = t < nl ? ds[2 * N][c][s] : 0.;
  }
}

// x = M^-T y for an N x N block (M^T solved as a fresh system).  Kept out of
// line: inlined into k_vadj_sweep's unrolled body (nvcc 12.9, sm_100a) the
// N = 5 solve returned non-zero x for y = 0; called out of line it is exact.
template <int N>
__device__ __noinline__ void solve_transposed(const double (&M)[N][N], double (&y)[N]) {
  double Mt[N][N], Z[N][N];
#pragma unroll
  for (int r = 0; r < N; ++r)
#pragma unroll
    for (int q = 0; q < N; ++q) {
      Mt[r][q] = M[q][r];
      Z[r][q] = 0.;
    }
  block_solve<N>(Mt, Z, y);
}

// Per-thread ring (see ring.cuh) for the two sequential passes of
// k_vadj_sweep: depth layers ahead, elems doubles per slot (the widest pass,
// the backward one: the reduced block and partial solution, h0 and h1, ahat
// or its inverse, |A| and J of the face / cell above).
template <int N>
struct VadjRing {
  static constexpr int depth = N == 3 ? 4 : 2;
  static constexpr int elems = 4 * N * N + 3 * N + 1;
};
template <int N>
constexpr size_t vadj_ring_bytes(int threads) {
  return (size_t)threads * VadjRing<N>::depth * VadjRing<N>::elems * sizeof(double);
}

template <int N>
__global__ void __launch_bounds__(128) k_vadj_sweep(Geo g, Phys p, AdjBufs b) {
  constexpr int E1 = VadjDims<N>::E1, ES = VadjDims<N>::ES, NN = N * N;
  constexpr int D = VadjRing<N>::depth;
  const int64_t ncol = (int64_t)(g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  const int64_t col = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncol) return;
  const int nl = g.nx1;
  const double* T = b.vic + col;
  double* S = b.vic + (int64_t)(nl + 2) * E1 * ncol + col;
  double* Z = S + (int64_t)nl * ES * ncol;
  auto Tp = [&](int t, int e) { return T + ((int64_t)t * E1 + e) * ncol; };
  auto Sat = [&](int i, int e) -> double& { return S[((int64_t)i * ES + e) * ncol]; };
  const int oAT = 0, oAH = NN, oD = 2 * NN, oT = 2 * NN + N, oH1 = 2 * NN + 2 * N;
  // T entries of index t: |A| (0), J (NN), du rows (2NN), rho (2NN+N),
  // output cotangent rows (2NN+N+1), g_fix (2NN+2N+1)
  const int tA = 0, tJ = NN, tDU = 2 * NN, tRHO = 2 * NN + N, tG = 2 * NN + N + 1,
            tGF = 2 * NN + 2 * N + 1;
  extern __shared__ double vadj_ring[];
  // ring pass: fetch(i, slot) issues layer i's copies; the sweep visits
  // layers i0, i0+step, ... (n of them)
  auto prologue = [&](auto fetch, int i0, int step, int n) {
#pragma unroll
    for (int k = 0; k < D; ++k) {
      if (k < n) fetch(i0 + k * step, k);
      else cp_async_commit();
    }
  };
  const int nt = blockDim.x, lane = threadIdx.x;

  const double dt = *b.dt;
  const double Aa = g.A1, hiv = 0.5 / g.vol, idt = 1. / dt, grav = p.grav1, V = g.vol;

  // (A) forward elimination as the forward column sweep, keeping the
  // inverse of each reduced diagonal block ahat_i (N = 3; the block itself
  // for N = 5), with the forward recurrence of the transposed solve beside
  // it: h_i = g_delta_i - a~_{i-1}^T h_{i-1}.  Its redistribution term
  // -V g_B e_0 is linear in g_B, which is known only at the end of this pass,
  // so it runs as h = h0 + g_B h1.
  constexpr int E_1 = 2 * NN + 2 * N + 2;
  static_assert(E_1 <= VadjRing<N>::elems, "ring slot");
  Ring r1{vadj_ring, E_1, nt, lane};
  auto fetch1 = [&](int i, int slot) {
    if (i < nl) {
#pragma unroll
      for (int e = 0; e < NN; ++e) cp_async_bytes8(r1.at(slot, e), Tp(i + 1, tA + e));
#pragma unroll
      for (int e = 0; e < NN; ++e) cp_async_bytes8(r1.at(slot, NN + e), Tp(i + 2, tJ + e));
#pragma unroll
      for (int r = 0; r < N; ++r) cp_async_bytes8(r1.at(slot, 2 * NN + r), Tp(i, tDU + r));
      cp_async_bytes8(r1.at(slot, 2 * NN + N), Tp(i, tRHO));
#pragma unroll
      for (int r = 0; r < N; ++r)  // output cotangent rows
        cp_async_bytes8(r1.at(slot, 2 * NN + N + 1 + r), Tp(i, tG + r));
      cp_async_bytes8(r1.at(slot, 2 * NN + 2 * N + 1), Tp(i, tGF));
    }
    cp_async_commit();
  };
  prologue(fetch1, 0, 1, D);
  double Am[N][N], Jp[N][N], Jc[N][N], ap[N][N], dp[N], h0[N], h1[N];
#pragma unroll
  for (int r = 0; r < N; ++r) {
    h0[r] = 0.;
    h1[r] = 0.;
#pragma unroll
    for (int q = 0; q < N; ++q) {
      Am[r][q] = *Tp(0, tA + r * N + q);
      Jp[r][q] = *Tp(0, tJ + r * N + q);
      Jc[r][q] = *Tp(1, tJ + r * N + q);
      ap[r][q] = 0.;
    }
  }
  // sum (rho V)^2 and Q = sum g_out[IDN] rho (rho V): the redistribution's
  // cotangents are g_B = Q / S and g_S = -Q B_dry / S^2
  double sum_a2 = 0., qg = 0.;
  for (int i = 0, slot = 0; i < nl; ++i) {
    double Ap[N][N], Jn[N][N], rhs[N];
    cp_async_wait<D - 1>();
#pragma unroll
    for (int r = 0; r < N; ++r) {
      rhs[r] = *r1.at(slot, 2 * NN + r) / dt;
#pragma unroll
      for (int q = 0; q < N; ++q) {
        Ap[r][q] = *r1.at(slot, r * N + q);
        Jn[r][q] = *r1.at(slot, NN + r * N + q);
      }
    }
    const double rho = *r1.at(slot, 2 * NN + N), ai = rho * V;
    sum_a2 += ai * ai;
    qg += *r1.at(slot, 2 * NN + N + 1) * rho * ai;
    {  // h_i from h_{i-1} and the reduced block of layer i-1 (ap)
      double g0[N], g1[N];
#pragma unroll
      for (int r = 0; r < N; ++r) {
        g0[r] = *r1.at(slot, 2 * NN + N + 1 + r);
        g1[r] = 0.;
      }
      g0[0] += *r1.at(slot, 2 * NN + 2 * N + 1);
      g1[0] = -V;
#pragma unroll
      for (int q = 0; q < N; ++q) {
        double s0 = 0., s1 = 0.;
#pragma unroll
        for (int r = 0; r < N; ++r) {
          s0 += ap[r][q] * h0[r];
          s1 += ap[r][q] * h1[r];
        }
        g0[q] -= s0;
        g1[q] -= s1;
      }
#pragma unroll
      for (int r = 0; r < N; ++r) {
        h0[r] = g0[r];
        h1[r] = g1[r];
        Sat(i, oT + r) = g0[r];
        Sat(i, oH1 + r) = g1[r];
      }
    }
    double a[N][N], bb[N][N], c[N][N];
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
      for (int q = 0; q < N; ++q) {
        double phi = 0.;
        if (r == 1 && q == 0) phi = grav;
        if (N == 3 && r == 2 && q == 1) phi = grav;
        if (N == 5 && r == IPR && q == IVX) phi = grav;
        a[r][q] = (Am[r][q] * Aa + Ap[r][q] * Aa) * hiv - phi;
        bb[r][q] = -(Am[r][q] + Jp[r][q]) * Aa * hiv;
        c[r][q] = -(Ap[r][q] - Jn[r][q]) * Aa * hiv;
      }
#pragma unroll
    for (int r = 0; r < N; ++r) a[r][r] += idt;
    if (i == 0) {
#pragma unroll
      for (int r = 0; r < N; ++r)
#pragma unroll
        for (int q = 0; q < N; ++q) a[r][q] += bb[r][q] * (q == 1 ? -1. : 1.);
    }
    if (i == nl - 1) {
#pragma unroll
      for (int r = 0; r < N; ++r)
#pragma unroll
        for (int q = 0; q < N; ++q) a[r][q] += c[r][q] * (q == 1 ? -1. : 1.);
    }
    if (i > 0) {
#pragma unroll
      for (int r = 0; r < N; ++r) {
        double bd = 0.;
#pragma unroll
        for (int q = 0; q < N; ++q) {
          double t = 0.;
#pragma unroll
          for (int kk = 0; kk < N; ++kk) t += bb[r][kk] * ap[kk][q];
          a[r][q] -= t;
          bd += bb[r][q] * dp[q];
        }
        rhs[r] = rhs[r] - bd;
      }
    }
    if constexpr (N == 3) {
      double inv[3][3];
      inverse3(a, inv);
#pragma unroll
      for (int r = 0; r < N; ++r)
#pragma unroll
        for (int q = 0; q < N; ++q) Sat(i, oAH + r * N + q) = inv[r][q];
      apply_inverse3(inv, c, rhs);
    } else {
#pragma unroll
      for (int r = 0; r < N; ++r)
#pragma unroll
        for (int q = 0; q < N; ++q) Sat(i, oAH + r * N + q) = a[r][q];
      block_solve<N>(a, c, rhs);
    }
    fetch1(i + D, slot);  // consumed: refill
    slot = slot + 1 == D ? 0 : slot + 1;
#pragma unroll
    for (int r = 0; r < N; ++r) {
      dp[r] = rhs[r];
      Sat(i, oD + r) = rhs[r];
#pragma unroll
      for (int q = 0; q < N; ++q) {
        ap[r][q] = c[r][q];
        Sat(i, oAT + r * N + q) = c[r][q];
      }
    }
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
      for (int q = 0; q < N; ++q) {
        Am[r][q] = Ap[r][q];
        Jp[r][q] = Jc[r][q];
        Jc[r][q] = Jn[r][q];
      }
  }
  cp_async_wait<0>();
  const double gb = qg / sum_a2;

  // (B) back substitution (B_dry accumulated from the top as in the forward
  // sweep) with the backward recurrence of the transposed solve beside it:
  // t_i = ahat_i^-T (h_i - b_{i+1}^T t_{i+1}),
  // b_{i+1} = -(|A|_{face i+1} + J_{cell i}) A hiv
  constexpr int E_2 = 4 * NN + 3 * N + 1;
  static_assert(E_2 <= VadjRing<N>::elems, "ring slot");
  // slot: a~_i (0), d'_i (NN), du_i[IDN] (NN+N), h0_i (NN+N+1), h1_i
  // (NN+2N+1), ahat_i or its inverse (NN+3N+1), |A| and J of index i+1
  // (2NN+3N+1, 3NN+3N+1)
  const int sD = NN, sDU = NN + N, sH0 = NN + N + 1, sH1 = NN + 2 * N + 1, sM = NN + 3 * N + 1,
            sA = 2 * NN + 3 * N + 1, sJ = 3 * NN + 3 * N + 1;
  Ring r2{vadj_ring, E_2, nt, lane};
  auto fetch2 = [&](int i, int slot) {
    if (i >= 0) {
#pragma unroll
      for (int e = 0; e < NN; ++e) {
        cp_async_bytes8(r2.at(slot, e), &Sat(i, oAT + e));
        cp_async_bytes8(r2.at(slot, sM + e), &Sat(i, oAH + e));
      }
#pragma unroll
      for (int r = 0; r < N; ++r) {
        cp_async_bytes8(r2.at(slot, sD + r), &Sat(i, oD + r));
        cp_async_bytes8(r2.at(slot, sH0 + r), &Sat(i, oT + r));
        cp_async_bytes8(r2.at(slot, sH1 + r), &Sat(i, oH1 + r));
      }
      cp_async_bytes8(r2.at(slot, sDU), Tp(i, tDU));
      if (i + 1 < nl) {
#pragma unroll
        for (int e = 0; e < NN; ++e) {
          cp_async_bytes8(r2.at(slot, sA + e), Tp(i + 1, tA + e));
          cp_async_bytes8(r2.at(slot, sJ + e), Tp(i + 1, tJ + e));
        }
      }
    }
    cp_async_commit();
  };
  double dn[N], tn[N];
#pragma unroll
  for (int r = 0; r < N; ++r) {
    dn[r] = dp[r];
    tn[r] = 0.;
  }
  double b_dry = (*Tp(nl - 1, tDU) - dn[0]) * 1. * V;
  prologue(fetch2, nl - 1, -1, nl);
  for (int i = nl - 1, slot = 0; i >= 0; --i) {
    cp_async_wait<D - 1>();
    if (i < nl - 1) {  // delta_i = d'_i - a~_i delta_{i+1}
      double d[N];
#pragma unroll
      for (int r = 0; r < N; ++r) {
        double t = 0.;
#pragma unroll
        for (int q = 0; q < N; ++q) t += *r2.at(slot, r * N + q) * dn[q];
        d[r] = *r2.at(slot, sD + r) - t;
      }
      b_dry += (*r2.at(slot, sDU) - d[0]) * 1. * V;
#pragma unroll
      for (int r = 0; r < N; ++r) {
        dn[r] = d[r];
        Sat(i, oD + r) = d[r];
      }
    }
    double y[N];
#pragma unroll
    for (int r = 0; r < N; ++r) y[r] = *r2.at(slot, sH0 + r) + gb * *r2.at(slot, sH1 + r);
    if (i + 1 < nl) {
#pragma unroll
      for (int q = 0; q < N; ++q) {
        double sacc = 0.;
#pragma unroll
        for (int r = 0; r < N; ++r) {
          double bq = -(*r2.at(slot, sA + r * N + q) + *r2.at(slot, sJ + r * N + q)) * Aa * hiv;
          sacc += bq * tn[r];
        }
        y[q] -= sacc;
      }
    }
    double tv[N];
    if constexpr (N == 3) {
#pragma unroll
      for (int q = 0; q < N; ++q) {  // ahat^-T y
        double s = 0.;
#pragma unroll
        for (int r = 0; r < N; ++r) s += *r2.at(slot, sM + r * N + q) * y[r];
        tv[q] = s;
      }
    } else {
      double M[N][N];
#pragma unroll
      for (int r = 0; r < N; ++r)
#pragma unroll
        for (int q = 0; q < N; ++q) M[r][q] = *r2.at(slot, sM + r * N + q);
      solve_transposed<N>(M, y);
#pragma unroll
      for (int r = 0; r < N; ++r) tv[r] = y[r];
    }
    fetch2(i - D, slot);  // consumed: refill
    slot = slot + 1 == D ? 0 : slot + 1;
#pragma unroll
    for (int r = 0; r < N; ++r) {
      tn[r] = tv[r];
      Sat(i, oT + r) = tv[r];
    }
  }
  cp_async_wait<0>();

  // cotangents of the redistribution's B_dry and S
  Z[0] = b_dry / sum_a2;
  Z[ncol] = -qg * b_dry / (sum_a2 * sum_a2);
  Z[2 * ncol] = gb;
}

// Few columns (3x3 blocks): the two solves of the adjoint column sweep by
// block cyclic reduction, one CTA per column, the column's system in shared
// memory.  g_B = Q / S needs only the column sums, so the right-hand side of
// the transposed solve is known before either solve: A delta = du / dt gives
// the forward solution (and B_dry), A^T t = g_delta + (g_fix - V g_B) e_0 the
// transposed one, each in log2(nl) parallel steps instead of nl sequential
// layers.  The blocks are those of k_vadj_sweep (|A| and J from the assembly
// in T, the same folds at the first and last layers); the outputs (delta and
// t in S, the cotangents in Z) are the sweep's, up to FP64 rounding.
constexpr int kVadjCrThreads = 128;
constexpr int64_t kVadjCrMaxCols = 148 * 64;  // above this the sweep fills the GPU
inline size_t vadj_cr_smem_bytes(int nl) {
  return ((size_t)nl * 30 + 2 * (kVadjCrThreads / 32)) * sizeof(double);
}

__global__ void __launch_bounds__(kVadjCrThreads) k_vadj_cr3(Geo g, Phys p, AdjBufs b) {
  constexpr int N = 3, NN = 9;
  constexpr int E1 = VadjDims<N>::E1, ES = VadjDims<N>::ES;
  extern __shared__ __align__(16) double vadj_cr[];
  const int64_t ncol = (int64_t)(g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  const int64_t col = blockIdx.x;
  const int nl = g.nx1, tid = threadIdx.x, nt = blockDim.x;
  const double* T = b.vic + col;
  double* S = b.vic + (int64_t)(nl + 2) * E1 * ncol + col;
  double* Z = S + (int64_t)nl * ES * ncol;
  auto Tp = [&](int t, int e) { return T[((int64_t)t * E1 + e) * ncol]; };
  auto Sat = [&](int i, int e) -> double& { return S[((int64_t)i * ES + e) * ncol]; };
  const int tA = 0, tJ = NN, tDU = 2 * NN, tRHO = 2 * NN + N, tG = 2 * NN + N + 1,
            tGF = 2 * NN + 2 * N + 1;
  const int oD = 2 * NN, oT = 2 * NN + N;
  double* Bl = vadj_cr;         // [nl][9] block of x_{i-1}
  double* Dg = Bl + 9 * nl;     // [nl][9] diagonal block
  double* Ab = Dg + 9 * nl;     // [nl][9] block of x_{i+1}
  double* R = Ab + 9 * nl;      // [nl][3] right-hand side, then solution
  double* red = R + 3 * nl;     // reduction scratch
  const double dt = *b.dt;
  const double Aa = g.A1, hiv = 0.5 / g.vol, idt = 1. / dt, grav = p.grav1, V = g.vol;
  // b_i (x_{i-1}), a_i (folded) and c_i (x_{i+1}) of layer i, as the sweep
  // forms them
  auto blocks = [&](int i, double (&a)[N][N], double (&bb)[N][N], double (&c)[N][N]) {
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
      for (int q = 0; q < N; ++q) {
        const int k = r * N + q;
        const double Am = Tp(i, tA + k), Ap = Tp(i + 1, tA + k);
        const double Jp = Tp(i, tJ + k), Jn = Tp(i + 2, tJ + k);
        double phi = 0.;
        if (r == 1 && q == 0) phi = grav;
        if (r == 2 && q == 1) phi = grav;
        a[r][q] = (Am * Aa + Ap * Aa) * hiv - phi;
        bb[r][q] = -(Am + Jp) * Aa * hiv;
        c[r][q] = -(Ap - Jn) * Aa * hiv;
      }
#pragma unroll
    for (int r = 0; r < N; ++r) a[r][r] += idt;
    if (i == 0) {
#pragma unroll
      for (int r = 0; r < N; ++r)
#pragma unroll
        for (int q = 0; q < N; ++q) a[r][q] += bb[r][q] * (q == 1 ? -1. : 1.);
    }
    if (i == nl - 1) {
#pragma unroll
      for (int r = 0; r < N; ++r)
#pragma unroll
        for (int q = 0; q < N; ++q) a[r][q] += c[r][q] * (q == 1 ? -1. : 1.);
    }
  };
  // (1) the system A delta = du / dt; sum (rho V)^2 and Q = sum g_out[IDN] rho (rho V)
  double sa2 = 0., qg = 0.;
  for (int i = tid; i < nl; i += nt) {
    double a[N][N], bb[N][N], c[N][N];
    blocks(i, a, bb, c);
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
      for (int q = 0; q < N; ++q) {
        Dg[i * 9 + r * 3 + q] = a[r][q];
        Bl[i * 9 + r * 3 + q] = i == 0 ? 0. : bb[r][q];
        Ab[i * 9 + r * 3 + q] = i == nl - 1 ? 0. : c[r][q];
      }
#pragma unroll
    for (int r = 0; r < N; ++r) R[i * 3 + r] = Tp(i, tDU + r) / dt;
    const double rho = Tp(i, tRHO), ai = rho * V;
    sa2 += ai * ai;
    qg += Tp(i, tG) * rho * ai;
  }
  cta_sum2(sa2, qg, red);  // (its barrier also completes the system)
  const double gb = qg / sa2;
  block_cr3_solve(Bl, Dg, Ab, R, nl);
  // (2) delta and B_dry; then the transposed system: row i of A^T couples
  // x_{i-1} by c_{i-1}^T and x_{i+1} by b_{i+1}^T
  double bdry = 0., unused = 0.;
  for (int i = tid; i < nl; i += nt) {
#pragma unroll
    for (int r = 0; r < N; ++r) Sat(i, oD + r) = R[i * 3 + r];
    bdry += (Tp(i, tDU) - R[i * 3]) * 1. * V;
  }
  __syncthreads();  // R is read
  for (int i = tid; i < nl; i += nt) {
    double a[N][N], bb[N][N], c[N][N];
    blocks(i, a, bb, c);
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
      for (int q = 0; q < N; ++q) {
        Dg[i * 9 + r * 3 + q] = a[q][r];
        const int k = q * N + r;  // transposed
        // c_{i-1} = -(|A|_{face i} - J_{cell i}) A hiv, b_{i+1} = -(|A|_{face i+1} + J_{cell i}) A hiv
        Bl[i * 9 + r * 3 + q] = i == 0 ? 0. : -(Tp(i, tA + k) - Tp(i + 1, tJ + k)) * Aa * hiv;
        Ab[i * 9 + r * 3 + q] =
            i == nl - 1 ? 0. : -(Tp(i + 1, tA + k) + Tp(i + 1, tJ + k)) * Aa * hiv;
      }
#pragma unroll
    for (int r = 0; r < N; ++r) R[i * 3 + r] = Tp(i, tG + r);
    R[i * 3] += -V * gb + Tp(i, tGF);
  }
  cta_sum2(bdry, unused, red);  // (its barrier also completes the system)
  block_cr3_solve(Bl, Dg, Ab, R, nl);
  for (int i = tid; i < nl; i += nt) {
#pragma unroll
    for (int r = 0; r < N; ++r) Sat(i, oT + r) = R[i * 3 + r];
  }
  if (tid == 0) {
    Z[0] = bdry / sa2;
    Z[ncol] = -qg * bdry / (sa2 * sa2);
    Z[2 * ncol] = gb;
  }
}

// Per cell m in [-1, nl] of every interior column: the block-dependence
// contraction into GW, and (interior cells) the redistribution's density
// term, the scalar mass-fix term and the cotangent of the explicit du.
template <int N, int NS>
__global__ void __launch_bounds__(128) k_vadj_contract(Geo g, Phys p, AdjBufs b) {
  constexpr int E1 = VadjDims<N>::E1, ES = VadjDims<N>::ES;
  const int nl = g.nx1;
  const int64_t ncol = (int64_t)(g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  const int64_t col0 = (int64_t)blockIdx.x * kCTC;
  const int m0 = -1 + (int)blockIdx.y * kCTL;  // first cell of the tile
  const int64_t sv = g.sv;
  const double* S = b.vic + (int64_t)(nl + 2) * E1 * ncol;
  const double* Z = S + (int64_t)nl * ES * ncol;
  const int oD = 2 * N * N, oT = 2 * N * N + N;
  // t and delta of layers m0-1 .. m0+kCTL (slot = layer - (m0-1)), extended:
  // t = 0 outside [0, nl), delta mirrored (normal row negated) at -1 and nl
  __shared__ double td[2 * N][kCTC][kCTL + 3];
  __shared__ double zs[3][kCTC];
  const int tid = threadIdx.x;
  for (int idx = tid; idx < 2 * N * kCTC * (kCTL + 2); idx += blockDim.x) {
    int c = idx % kCTC, rest = idx / kCTC;
    int s = rest % (kCTL + 2), e = rest / (kCTL + 2);
    int64_t col = col0 + c;
    int layer = m0 - 1 + s;
    double x = 0.;
    if (col < ncol) {
      if (e < N) {  // delta
        int src = layer < 0 ? 0 : (layer >= nl ? nl - 1 : layer);
        if (layer >= -1 && layer <= nl) {
          x = S[((int64_t)src * ES + oD + e) * ncol + col];
          if ((layer == -1 || layer == nl) && e == 1) x = -x;
        }
      } else if (layer >= 0 && layer < nl) {  // t
        x = S[((int64_t)layer * ES + oT + (e - N)) * ncol + col];
      }
    }
    td[e][c][s] = x;
  }
  if (tid < 3 * kCTC) {
    int c = tid % kCTC, k = tid / kCTC;
    zs[k][c] = col0 + c < ncol ? Z[k * ncol + col0 + c] : 0.;
  }
  __syncthreads();
  const double gm1c = p.gammad - 1.;
  const double gm1f = 0.5 * (p.gammad + p.gammad) - 1.;
  const double Aa = g.A1, hiv = 0.5 / g.vol, V = g.vol, dt = *b.dt;
  const double coef = Aa * hiv;
  for (int idx = tid; idx < kCTC * kCTL; idx += blockDim.x) {
    int s = idx % kCTL, c = idx / kCTL;
    int64_t col = col0 + c;
    int m = m0 + s;
    if (col >= ncol || m > nl) continue;
    const int64_t cb = adj_column_base(g, col);
    const int64_t off = cb + m;
    // slots of layers m-1, m, m+1
    const int sm1 = s, s0 = s + 1, sp1 = s + 2;
    auto D_ = [&](int slot, int r) { return td[r][c][slot]; };
    auto T_ = [&](int slot, int r) { return td[N + r][c][slot]; };
    double wm[5], wc[5], wp[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      wc[v] = b.W[v * sv + off];
      wm[v] = m - 1 >= -1 ? b.W[v * sv + off - 1] : 0.;
      wp[v] = m + 1 <= nl ? b.W[v * sv + off + 1] : 0.;
    }
    double gw[5] = {0., 0., 0., 0., 0.};
    double y[N], x[N];
    // interface m (cells m-1, m): w_m is its right state
    if (m >= 0) {
#pragma unroll
      for (int r = 0; r < N; ++r) {
        y[r] = coef * (T_(sm1, r) - T_(s0, r));
        x[r] = D_(s0, r) - D_(sm1, r);
      }
      absA_bilinear_vjp<N>(gm1f, wm, wc, y, x, nullptr, gw);
    }
    // interface m+1 (cells m, m+1): w_m is its left state
    if (m + 1 <= nl) {
#pragma unroll
      for (int r = 0; r < N; ++r) {
        y[r] = coef * (T_(s0, r) - T_(sp1, r));
        x[r] = D_(sp1, r) - D_(s0, r);
      }
      absA_bilinear_vjp<N>(gm1f, wc, wp, y, x, gw, nullptr);
    }
    // flux Jacobian of cell m
#pragma unroll
    for (int r = 0; r < N; ++r) {
      y[r] = coef * (T_(sp1, r) - T_(sm1, r));
      x[r] = D_(s0, r);
    }
    jac_bilinear_vjp<N>(gm1c, wc, y, x, gw);
    if (m >= 0 && m < nl) {
      // redistribution: du_out[IDN] = delta_0 + rho (rho V) B / S
      double go = b.GD[IDN * sv + off];
      double rho = wc[IDN];
      gw[IDN] += go * 2. * rho * V * zs[0][c] + zs[1][c] * 2. * rho * V * V;
      // scalar mass fix: ds_n += fix * r_n, fix = delta_0 - du_e[IDN]
      double fix = D_(s0, 0) - b.D[IDN * sv + off];
      double gfix = 0.;
#pragma unroll
      for (int n = 0; n < NS; ++n) {
        double gds = b.GD[(5 + n) * sv + off];
        gfix += gds * b.R[n * sv + off];
        b.GW[(5 + n) * sv + off] += gds * fix;
      }
      // cotangent of the explicit du rows
      b.GD[IDN * sv + off] = T_(s0, 0) / dt + V * zs[2][c] - gfix;
#pragma unroll
      for (int r = 1; r < N; ++r) b.GD[sel<N>(r) * sv + off] = T_(s0, r) / dt;
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) b.GW[v * sv + off] += gw[v];
  }
}

// SNAPB_VADJ_SOLVE = "sweep" or "cr" forces the adjoint's column solver (the
// sweep, or cyclic reduction where it applies); by default cyclic reduction
// takes up to kVadjCrMaxCols columns of 3x3 blocks
static int vadj_solver_env() {
  const char* e = std::getenv("SNAPB_VADJ_SOLVE");
  if (!e) return 0;
  if (std::strcmp(e, "sweep") == 0) return 1;
  if (std::strcmp(e, "cr") == 0) return 2;
  return 0;
}

template <int N, int NS>
static cudaError_t launch_vic_adj_n(const Geo& g, const Phys& p, const AdjBufs& b,
                                    cudaStream_t st) {
  const int64_t ncol = (int64_t)(g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  const int nl = g.nx1;
  dim3 ga((unsigned)((ncol + kATC - 1) / kATC), (unsigned)((nl + 2 + kATL<N> - 1) / kATL<N>));
  k_vadj_assemble<N, NS><<<ga, 256, 0, st>>>(g, p, b);
  const size_t cr_smem = vadj_cr_smem_bytes(nl);
  const int forced = vadj_solver_env();
  const bool cr_fits = N == 3 && cr_smem <= 200 * 1024;
  if (cr_fits && (forced == 2 || (forced == 0 && ncol <= kVadjCrMaxCols))) {
    raise_smem_limit(k_vadj_cr3, 200 * 1024);  // once per kernel: the largest plan
    k_vadj_cr3<<<(unsigned)ncol, kVadjCrThreads, cr_smem, st>>>(g, p, b);
  } else {
    // the ring takes vadj_ring_bytes per thread: 32-thread CTAs
    const int bs = 32;
    raise_smem_limit(k_vadj_sweep<N>, vadj_ring_bytes<N>(bs));
    k_vadj_sweep<N><<<(unsigned)((ncol + bs - 1) / bs), bs, vadj_ring_bytes<N>(bs), st>>>(g, p,
                                                                                         b);
  }
  dim3 gc((unsigned)((ncol + kCTC - 1) / kCTC), (unsigned)((nl + 2 + kCTL - 1) / kCTL));
  k_vadj_contract<N, NS><<<gc, 128, 0, st>>>(g, p, b);
  return cudaGetLastError();
}

template <int NS>
static cudaError_t launch_vic_adj_ns(const Geo& g, const Phys& p, const AdjBufs& b,
                                     cudaStream_t st) {
  if (vic_n_adj(p) == 5) return launch_vic_adj_n<5, NS>(g, p, b, st);
  return launch_vic_adj_n<3, NS>(g, p, b, st);
}

// reverse of snapb_riemann's hydro solvers, one thread per face
__global__ void k_riemann_adj(int64_t n, int solver, int ivx, double gamma, const double* wl,
                              const double* wr, const double* gflx, double* gwl, double* gwr) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  double L[5], R[5], gF[5], gL[5] = {0., 0., 0., 0., 0.}, gR[5] = {0., 0., 0., 0., 0.};
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    L[v] = wl[v * n + t];
    R[v] = wr[v * n + t];
    gF[v] = gflx[v * n + t];
  }
  riemann_vjp_rev(solver, L, R, ivx, gamma, gF, gL, gR);
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    gwl[v * n + t] = gL[v];
    gwr[v * n + t] = gR[v];
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <int NS>
static cudaError_t launch_sweeps_adj_ns(const Geo& g, const Phys& p, const AdjBufs& b,
                                        cudaStream_t st) {
  const bool a1 = g.nc1 > 1, a2 = g.nc2 > 1, a3 = g.nc3 > 1;
  const int ni = g.iu - g.il + 1;
  for (int ax = 3; ax >= 2; --ax) {
    if ((ax == 3 && !a3) || (ax == 2 && !a2)) continue;
    ScopedTimer tm(SNAPB_K_ADJ_X23, st);
    int nax = ax == 2 ? g.nx2 : g.nx3;
    int no = ax == 2 ? (g.ku - g.kl + 1) : (g.ju - g.jl + 1);
    int64_t lines = (int64_t)ni * no;
    // enough (line, segment) pairs for ~4 waves of 148 SMs x 4 CTAs of 128
    int64_t want = 148LL * 4 * 128 * 4;
    int nseg = (int)std::min<int64_t>(std::max<int64_t>(1, want / std::max<int64_t>(lines, 1)),
                                      (nax + 1 + 7) / 8);
    int seglen = (nax + 1 + nseg - 1) / nseg;
    nseg = (nax + 1 + seglen - 1) / seglen;
    dim3 grid((unsigned)((lines + 127) / 128), (unsigned)nseg);
    if (ax == 2)
      k_march_adj<NS, 2><<<grid, 128, 0, st>>>(g, p, b, seglen);
    else
      k_march_adj<NS, 3><<<grid, 128, 0, st>>>(g, p, b, seglen);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  ScopedTimer tm(SNAPB_K_ADJ_X1, st);
  if (a1) {
    const int nv = 5 + NS;
    size_t per = (size_t)2 * nv * g.nc1 * sizeof(double);
    int C = (int)std::max<size_t>(1, (48 * 1024) / per);
    C = std::min(C, 8);
    size_t smem = per * C;
    raise_smem_limit(k_x1_adj<NS>, 200 * 1024);
    int64_t ncol = (int64_t)g.nc2 * g.nc3;
    k_x1_adj<NS><<<(unsigned)((ncol + C - 1) / C), 256, smem, st>>>(g, p, b, C);
  } else {
    k_cell_adj<NS><<<(unsigned)((g.sv + 255) / 256), 256, 0, st>>>(g, p, b);
  }
  return cudaGetLastError();
}

cudaError_t launch_sweeps_adj(const Geo& g, const Phys& p, const AdjBufs& b, cudaStream_t st) {
  switch (p.nscalar) {
    case 0: return launch_sweeps_adj_ns<0>(g, p, b, st);
    case 1: return launch_sweeps_adj_ns<1>(g, p, b, st);
    case 2: return launch_sweeps_adj_ns<2>(g, p, b, st);
    case 3: return launch_sweeps_adj_ns<3>(g, p, b, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_vic_adj(const Geo& g, const Phys& p, const AdjBufs& b, cudaStream_t st) {
  switch (p.nscalar) {
    case 0: return launch_vic_adj_ns<0>(g, p, b, st);
    case 1: return launch_vic_adj_ns<1>(g, p, b, st);
    case 2: return launch_vic_adj_ns<2>(g, p, b, st);
    case 3: return launch_vic_adj_ns<3>(g, p, b, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace snapb

// ---------------------------------------------------------------------------
// extern "C" entry points
// ---------------------------------------------------------------------------
using namespace snapb;

namespace {

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

struct AdjLayout {
  size_t W, R, D, GD, GW, VIC, total;
};

AdjLayout adj_layout(const snapb_hydro_config& c) {
  Geo g = make_geo(c);
  Phys p = make_phys(c);
  AdjLayout L;
  size_t sv = (size_t)g.sv * sizeof(double), o = 0;
  int nv = 5 + c.nscalar;
  L.W = o;
  o = al256(o + 5 * sv);
  L.R = o;
  o = al256(o + (size_t)c.nscalar * sv);
  L.D = o;
  o = al256(o + nv * sv);
  L.GD = o;
  o = al256(o + nv * sv);
  L.GW = o;
  o = al256(o + nv * sv);
  L.VIC = o;
  o = al256(o + vic_adj_scratch_bytes(g, p));
  L.total = o;
  return L;
}

const char* check_adjoint(const snapb_hydro_config* c) {
  if (const char* e = internal_check_config(c)) return e;
  if (c->nu_iso > 0. || c->kappa_iso > 0.) return "the adjoint does not cover diffusion";
  if (c->non_hydrostatic != 1.) return "the adjoint needs non_hydrostatic = 1";
  if (c->nghost > kMaxGhost) return "the adjoint supports nghost <= 8";
  const int n[3] = {c->nx1, c->nx2, c->nx3};
  for (int a = 0; a < 3; ++a)
    if (n[a] > 1 && (c->bc[2 * a] == SNAPB_BC_CUSTOM || c->bc[2 * a + 1] == SNAPB_BC_CUSTOM))
      return "the adjoint needs reflecting, periodic or outflow boundaries on active axes";
  return nullptr;
}

template <class P>
P* wsp(void* ws, size_t off) {
  return reinterpret_cast<P*>(static_cast<char*>(ws) + off);
}

int cuda_rc(cudaError_t e, const char* where) {
  if (e == cudaSuccess) return SNAPB_OK;
  return internal_fail(SNAPB_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

void axes(const Geo& g, const snapb_hydro_config& c, AxisAdj& a1, AxisAdj& a2, AxisAdj& a3) {
  a1 = make_axis(g.nc1, c.nghost, c.bc[0], c.bc[1]);
  a2 = make_axis(g.nc2, c.nghost, c.bc[2], c.bc[3]);
  a3 = make_axis(g.nc3, c.nghost, c.bc[4], c.bc[5]);
}

// recompute w (with the x1 ghost revision), r and, for the implicit solve,
// the explicit du of the stage input, then run the reverse kernels
int reverse_core(const snapb_hydro_config* c, const Geo& g, Phys p, const double* dt,
                 const double* u, const double* s, AdjBufs& ab, cudaStream_t st,
                 const char* who) {
  StageBufs b;
  std::memset(&b, 0, sizeof(b));
  b.dt = dt;
  b.u = const_cast<double*>(u);
  b.w = const_cast<double*>(ab.W);
  b.s = const_cast<double*>(s);
  b.R = const_cast<double*>(ab.R);
  b.D = const_cast<double*>(ab.D);
  b.write_du = 1;
  const bool a1 = g.nc1 > 1, a2 = g.nc2 > 1, a3 = g.nc3 > 1;
  const int last_axis = a3 ? 3 : (a2 ? 2 : 1);
  cudaError_t e;
  {
    ScopedTimer t(SNAPB_K_ADJ_RECOMPUTE, st);
    e = a1 ? launch_x1(g, p, b, last_axis == 1, st) : launch_c2p_only(g, p, b, st);
    if (e != cudaSuccess) return cuda_rc(e, who);
    if (p.implicit_scheme != 0) {
      if (a2 && (e = launch_march(2, g, p, b, !a1, last_axis == 2, st)) != cudaSuccess)
        return cuda_rc(e, who);
      if (a3 && (e = launch_march(3, g, p, b, !a1 && !a2, true, st)) != cudaSuccess)
        return cuda_rc(e, who);
    }
    e = cudaMemsetAsync(ab.GW, 0, (size_t)(5 + p.nscalar) * g.sv * sizeof(double), st);
    if (e != cudaSuccess) return cuda_rc(e, who);
  }
  if (p.implicit_scheme != 0) {
    ScopedTimer t(SNAPB_K_ADJ_VIC, st);
    if ((e = launch_vic_adj(g, p, ab, st)) != cudaSuccess) return cuda_rc(e, who);
  }
  if ((e = launch_sweeps_adj(g, p, ab, st)) != cudaSuccess) return cuda_rc(e, who);
  return SNAPB_OK;
}

}  // namespace

extern "C" {

size_t snapb_adjoint_workspace_size(const snapb_hydro_config* cfg) {
  if (check_adjoint(cfg)) return 0;
  return adj_layout(*cfg).total;
}

int snapb_stage_adjoint(const snapb_hydro_config* cfg, int stage, const double* dt,
                        const double* u, const double* s, const double* gu_out,
                        const double* gs_out, double* gu, double* gs, double* gu0, double* gs0,
                        void* workspace, size_t workspace_bytes, void* stream) {
  if (const char* e = check_adjoint(cfg))
    return internal_fail(SNAPB_ERR_ARG, std::string("stage_adjoint: ") + e);
  if (stage < 0 || stage > 2) return internal_fail(SNAPB_ERR_ARG, "stage_adjoint: stage in [0, 2]");
  if (!dt || !u || !gu_out || !gu || !gu0)
    return internal_fail(SNAPB_ERR_ARG, "stage_adjoint: null pointer");
  if (cfg->nscalar > 0 && (!s || !gs_out || !gs || !gs0))
    return internal_fail(SNAPB_ERR_ARG, "stage_adjoint: scalars need s, gs_out, gs and gs0");
  AdjLayout L = adj_layout(*cfg);
  if (!workspace || workspace_bytes < L.total)
    return internal_fail(SNAPB_ERR_WORKSPACE, "stage_adjoint: workspace smaller than " +
                                                  std::to_string(L.total) + " bytes");
  cudaStream_t st = (cudaStream_t)stream;
  Geo g = make_geo(*cfg);
  Phys p = make_phys(*cfg);
  AdjBufs ab;
  std::memset(&ab, 0, sizeof(ab));
  ab.dt = dt;
  ab.u = u;
  ab.s = s;
  ab.W = wsp<double>(workspace, L.W);
  ab.R = wsp<double>(workspace, L.R);
  ab.D = wsp<double>(workspace, L.D);
  ab.GD = wsp<double>(workspace, L.GD);
  ab.GW = wsp<double>(workspace, L.GW);
  ab.vic = wsp<double>(workspace, L.VIC);
  ab.gu = gu;
  ab.gs = gs;
  CombineArgs ca;
  ca.gu_out = gu_out;
  ca.gs_out = gs_out;
  ca.gu = gu;
  ca.gs = gs;
  ca.gu0 = gu0;
  ca.gs0 = gs0;
  ca.GD = ab.GD;
  rk3_weights(stage, ca.w0, ca.w1, ca.w2);
  ca.ns = cfg->nscalar;
  axes(g, *cfg, ca.a1, ca.a2, ca.a3);
  cudaError_t e;
  {
    ScopedTimer t(SNAPB_K_ADJ_COMBINE, st);
    k_adj_combine<<<(unsigned)((g.sv + 255) / 256), 256, 0, st>>>(g, ca);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return cuda_rc(e, "stage_adjoint combine");
  return reverse_core(cfg, g, p, dt, u, s, ab, st, "stage_adjoint");
}

int snapb_hydro_forward_adjoint(const snapb_hydro_config* cfg, const double* dt,
                                const double* u, const double* g_du, double* g_u,
                                void* workspace, size_t workspace_bytes, void* stream) {
  if (const char* e = check_adjoint(cfg))
    return internal_fail(SNAPB_ERR_ARG, std::string("hydro_forward_adjoint: ") + e);
  if (!dt || !u || !g_du || !g_u)
    return internal_fail(SNAPB_ERR_ARG, "hydro_forward_adjoint: null pointer");
  AdjLayout L = adj_layout(*cfg);
  if (!workspace || workspace_bytes < L.total)
    return internal_fail(SNAPB_ERR_WORKSPACE, "hydro_forward_adjoint: workspace smaller than " +
                                                  std::to_string(L.total) + " bytes");
  cudaStream_t st = (cudaStream_t)stream;
  Geo g = make_geo(*cfg);
  Phys p = make_phys(*cfg);
  p.nscalar = 0;
  AdjBufs ab;
  std::memset(&ab, 0, sizeof(ab));
  ab.dt = dt;
  ab.u = u;
  ab.W = wsp<double>(workspace, L.W);
  ab.R = wsp<double>(workspace, L.R);
  ab.D = wsp<double>(workspace, L.D);
  ab.GD = wsp<double>(workspace, L.GD);
  ab.GW = wsp<double>(workspace, L.GW);
  ab.vic = wsp<double>(workspace, L.VIC);
  ab.gu = g_u;
  cudaError_t e = cudaMemsetAsync(g_u, 0, (size_t)5 * g.sv * sizeof(double), st);
  if (e != cudaSuccess) return cuda_rc(e, "hydro_forward_adjoint clear");
  k_mask_interior<<<(unsigned)((g.sv + 255) / 256), 256, 0, st>>>(g, g_du, ab.GD, 5);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_rc(e, "hydro_forward_adjoint mask");
  return reverse_core(cfg, g, p, dt, u, nullptr, ab, st, "hydro_forward_adjoint");
}

int snapb_riemann_adjoint(const snapb_hydro_config* cfg, int solver, int dim, const double* wl,
                          const double* wr, const double* g_flx, double* g_wl, double* g_wr,
                          void* stream) {
  if (const char* e = internal_check_config(cfg))
    return internal_fail(SNAPB_ERR_ARG, std::string("riemann_adjoint: ") + e);
  if (dim < 1 || dim > 3 || !wl || !wr || !g_flx || !g_wl || !g_wr ||
      solver < SNAPB_RIEMANN_ROE || solver > SNAPB_RIEMANN_HLLC)
    return internal_fail(SNAPB_ERR_ARG, "riemann_adjoint: bad arguments (hydro solvers only)");
  Geo g = make_geo(*cfg);
  k_riemann_adj<<<(unsigned)((g.sv + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      g.sv, solver, IPR - dim, cfg->gammad, wl, wr, g_flx, g_wl, g_wr);
  return cuda_rc(cudaGetLastError(), "riemann_adjoint");
}

int snapb_bc_adjoint(const snapb_hydro_config* cfg, const double* g_in, double* g_out, int nv,
                     int kind, void* stream) {
  if (const char* e = internal_check_config(cfg))
    return internal_fail(SNAPB_ERR_ARG, std::string("bc_adjoint: ") + e);
  if (!g_in || !g_out || g_in == g_out || nv < 1 || kind < SNAPB_PRIMITIVE || kind > SNAPB_SCALAR)
    return internal_fail(SNAPB_ERR_ARG, "bc_adjoint: bad arguments (out-of-place only)");
  if (cfg->nghost > kMaxGhost) return internal_fail(SNAPB_ERR_ARG, "bc_adjoint: nghost <= 8");
  Geo g = make_geo(*cfg);
  AxisAdj a1, a2, a3;
  axes(g, *cfg, a1, a2, a3);
  k_bc_adjoint<<<(unsigned)((g.sv + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      g, g_in, g_out, nv, kind != SNAPB_SCALAR ? 1 : 0, a1, a2, a3);
  return cuda_rc(cudaGetLastError(), "bc_adjoint");
}

}  // extern "C"
