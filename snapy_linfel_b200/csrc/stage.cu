// stage.cu — the fused per-direction sweeps of one RK stage (FP64 plain form).
//
//   k_x1     one CTA per group of x1 columns (x1 is the contiguous, vertical
//            axis): U->W into shared memory, the isentropic x1 ghost revision,
//            W written back for the other sweeps, WENO/PLM reconstruction +
//            Riemann flux at every x1 face of the column in registers, and the
//            x1 flux difference per cell.  Interface states never touch HBM.
//   k_march  x2 / x3 sweeps: one thread per (x1 cell, other horizontal index)
//            marches along the sweep axis with a six-cell register window;
//            consecutive threads are consecutive x1 cells, so every load is
//            coalesced.  The last active direction finalises the cell:
//            du = -dt * div / V + gravity (+ diffusion) and either the RK
//            combination in place or du for the implicit solve.
//   k_diff   isotropic viscosity / heat-conduction flux differences.
//
// Reference path: HydroImpl::forward (src/hydro/hydro_forward.cpp:14-217),
// ReconstructImpl::forward (src/recon/reconstruct.cpp:75-154), the Riemann
// solvers (src/riemann/*_impl.h), divergence (src/coord/coordinate.cpp:352-396),
// gravity (src/forcing/const_gravity.cpp:26-45), hydrostatic revisions
// (src/hydro/hydro.cpp:217-269), ScalarImpl::forward (src/scalar/scalar.cpp:50-132).
#include <algorithm>

#include "kernels.cuh"

namespace snapb {

// du = -dt*div + forcing for one cell, then the RK combination (or du for the
// implicit solve).  d holds the flux-difference sums of the nvar hydro
// variables followed by the scalars; wc is the cell's primitive state.
template <int NS>
__device__ __forceinline__ void finalize_cell(const Geo& g, const Phys& p, const StageBufs& b,
                                              int64_t off, const double* d, const double* wc) {
  const int64_t sv = g.sv;
  const double dt = *b.dt;
  double du[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) du[v] = -dt * (d[v] / g.vol);
  if (p.grav1 != 0.) {
    du[IVX] += dt * wc[IDN] * p.grav1 * p.nh;
    du[IPR] += dt * wc[IDN] * wc[IVX] * p.grav1 * p.nh;
  }
  if (p.grav2 != 0.) {
    du[IVY] += dt * wc[IDN] * p.grav2;
    du[IPR] += dt * wc[IDN] * wc[IVY] * p.grav2;
  }
  if (p.grav3 != 0.) {
    du[IVZ] += dt * wc[IDN] * p.grav3;
    du[IPR] += dt * wc[IDN] * wc[IVZ] * p.grav3;
  }
  if (p.nu > 0. || p.kappa > 0.) {
#pragma unroll
    for (int v = 0; v < 5; ++v) du[v] -= dt * (b.DD[v * sv + off] / g.vol);
  }
  if (p.has_grav && p.nh < 1.) {
    double rg = b.RG[off];
    du[IVX] += dt * rg * (1. - p.nh);
    du[IPR] += dt * wc[IVX] * rg * (1. - p.nh);
  }
  double ds[NS > 0 ? NS : 1];
#pragma unroll
  for (int n = 0; n < NS; ++n) ds[n] = -dt * (d[5 + n] / g.vol);
  if (b.write_du) {
#pragma unroll
    for (int v = 0; v < 5; ++v) b.D[v * sv + off] = du[v];
#pragma unroll
    for (int n = 0; n < NS; ++n) b.D[(5 + n) * sv + off] = ds[n];
    return;
  }
  double unew_rho = 0.;
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    int64_t o = v * sv + off;
    double uo = b.u[o];
    double u0v;
    if (b.stage == 0) {
      u0v = uo;
      b.u0[o] = uo;
    } else {
      u0v = b.u0[o];
    }
    double un = b.wgt0 * u0v + b.wgt1 * uo + b.wgt2 * du[v];
    b.u[o] = un;
    if (v == IDN) unew_rho = un;
  }
#pragma unroll
  for (int n = 0; n < NS; ++n) {
    int64_t o = n * sv + off;
    double so = b.s[o];
    double s0v;
    if (b.stage == 0) {
      s0v = so;
      b.s0[o] = so;
    } else {
      s0v = b.s0[o];
    }
    double sn = b.wgt0 * s0v + b.wgt1 * so + b.wgt2 * ds[n];
    b.s[o] = sn;
    if (b.r) b.r[o] = sn / unew_rho;
  }
}

// ---------------------------------------------------------------------------
// x1 column kernel
// ---------------------------------------------------------------------------
size_t x1_smem_per_column(const Geo& g, int nvt) {
  // w + face fluxes per variable, plus left/right face pressures
  return (size_t)(2 * nvt + 2) * g.nc1 * sizeof(double);
}

int x1_columns_per_cta(const Geo& g, int nvt) {
  size_t per = x1_smem_per_column(g, nvt);
  int c = (int)std::max<size_t>(1, (96 * 1024) / per);
  return std::min(c, 16);
}

template <int NS>
__global__ void __launch_bounds__(256) k_x1(Geo g, Phys p, StageBufs b, int C, int last) {
  constexpr int NV = 5 + NS;
  extern __shared__ double sm[];
  const int nc1 = g.nc1;
  double* sw = sm;
  double* sf = sw + (size_t)C * NV * nc1;
  double* spl = sf + (size_t)C * NV * nc1;
  double* spr = spl + (size_t)C * nc1;
  const int64_t ncol = (int64_t)g.nc2 * g.nc3;
  const int64_t col0 = (int64_t)blockIdx.x * C;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int64_t sv = g.sv;
  const double gm1 = p.gammad - 1.;

  // (1) U -> W for every cell of the columns (ghosts included)
  for (int idx = tid; idx < C * nc1; idx += nt) {
    int c = idx / nc1, i = idx - c * nc1;
    int64_t col = col0 + c;
    if (col >= ncol) continue;
    int64_t off = col * nc1 + i;
    double uc[5], wc[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) uc[v] = b.u[v * sv + off];
    cons2prim_cell(uc, wc, gm1);
#pragma unroll
    for (int v = 0; v < 5; ++v) sw[(c * NV + v) * nc1 + i] = wc[v];
#pragma unroll
    for (int n = 0; n < NS; ++n) {
      double rr = b.s[n * sv + off] / uc[IDN];
      sw[(c * NV + 5 + n) * nc1 + i] = rr;
      b.R[n * sv + off] = rr;
    }
  }
  __syncthreads();

  // (2) isentropic extrapolation of p and rho into the x1 ghosts, one thread
  // per (column, end)
  if (p.grav1 != 0. && tid < 2 * C && col0 + (tid >> 1) < ncol) {
    const int c = tid >> 1, top = tid & 1;
    double* pp = sw + (c * NV + IPR) * nc1;
    double* rr = sw + (c * NV + IDN) * nc1;
    const double gamma = p.gammad;
    const double a = (gamma - 1.) / gamma, ig = 1. / gamma, ia = 1. / a;
    const double grav = -p.grav1, dz = g.dx1;
    const int e = top ? g.iu : g.il, dir = top ? 1 : -1;
    const double K = pp[e] / pow(rr[e], gamma);
    const double kg = pow(K, ig);
    for (int n = 0; n < g.ng; ++n) {
      double h = top ? pow(pp[e + dir * n], a) - a * grav * dz / kg
                     : pow(pp[e + dir * n], a) + a * grav * dz / kg;
      pp[e + dir * (n + 1)] = pow(h, ia);
      rr[e + dir * (n + 1)] = pow(pp[e + dir * (n + 1)] / K, ig);
    }
  }
  __syncthreads();

  // (3) W back to HBM for the x2/x3 sweeps, the implicit solve and the CFL
  for (int idx = tid; idx < C * nc1; idx += nt) {
    int c = idx / nc1, i = idx - c * nc1;
    int64_t col = col0 + c;
    if (col >= ncol) continue;
    int64_t off = col * nc1 + i;
#pragma unroll
    for (int v = 0; v < 5; ++v) b.w[v * sv + off] = sw[(c * NV + v) * nc1 + i];
  }

  // (4) x1 faces il .. iu+1 of interior columns
  const int nf = g.nx1 + 1;
  for (int idx = tid; idx < C * nf; idx += nt) {
    int c = idx / nf, f = g.il + (idx - c * nf);
    int64_t col = col0 + c;
    if (col >= ncol) continue;
    int j = umod(col, g.nc2), k = udiv(col, g.nc2);
    if (j < g.jl || j > g.ju || k < g.kl || k > g.ku) continue;
    const double* base = sw + (size_t)c * NV * nc1;
    double L[NV], R[NV], F[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double q[6];
#pragma unroll
      for (int t = 0; t < 6; ++t) q[t] = base[v * nc1 + min(max(f - 3 + t, 0), nc1 - 1)];
      if (v < 5) {
        int typ = (p.r1_shock || v == IDN) ? p.r1_type : interp2_of(p.r1_type);
        face_states(typ, p.r1_scale != 0, q, L[v], R[v]);
      } else {
        face_states(p.rs_type, p.rs_scale != 0, q, L[v], R[v]);
        L[v] = L[v] < 0. ? 0. : L[v];
        R[v] = R[v] < 0. ? 0. : R[v];
      }
    }
    if (p.grav1 != 0.) {
      if (f == g.il) {
        L[IPR] = R[IPR];
        L[IDN] = R[IDN];
      }
      if (f == g.iu + 1) {
        R[IPR] = L[IPR];
        R[IDN] = L[IDN];
      }
    }
    spl[c * nc1 + f] = L[IPR];
    spr[c * nc1 + f] = R[IPR];
    if (p.disable1) {
#pragma unroll
      for (int v = 0; v < 5; ++v) F[v] = 0.;
    } else {
      riemann_flux(p.riemann, L, R, IVX, p.gammad, F);
    }
#pragma unroll
    for (int n = 0; n < NS; ++n) F[5 + n] = F[IDN] > 0. ? F[IDN] * L[5 + n] : F[IDN] * R[5 + n];
#pragma unroll
    for (int v = 0; v < NV; ++v) sf[(c * NV + v) * nc1 + f] = F[v];
  }
  __syncthreads();

  // (5) flux difference per interior cell
  const bool need_rg = p.grav1 != 0. && p.has_grav && p.nh < 1.;
  for (int idx = tid; idx < C * g.nx1; idx += nt) {
    int c = idx / g.nx1, i = g.il + (idx - c * g.nx1);
    int64_t col = col0 + c;
    if (col >= ncol) continue;
    int j = umod(col, g.nc2), k = udiv(col, g.nc2);
    if (j < g.jl || j > g.ju || k < g.kl || k > g.ku) continue;
    int64_t off = col * nc1 + i;
    double d[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const double* fv = sf + (c * NV + v) * nc1;
      d[v] = g.A1 * fv[i + 1] - g.A1 * fv[i];
    }
    if (need_rg) b.RG[off] = (spl[c * nc1 + i + 1] - spr[c * nc1 + i]) / g.dx1;
    if (last) {
      double wc[5];
#pragma unroll
      for (int v = 0; v < 5; ++v) wc[v] = sw[(c * NV + v) * nc1 + i];
      finalize_cell<NS>(g, p, b, off, d, wc);
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) b.D[v * sv + off] = d[v];
    }
  }
}

// U -> W (and scalar mixing ratios) when x1 is inactive
template <int NS>
__global__ void k_c2p_r(Geo g, Phys p, StageBufs b) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.sv) return;
  double uc[5], wc[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) uc[v] = b.u[v * g.sv + t];
  cons2prim_cell(uc, wc, p.gammad - 1.);
#pragma unroll
  for (int v = 0; v < 5; ++v) b.w[v * g.sv + t] = wc[v];
#pragma unroll
  for (int n = 0; n < NS; ++n) b.R[n * g.sv + t] = b.s[n * g.sv + t] / uc[IDN];
}

// ---------------------------------------------------------------------------
// x2 / x3 marching sweeps
// ---------------------------------------------------------------------------
template <int NS, int AX>
__global__ void __launch_bounds__(128) k_march(Geo g, Phys p, StageBufs b, int seglen, int first,
                                               int last) {
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
  if (f0 > hi) return;
  const int f1 = min(f0 + seglen, hi + 1);
  const int64_t base = i + o * ost;
  const int64_t sv = g.sv;
  const int ivx = AX == 2 ? IVY : IVZ;
  const double A = AX == 2 ? g.A2 : g.A3;
  const int disabled = AX == 2 ? p.disable2 : p.disable3;

  const int ncax = AX == 2 ? g.nc2 : g.nc3;
  double q[NV][6];
  // window slots outside the array (only possible for stencils narrower than
  // the ghost width allows) are clamped; they never enter a narrower stencil
  auto load = [&](int cell, int slot) {
    cell = min(max(cell, 0), ncax - 1);
    int64_t off = base + cell * st;
#pragma unroll
    for (int v = 0; v < 5; ++v) q[v][slot] = b.w[v * sv + off];
#pragma unroll
    for (int n = 0; n < NS; ++n) q[5 + n][slot] = b.R[n * sv + off];
  };
#pragma unroll
  for (int t = 0; t < 5; ++t) load(f0 - 3 + t, t);

  double Fp[NV];
  for (int f = f0; f <= f1; ++f) {
    load(f + 2, 5);
    double L[NV], R[NV], F[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      if (v < 5) {
        int typ = (p.r23_shock || v == IDN) ? p.r23_type : interp2_of(p.r23_type);
        face_states(typ, p.r23_scale != 0, q[v], L[v], R[v]);
      } else {
        face_states(p.rs_type, p.rs_scale != 0, q[v], L[v], R[v]);
        L[v] = L[v] < 0. ? 0. : L[v];
        R[v] = R[v] < 0. ? 0. : R[v];
      }
    }
    if (disabled) {
#pragma unroll
      for (int v = 0; v < 5; ++v) F[v] = 0.;
    } else {
      riemann_flux(p.riemann, L, R, ivx, p.gammad, F);
    }
#pragma unroll
    for (int n = 0; n < NS; ++n) F[5 + n] = F[IDN] > 0. ? F[IDN] * L[5 + n] : F[IDN] * R[5 + n];
    if (f > f0) {
      const int64_t off = base + (int64_t)(f - 1) * st;
      double d[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        d[v] = A * F[v] - A * Fp[v];
        if (!first) d[v] = b.D[v * sv + off] + d[v];
      }
      if (last) {
        double wc[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) wc[v] = q[v][2];
        finalize_cell<NS>(g, p, b, off, d, wc);
      } else {
#pragma unroll
        for (int v = 0; v < NV; ++v) b.D[v * sv + off] = d[v];
      }
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      Fp[v] = F[v];
#pragma unroll
      for (int t = 0; t < 5; ++t) q[v][t] = q[v][t + 1];
    }
  }
}

// ---------------------------------------------------------------------------
// diffusion (src/forcing/diffusion.cpp:152-240), uniform Cartesian
// ---------------------------------------------------------------------------
__device__ __forceinline__ int64_t axis_stride(const Geo& g, int a) {
  return a == 0 ? (int64_t)1 : (a == 1 ? g.s2 : g.s3);
}
__device__ __forceinline__ double axis_dx(const Geo& g, int a) {
  return a == 0 ? g.dx1 : (a == 1 ? g.dx2 : g.dx3);
}
__device__ __forceinline__ bool axis_active(const Geo& g, int a) {
  return a == 0 ? g.nc1 > 1 : (a == 1 ? g.nc2 > 1 : g.nc3 > 1);
}

__device__ double div_vel(const Geo& g, const double* w, int64_t t) {
  double dv = 0.;
  for (int a = 0; a < 3; ++a) {
    if (!axis_active(g, a)) continue;
    int64_t s = axis_stride(g, a);
    const double* v = w + (IVX + a) * g.sv;
    dv += (v[t + s] - v[t - s]) / (2. * axis_dx(g, a));
  }
  return dv;
}

// viscous + conductive flux at the face between t - s_a and t
__device__ void diff_face(const Geo& g, const Phys& p, const double* w, int a, int64_t t,
                          double* F) {
  const int64_t sv = g.sv;
  const int64_t s = axis_stride(g, a);
  const double dxa = axis_dx(g, a);
  const double* rho = w + IDN * sv;
#pragma unroll
  for (int v = 0; v < 5; ++v) F[v] = 0.;
  double rho_face = 0.5 * (rho[t] + rho[t - s]);
  if (p.nu > 0.) {
    double div_face = 0.5 * (div_vel(g, w, t) + div_vel(g, w, t - s));
    const double* va = w + (IVX + a) * sv;
    for (int bb = 0; bb < 3; ++bb) {
      const double* vb = w + (IVX + bb) * sv;
      double stress = (vb[t] - vb[t - s]) / dxa;
      if (bb == a) {
        stress = 2. * stress - (2. / 3.) * div_face;
      } else if (axis_active(g, bb)) {
        int64_t sb = axis_stride(g, bb);
        double dxb = axis_dx(g, bb);
        double d0 = (va[t + sb] - va[t - sb]) / (2. * dxb);
        double d1 = (va[t - s + sb] - va[t - s - sb]) / (2. * dxb);
        stress += 0.5 * (d0 + d1);
      }
      double m = -p.nu * rho_face * stress;
      F[IVX + bb] = m;
      F[IPR] += 0.5 * (vb[t] + vb[t - s]) * m;
    }
  }
  if (p.kappa > 0.) {
    const double* pr = w + IPR * sv;
    double cv = p.rgas / (p.gammad - 1.);
    double T0 = pr[t] / (rho[t] * p.rgas), T1 = pr[t - s] / (rho[t - s] * p.rgas);
    F[IPR] -= p.kappa * (0.5 * (rho[t] * cv + rho[t - s] * cv)) * ((T0 - T1) / dxa);
  }
}

__global__ void k_diff(Geo g, Phys p, StageBufs b) {
  const int ni = g.iu - g.il + 1, nj = g.ju - g.jl + 1, nk = g.ku - g.kl + 1;
  int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (int64_t)ni * nj * nk) return;
  int i = g.il + umod(tid, ni);
  int j = g.jl + umod(udiv(tid, ni), nj);
  int k = g.kl + udiv(tid, (int64_t)ni * nj);
  int64_t t = (int64_t)k * g.s3 + (int64_t)j * g.s2 + i;
  double acc[5] = {0., 0., 0., 0., 0.};
  const double A[3] = {g.A1, g.A2, g.A3};
  for (int a = 0; a < 3; ++a) {
    if (!axis_active(g, a)) continue;
    double Fm[5], Fp[5];
    diff_face(g, p, b.w, a, t, Fm);
    diff_face(g, p, b.w, a, t + axis_stride(g, a), Fp);
#pragma unroll
    for (int v = 0; v < 5; ++v) acc[v] += A[a] * Fp[v] - A[a] * Fm[v];
  }
#pragma unroll
  for (int v = 0; v < 5; ++v) b.DD[v * g.sv + t] = acc[v];
}

// stand-alone finalisation when no march kernel runs last (1-D with diffusion)
template <int NS>
__global__ void k_finalize(Geo g, Phys p, StageBufs b) {
  constexpr int NV = 5 + NS;
  const int ni = g.iu - g.il + 1, nj = g.ju - g.jl + 1, nk = g.ku - g.kl + 1;
  int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (int64_t)ni * nj * nk) return;
  int i = g.il + umod(tid, ni);
  int j = g.jl + umod(udiv(tid, ni), nj);
  int k = g.kl + udiv(tid, (int64_t)ni * nj);
  int64_t off = (int64_t)k * g.s3 + (int64_t)j * g.s2 + i;
  double d[NV], wc[5];
#pragma unroll
  for (int v = 0; v < NV; ++v) d[v] = b.D[v * g.sv + off];
#pragma unroll
  for (int v = 0; v < 5; ++v) wc[v] = b.w[v * g.sv + off];
  finalize_cell<NS>(g, p, b, off, d, wc);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
cudaError_t launch_finalize(const Geo& g, const Phys& p, const StageBufs& b, cudaStream_t st) {
  int64_t n = (int64_t)(g.iu - g.il + 1) * (g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  unsigned grid = (unsigned)((n + 127) / 128);
  switch (p.nscalar) {
    case 0: k_finalize<0><<<grid, 128, 0, st>>>(g, p, b); break;
    case 1: k_finalize<1><<<grid, 128, 0, st>>>(g, p, b); break;
    case 2: k_finalize<2><<<grid, 128, 0, st>>>(g, p, b); break;
    case 3: k_finalize<3><<<grid, 128, 0, st>>>(g, p, b); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <int NS>
static cudaError_t launch_x1_t(const Geo& g, const Phys& p, const StageBufs& b, bool last,
                               cudaStream_t st) {
  const int nvt = 5 + NS;
  int C = x1_columns_per_cta(g, nvt);
  size_t smem = (size_t)C * x1_smem_per_column(g, nvt);
  if (smem > 200 * 1024) return cudaErrorInvalidConfiguration;
  raise_smem_limit(k_x1<NS>, 200 * 1024);
  int64_t ncol = (int64_t)g.nc2 * g.nc3;
  int64_t grid = (ncol + C - 1) / C;
  k_x1<NS><<<(unsigned)grid, 256, smem, st>>>(g, p, b, C, last ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_x1(const Geo& g, const Phys& p, const StageBufs& b, bool last,
                      cudaStream_t st) {
  switch (p.nscalar) {
    case 0: return launch_x1_t<0>(g, p, b, last, st);
    case 1: return launch_x1_t<1>(g, p, b, last, st);
    case 2: return launch_x1_t<2>(g, p, b, last, st);
    case 3: return launch_x1_t<3>(g, p, b, last, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_c2p_only(const Geo& g, const Phys& p, const StageBufs& b, cudaStream_t st) {
  unsigned grid = (unsigned)((g.sv + 255) / 256);
  switch (p.nscalar) {
    case 0: k_c2p_r<0><<<grid, 256, 0, st>>>(g, p, b); break;
    case 1: k_c2p_r<1><<<grid, 256, 0, st>>>(g, p, b); break;
    case 2: k_c2p_r<2><<<grid, 256, 0, st>>>(g, p, b); break;
    case 3: k_c2p_r<3><<<grid, 256, 0, st>>>(g, p, b); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <int NS, int AX>
static cudaError_t launch_march_t(const Geo& g, const Phys& p, const StageBufs& b, bool first,
                                  bool last, cudaStream_t st) {
  int ni = g.iu - g.il + 1;
  int no = AX == 2 ? g.ku - g.kl + 1 : g.ju - g.jl + 1;
  int n = AX == 2 ? g.nx2 : g.nx3;
  int seglen = 32;
  int64_t threads = (int64_t)ni * no;
  // keep at least ~4 waves of threads on 148 SMs: shorter segments for small grids
  while (seglen > 8 && threads * ((n + seglen - 1) / seglen) < 148LL * 1024 * 2) seglen /= 2;
  dim3 grid((unsigned)((threads + 127) / 128), (unsigned)((n + seglen - 1) / seglen));
  k_march<NS, AX><<<grid, 128, 0, st>>>(g, p, b, seglen, first ? 1 : 0, last ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_march(int axis, const Geo& g, const Phys& p, const StageBufs& b, bool first,
                         bool last, cudaStream_t st) {
#define SNAPB_MARCH(NS)                                                  \
  case NS:                                                               \
    return axis == 2 ? launch_march_t<NS, 2>(g, p, b, first, last, st)  \
                     : launch_march_t<NS, 3>(g, p, b, first, last, st);
  switch (p.nscalar) {
    SNAPB_MARCH(0)
    SNAPB_MARCH(1)
    SNAPB_MARCH(2)
    SNAPB_MARCH(3)
  }
#undef SNAPB_MARCH
  return cudaErrorInvalidValue;
}

cudaError_t launch_diffusion(const Geo& g, const Phys& p, const StageBufs& b, cudaStream_t st) {
  int64_t n = (int64_t)(g.iu - g.il + 1) * (g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  k_diff<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(g, p, b);
  return cudaGetLastError();
}

}  // namespace snapb
