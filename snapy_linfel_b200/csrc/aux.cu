// aux.cu — element-wise and reduction kernels around the sweeps: EOS,
// boundary fills, CFL limit, positivity check, and the operator-level
// reconstruct / Riemann entry points (one module call each).
#include <algorithm>
#include <cfloat>
#include <cstring>

#include "kernels.cuh"

namespace snapb {

// ---------------------------------------------------------------------------
// EOS (src/eos/ideal_gas.cpp:67-109)
// ---------------------------------------------------------------------------
__global__ void k_cons2prim(int64_t n, int64_t sv, double gm1, const double* u, double* w) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  double uc[5], wc[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) uc[v] = u[v * sv + t];
  cons2prim_cell(uc, wc, gm1);
#pragma unroll
  for (int v = 0; v < 5; ++v) w[v * sv + t] = wc[v];
}

__global__ void k_prim2cons(int64_t n, int64_t sv, double gm1, const double* w, double* u) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  double rho = w[IDN * sv + t];
  double v1 = w[IVX * sv + t], v2 = w[IVY * sv + t], v3 = w[IVZ * sv + t];
  double m1 = v1 * rho, m2 = v2 * rho, m3 = v3 * rho;
  u[IDN * sv + t] = rho;
  u[IVX * sv + t] = m1;
  u[IVY * sv + t] = m2;
  u[IVZ * sv + t] = m3;
  double ke = 0.5 * (v1 * m1 + v2 * m2 + v3 * m3);
  u[IPR * sv + t] = w[IPR * sv + t] / gm1 + ke;
}

cudaError_t launch_cons2prim(const Geo& g, const Phys& p, const double* u, double* w,
                             cudaStream_t st) {
  k_cons2prim<<<(unsigned)((g.sv + 255) / 256), 256, 0, st>>>(g.sv, g.sv, p.gammad - 1., u, w);
  return cudaGetLastError();
}

cudaError_t launch_prim2cons(const Geo& g, const Phys& p, const double* w, double* u,
                             cudaStream_t st) {
  k_prim2cons<<<(unsigned)((g.sv + 255) / 256), 256, 0, st>>>(g.sv, g.sv, p.gammad - 1., w, u);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Boundary fills (src/bc/bc_func.cpp:7-63), applied x1-inner, x1-outer, ...,
// x3-outer (src/mesh/meshblock.cpp:717-730).  Each fill copies from cells
// that are interior along its own axis, so the sequence composes per axis:
// the final value of a cell is var[m3(k)][m2(j)][m1(i)] times the sign flips
// of the reflecting axes it crossed.  One thread per cell of the ghost shell
// (bc_shell_cell enumerates exactly the ghost cells).
// ---------------------------------------------------------------------------
struct AxisBC {
  int n, ng, lo_type, hi_type;
};

__device__ __forceinline__ int bc_map(const AxisBC& a, int i, bool& flip) {
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

__global__ void k_bc(Geo g, AxisBC a1, AxisBC a2, AxisBC a3, double* var, int nv,
                     int flip_normals) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= bc_shell_slots(g)) return;
  const int nc1 = g.nc1, nc2 = g.nc2;
  const int64_t sv = g.sv;
  int i, j, k;
  const int64_t t = bc_shell_cell(g, s, i, j, k);
  bool f1, f2, f3;
  int si = bc_map(a1, i, f1), sj = bc_map(a2, j, f2), sk = bc_map(a3, k, f3);
  if (si == i && sj == j && sk == k) return;  // interior (or identity-mapped) cell
  int64_t src = ((int64_t)sk * nc2 + sj) * nc1 + si;
  // loads of a group of variables before its stores (a thread's source cell
  // is never its target; the compiler cannot see that the stores miss it)
  constexpr int kGroup = 8;
  for (int v0 = 0; v0 < nv; v0 += kGroup) {
    double xs[kGroup];
#pragma unroll
    for (int q = 0; q < kGroup; ++q)
      if (v0 + q < nv) xs[q] = var[(v0 + q) * sv + src];
#pragma unroll
    for (int q = 0; q < kGroup; ++q) {
      const int v = v0 + q;
      if (v >= nv) break;
      double x = xs[q];
      if (flip_normals) {
        if ((v == IVX && f1) || (v == IVY && f2) || (v == IVZ && f3)) x = -x;
      }
      var[v * sv + t] = x;
    }
  }
}

cudaError_t launch_bc(const Geo& g, const snapb_hydro_config& c, double* var, int nv, int kind,
                      cudaStream_t st) {
  AxisBC a1{g.nc1, g.ng, c.bc[0], c.bc[1]};
  AxisBC a2{g.nc2, g.ng, c.bc[2], c.bc[3]};
  AxisBC a3{g.nc3, g.ng, c.bc[4], c.bc[5]};
  int flip = (kind == SNAPB_CONSERVED || kind == SNAPB_PRIMITIVE) ? 1 : 0;
  const int64_t n = bc_shell_slots_host(g);
  if (n == 0) return cudaSuccess;
  k_bc<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, a1, a2, a3, var, nv, flip);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// CFL limit (src/hydro/hydro.cpp:118-180).  slots[0..2] receive the per-axis
// minima as ordered 64-bit patterns (all candidates are positive doubles).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_min(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x = fmin(x, __shfl_xor_sync(0xffffffffu, x, o));
  return x;
}

__global__ void k_cfl(Geo g, double gammad, int use1, int use2, int use3, const double* w,
                      unsigned long long* slots) {
  const int ni = g.iu - g.il + 1, nj = g.ju - g.jl + 1, nk = g.ku - g.kl + 1;
  const int64_t n = (int64_t)ni * nj * nk;
  double m1 = DBL_MAX, m2 = DBL_MAX, m3 = DBL_MAX;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    int i = g.il + umod(t, ni);
    int j = g.jl + umod(udiv(t, ni), nj);
    int k = g.kl + udiv(t, (int64_t)ni * nj);
    int64_t o = (int64_t)k * g.s3 + (int64_t)j * g.s2 + i;
    double rho = w[IDN * g.sv + o], pr = w[IPR * g.sv + o];
    double cs = sqrt(gammad * pr / rho);
    if (use1) m1 = fmin(m1, g.dx1 / (fabs(w[IVX * g.sv + o]) + cs));
    if (use2) m2 = fmin(m2, g.dx2 / (fabs(w[IVY * g.sv + o]) + cs));
    if (use3) m3 = fmin(m3, g.dx3 / (fabs(w[IVZ * g.sv + o]) + cs));
  }
  __shared__ double red[3][32];
  m1 = warp_min(m1);
  m2 = warp_min(m2);
  m3 = warp_min(m3);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][wid] = m1;
    red[1][wid] = m2;
    red[2][wid] = m3;
  }
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    m1 = lane < nw ? red[0][lane] : DBL_MAX;
    m2 = lane < nw ? red[1][lane] : DBL_MAX;
    m3 = lane < nw ? red[2][lane] : DBL_MAX;
    m1 = warp_min(m1);
    m2 = warp_min(m2);
    m3 = warp_min(m3);
    if (lane == 0) {
      atomicMin(&slots[0], (unsigned long long)__double_as_longlong(m1));
      atomicMin(&slots[1], (unsigned long long)__double_as_longlong(m2));
      atomicMin(&slots[2], (unsigned long long)__double_as_longlong(m3));
    }
  }
}

__global__ void k_cfl_final(const unsigned long long* slots, int use1, int use2, int use3,
                            double dt_diff, double* dt_out) {
  double d1 = use1 ? __longlong_as_double((long long)slots[0]) : 1.e9;
  double d2 = use2 ? __longlong_as_double((long long)slots[1]) : 1.e9;
  double d3 = use3 ? __longlong_as_double((long long)slots[2]) : 1.e9;
  double dt = fmin(d1, fmin(d2, d3));
  if (dt_diff > 0.) dt = fmin(dt, dt_diff);
  *dt_out = dt;
}

__global__ void k_fill_ull(unsigned long long* p, int n, unsigned long long v) {
  if ((int)threadIdx.x < n) p[threadIdx.x] = v;
}

cudaError_t launch_cfl(const Geo& g, const Phys& p, const double* w, double* slots,
                       double* dt_out, cudaStream_t st) {
  int scheme = p.implicit_scheme;
  int use1 = g.nc1 > 1, use2 = g.nc2 > 1, use3 = g.nc3 > 1;
  if (scheme != 0) {
    use1 = use1 && (!(scheme & 1) || (g.nc3 == 1 && g.nc2 == 1));
    use2 = use2 && !((scheme >> 1) & 1);
    use3 = use3 && !((scheme >> 2) & 1);
  }
  double dt_diff = -1.;
  double coeff = fmax(p.nu, p.kappa);
  if (coeff > 0.) {
    int ndim = 0;
    double dxm = DBL_MAX;
    if (g.nc1 > 1) ++ndim, dxm = fmin(dxm, g.dx1);
    if (g.nc2 > 1) ++ndim, dxm = fmin(dxm, g.dx2);
    if (g.nc3 > 1) ++ndim, dxm = fmin(dxm, g.dx3);
    if (ndim > 0) dt_diff = dxm * dxm / (2. * ndim * coeff);
  }
  auto* sl = reinterpret_cast<unsigned long long*>(slots);
  double big = DBL_MAX;
  unsigned long long big_bits;
  std::memcpy(&big_bits, &big, sizeof(big));
  k_fill_ull<<<1, 32, 0, st>>>(sl, 3, big_bits);
  int64_t n = (int64_t)(g.iu - g.il + 1) * (g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
  k_cfl<<<blocks, 256, 0, st>>>(g, p.gammad, use1, use2, use3, w, sl);
  k_cfl_final<<<1, 1, 0, st>>>(sl, use1, use2, use3, dt_diff, dt_out);
  return cudaGetLastError();
}

cudaError_t launch_cfl_final(const Geo& g, const Phys& p, unsigned long long* slots,
                             double* dt_out, cudaStream_t st) {
  int scheme = p.implicit_scheme;
  int use1 = g.nc1 > 1, use2 = g.nc2 > 1, use3 = g.nc3 > 1;
  if (scheme != 0) {
    use1 = use1 && (!(scheme & 1) || (g.nc3 == 1 && g.nc2 == 1));
    use2 = use2 && !((scheme >> 1) & 1);
    use3 = use3 && !((scheme >> 2) & 1);
  }
  double dt_diff = -1.;
  double coeff = fmax(p.nu, p.kappa);
  if (coeff > 0.) {
    int ndim = 0;
    double dxm = DBL_MAX;
    if (g.nc1 > 1) ++ndim, dxm = fmin(dxm, g.dx1);
    if (g.nc2 > 1) ++ndim, dxm = fmin(dxm, g.dx2);
    if (g.nc3 > 1) ++ndim, dxm = fmin(dxm, g.dx3);
    if (ndim > 0) dt_diff = dxm * dxm / (2. * ndim * coeff);
  }
  k_cfl_final<<<1, 1, 0, st>>>(slots, use1, use2, use3, dt_diff, dt_out);
  return cudaGetLastError();
}

__global__ void k_scale_dt(const double* in, double f, double* out) { *out = f * *in; }

cudaError_t launch_scale_dt(const double* dt_in, double cfl, int redo, double* dt_out,
                            cudaStream_t st) {
  // pow(2, -redo) * cfl * dt  (src/mesh/meshblock.cpp:527)
  double f = ldexp(1.0, -redo) * cfl;
  k_scale_dt<<<1, 1, 0, st>>>(dt_in, f, dt_out);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Positivity check (src/mesh/meshblock.cpp:974-1016):
// flags[0] density <= 0, flags[1] total energy <= 0, flags[2] pressure <= 0
// ---------------------------------------------------------------------------
__global__ void k_check(Geo g, double gm1, const double* u, int* flags) {
  const int ni = g.iu - g.il + 1, nj = g.ju - g.jl + 1, nk = g.ku - g.kl + 1;
  const int64_t n = (int64_t)ni * nj * nk;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    int i = g.il + umod(t, ni);
    int j = g.jl + umod(udiv(t, ni), nj);
    int k = g.kl + udiv(t, (int64_t)ni * nj);
    int64_t o = (int64_t)k * g.s3 + (int64_t)j * g.s2 + i;
    double uc[5], wc[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) uc[v] = u[v * g.sv + o];
    if (!(uc[IDN] > 0.)) atomicOr(&flags[0], 1);
    if (!(uc[IPR] > 0.)) atomicOr(&flags[1], 1);
    cons2prim_cell(uc, wc, gm1);
    if (!(wc[IPR] > 0.)) atomicOr(&flags[2], 1);
  }
}

__global__ void k_zero_int(int* p, int n) {
  if ((int)threadIdx.x < n) p[threadIdx.x] = 0;
}

cudaError_t launch_check_positive(const Geo& g, const Phys& p, const double* u, int* flags,
                                  cudaStream_t st) {
  k_zero_int<<<1, 32, 0, st>>>(flags, 3);
  int64_t n = (int64_t)(g.iu - g.il + 1) * (g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
  k_check<<<blocks, 256, 0, st>>>(g, p.gammad - 1., u, flags);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Operator level: ReconstructImpl::forward and RiemannSolverImpl::forward on
// whole arrays, with the reference's edge replication, for parity checks of
// the individual modules.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int stencil_radius(int type) {
  return type == SNAPB_RECON_DC ? 0
         : (type == SNAPB_RECON_WENO5 || type == SNAPB_RECON_CP5) ? 2
                                                                   : 1;
}

__global__ void k_reconstruct(Geo g, Phys p, int dim, int group, const double* w, int nv,
                              double* wlr) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.sv * nv) return;
  int v = udiv(t, g.sv);
  int64_t cell = t - (int64_t)v * g.sv;
  int i = umod(cell, g.nc1);
  int j = umod(udiv(cell, g.nc1), g.nc2);
  int k = udiv(cell, (int64_t)g.nc1 * g.nc2);
  int n, pos;
  int64_t st;
  if (dim == 3) n = g.nc1, pos = i, st = 1;
  else if (dim == 2) n = g.nc2, pos = j, st = g.s2;
  else n = g.nc3, pos = k, st = g.s3;
  int type, shock, scale;
  if (group == 1) type = p.rs_type, shock = 1, scale = p.rs_scale;
  else if (dim == 3) type = p.r1_type, shock = p.r1_shock, scale = p.r1_scale;
  else type = p.r23_type, shock = p.r23_shock, scale = p.r23_scale;
  if (group == 0 && !shock && v >= IVX && v <= IPR) type = interp2_of(type);
  int r = stencil_radius(type);
  int il = r + 1, iu = n - (r + 1);
  const double* line = w + (int64_t)v * g.sv + cell - (int64_t)pos * st;
  auto win = [&](int f, double* q) {  // six cells around face f, clamped
#pragma unroll
    for (int m = 0; m < 6; ++m) q[m] = line[(int64_t)min(max(f - 3 + m, 0), n - 1) * st];
  };
  double q[6], wl, wr;
  // wlr[IRT] slot pos: left face of cell o, o clamped to [il, iu]
  int o = min(max(pos, il), iu);
  if (type == SNAPB_RECON_DC) o = max(pos, il);
  win(o, q);
  face_states(type, scale != 0, q, wl, wr);
  double vr = wr;
  // wlr[ILT] slot pos: right face of cell o-1, o clamped to [il, iu] (dc: to n-1)
  o = min(max(pos, il), iu);
  if (type == SNAPB_RECON_DC) o = max(pos, il);
  win(o, q);
  face_states(type, scale != 0, q, wl, wr);
  double vl = wl;
  if (group == 1) {
    vl = vl < 0. ? 0. : vl;
    vr = vr < 0. ? 0. : vr;
  }
  wlr[t] = vl;                    // ILT
  wlr[(int64_t)nv * g.sv + t] = vr;  // IRT
}

cudaError_t launch_reconstruct(const Geo& g, const Phys& p, int dim, int group, const double* w,
                               int nv, double* wlr, cudaStream_t st) {
  int64_t n = g.sv * nv;
  k_reconstruct<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, p, dim, group, w, nv, wlr);
  return cudaGetLastError();
}

__global__ void k_riemann(int64_t sv, int solver, int ivx, double gamma, const double* wl,
                          const double* wr, int nv, double* flx, double* fp, const double* vel) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= sv) return;
  if (solver == SNAPB_RIEMANN_UPWIND) {
    double ve = vel[t];
    for (int v = 0; v < nv; ++v)
      flx[v * sv + t] = ve > 0. ? ve * wl[v * sv + t] : ve * wr[v * sv + t];
    return;
  }
  double L[5], R[5], F[5], P;
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    L[v] = wl[v * sv + t];
    R[v] = wr[v * sv + t];
  }
  riemann_flux(solver, L, R, ivx, gamma, F, &P);
#pragma unroll
  for (int v = 0; v < 5; ++v) flx[v * sv + t] = F[v];
  if (fp) fp[t] = P;
}

cudaError_t launch_riemann(const Geo& g, const Phys& p, int solver, int dim, const double* wl,
                           const double* wr, int nv, double* flx, double* fp, const double* vel,
                           cudaStream_t st) {
  int ivx = IPR - dim;
  k_riemann<<<(unsigned)((g.sv + 255) / 256), 256, 0, st>>>(g.sv, solver, ivx, p.gammad, wl, wr,
                                                           nv, flx, fp, vel);
  return cudaGetLastError();
}

}  // namespace snapb
