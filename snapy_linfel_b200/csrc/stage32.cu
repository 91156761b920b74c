// stage32.cu — one RK stage in the FP32 perturbation form.
//
// State: u' = u - (rho_bar, 0, 0, 0, p_bar/(gamma-1)) in FP32 over an FP64
// reference profile rho_bar(x1), p_bar(x1) (x1 = vertical).  The sweeps are
// the same fused kernels as the FP64 form (stage.cu) in FP32 arithmetic, with
// three places where FP64 stays:
//   * the reference tables (k_ref32): x1 face reference pressures pf, the
//     offsets of each side's reconstructed reference pressure from pf, and
//     the residual of the reference x1 momentum balance
//     rbar_i = -(A1 pf_{i+1} - A1 pf_i)/V + rho_bar_i g1, formed in FP64 and
//     stored after the cancellation;
//   * the isentropic x1 ghost revision (pow of full values) in FP64;
//   * the implicit column solve (vic.cu, FP64 elimination on full states).
// The momentum fluxes carry the pressure as p' = p - pf (pert.cuh), so the
// large hydrostatic pressure never enters an FP32 difference.
#include <algorithm>
#include <type_traits>

#include "kernels.cuh"
#include "bulk.cuh"
#include "pert.cuh"

namespace snapb {

// ---------------------------------------------------------------------------
// reference tables
// ---------------------------------------------------------------------------
__global__ void k_ref32(Geo g, Phys p, const double* rb_in, const double* pb_in, double* rbw,
                        double* pbw, StageBufs32 b) {
  const int nc1 = g.nc1;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t <= nc1) {
    // reference pressure at face t from each side, with the x1 pressure
    // interpolation (linear: cp5 / cp3 / dc)
    int typ = (p.r1_shock) ? p.r1_type : interp2_of(p.r1_type);
    double q[6];
    for (int m = 0; m < 6; ++m) {
      int c = min(max(t - 3 + m, 0), nc1 - 1);
      q[m] = pb_in ? pb_in[c] : 0.;
    }
    double pl, pr;
    face_states<double>(typ, false, q, pl, pr);
    if (typ != SNAPB_RECON_CP5 && typ != SNAPB_RECON_CP3 && typ != SNAPB_RECON_DC) {
      pl = pr = q[2];  // non-linear pressure interpolation: only with a zero reference
    }
    double pfv = 0.5 * (pl + pr);
    b.pf[t] = pfv;
    b.offL[t] = (float)(pl - pfv);
    b.offR[t] = (float)(pr - pfv);
  }
  if (t < nc1) {
    double r = rb_in ? rb_in[t] : 0.;
    double pr = pb_in ? pb_in[t] : 0.;
    rbw[t] = r;
    pbw[t] = pr;
    b.rbf[t] = (float)r;
    b.pbf[t] = (float)pr;
  }
}

// second pass: the x1 momentum residual needs pf on both faces of a cell
__global__ void k_ref32_residual(Geo g, Phys p, StageBufs32 b) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.nc1) return;
  double res = 0.;
  if (i + 1 <= g.nc1) res = -(g.A1 * b.pf[i + 1] - g.A1 * b.pf[i]) / g.vol;
  res += b.rb[i] * p.grav1;
  b.rbar[i] = (float)res;
}

// ---------------------------------------------------------------------------
// finalize: du' = -dt div'/V + gravity (with the FP64 reference residual),
// then RK on u' or du for the implicit solve
// ---------------------------------------------------------------------------
template <int NS>
__device__ __forceinline__ void finalize32(const Geo& g, const Phys& p, const StageBufs32& b,
                                           int64_t off, int xi, const float* d, const float* wc) {
  const int64_t sv = g.sv;
  const float dt = (float)*b.dt;
  const float ivol = (float)(1.0 / g.vol);
  float rho = b.rbf[xi] + wc[IDN];
  float du[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) du[v] = -dt * (d[v] * ivol);
  if (g.nc1 > 1) du[IVX] += dt * b.rbar[xi];  // reference pressure gradient + rho_bar g1
  if (p.grav1 != 0.) {
    du[IVX] += dt * wc[IDN] * (float)p.grav1;
    du[IPR] += dt * rho * wc[IVX] * (float)p.grav1;
  }
  if (p.grav2 != 0.) {
    du[IVY] += dt * rho * (float)p.grav2;
    du[IPR] += dt * rho * wc[IVY] * (float)p.grav2;
  }
  if (p.grav3 != 0.) {
    du[IVZ] += dt * rho * (float)p.grav3;
    du[IPR] += dt * rho * wc[IVZ] * (float)p.grav3;
  }
  float ds[NS > 0 ? NS : 1];
#pragma unroll
  for (int n = 0; n < NS; ++n) ds[n] = -dt * (d[5 + n] * ivol);
  if (b.write_du) {
#pragma unroll
    for (int v = 0; v < 5; ++v) b.D[v * sv + off] = du[v];
#pragma unroll
    for (int n = 0; n < NS; ++n) b.D[(5 + n) * sv + off] = ds[n];
    return;
  }
  const float w0 = (float)b.wgt0, w1 = (float)b.wgt1, w2 = (float)b.wgt2;
  float unew_rho = 0.f;
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    int64_t o = v * sv + off;
    float uo = b.u[o];
    float u0v;
    if (b.stage == 0) {
      u0v = uo;
      b.u0[o] = uo;
    } else {
      u0v = b.u0[o];
    }
    float un = w0 * u0v + w1 * uo + w2 * du[v];
    b.u[o] = un;
    if (v == IDN) unew_rho = b.rbf[xi] + un;
  }
#pragma unroll
  for (int n = 0; n < NS; ++n) {
    int64_t o = n * sv + off;
    float so = b.s[o];
    float s0v;
    if (b.stage == 0) {
      s0v = so;
      b.s0[o] = so;
    } else {
      s0v = b.s0[o];
    }
    float sn = w0 * s0v + w1 * so + w2 * ds[n];
    b.s[o] = sn;
    if (b.r) b.r[o] = sn / unew_rho;
  }
}

// U' -> W' of one cell at x1 index xi (p' = (gamma-1)(E' - KE): no
// reference-sized cancellation)
__device__ __forceinline__ void cons2prim_pert(const float* u, float* w, float rbar, float gm1) {
  float rho = rbar + u[IDN];
  float ir = fdiv(1.f, rho);
  w[IDN] = u[IDN];
  w[IVX] = u[IVX] * ir;
  w[IVY] = u[IVY] * ir;
  w[IVZ] = u[IVZ] * ir;
  float ke = 0.5f * (w[IVX] * u[IVX] + w[IVY] * u[IVY] + w[IVZ] * u[IVZ]);
  w[IPR] = gm1 * (u[IPR] - ke);
}

// ---------------------------------------------------------------------------
// x1 column kernel
// ---------------------------------------------------------------------------
// One warp per x1 column, C columns per tile (CTA of 32 C threads).  Shared
// memory of a tile: W' rows [C][NV][nc1], the full density row [C][nc1]
// (rho_bar + rho', the reconstructed density), then the staging planes of the
// tile's U' and scalar slabs, [NV][ps] with ps >= C nc1 + 3, 16-byte aligned.
size_t x1_smem32_per_column(const Geo& g, int nvt) {
  return (size_t)(2 * nvt + 1) * g.nc1 * sizeof(float);
}
// The layout follows the longest column of the launch (nc1max): a batched
// launch stages the next tile, possibly of another member, while the current
// one's rows are read, so the staging planes start after the rows of any tile.
struct X1Smem {
  int64_t fo, ps;  // float offset of the staging planes, plane stride
  __host__ __device__ X1Smem(int nc1max, int nvt, int C) {
    fo = (((int64_t)C * (nvt + 1) * nc1max) + 3) & ~(int64_t)3;
    ps = ((int64_t)C * nc1max + 3 + 3) & ~(int64_t)3;
  }
  __host__ __device__ size_t bytes(int nvt) const {
    return (size_t)(fo + ps * nvt) * sizeof(float);
  }
};
size_t x1_smem32_bytes(int nc1max, int nvt, int C) { return X1Smem(nc1max, nvt, C).bytes(nvt); }

// set by a CTA of the x1 sweep whose bulk copy did not complete in time
__device__ int snapb_x1_bulk_timeout = 0;

// Isentropic x1 ghost revision on full values, in FP64, written into W' of the
// ghost cells (density and pressure rows).  The recurrence
// p_{n+1} = (p_n^a + c)^(1/a) has h_n = p_n^a = p_e^a + n c, so every ghost
// level is independent: one slot per (column, end, level), all columns of the
// block (ghost columns included), slot = (col * 2 + top) * ng + n.  The x1
// sweep reads these W' values for its ghost cells and leaves them in place.
__device__ __forceinline__ void x1_ghost_revision32(const Geo& g, const Phys& p,
                                                    const StageBufs32& b, int64_t slot) {
  const int ng = g.ng;
  const int64_t col = slot / (2 * ng);
  const int rest = (int)(slot - col * 2 * ng);
  const int top = rest / ng, n = rest - top * ng;
  const int64_t sv = g.sv, cb = col * g.nc1;  // (k, j, 0) offset: s2 = nc1
  const int e = top ? g.iu : g.il, dir = top ? 1 : -1;
  float ue[5], we[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) ue[v] = b.u[v * sv + cb + e];
  cons2prim_pert(ue, we, b.rbf[e], (float)(p.gammad - 1.));
  const double gam = p.gammad;
  const double a = (gam - 1.) / gam, ig = 1. / gam, ia = 1. / a;
  const double grav = -p.grav1, dz = g.dx1;
  const double ps = b.pb[e] + we[IPR], rs = b.rb[e] + we[IDN];
  const double K = ps / pow(rs, gam), kg = pow(K, ig);
  const double step = (top ? -a : a) * grav * dz / kg;
  const double h = pow(ps, a) + (n + 1) * step;
  const double pn = pow(h, ia);
  const double rn = pow(pn / K, ig);
  const int cell = e + dir * (n + 1);  // ghosts only; the edge cell is never written
  b.w[IPR * sv + cb + cell] = (float)(pn - b.pb[cell]);
  b.w[IDN * sv + cb + cell] = (float)(rn - b.rb[cell]);
}

__global__ void __launch_bounds__(256) k_x1_ghost_revision32(Geo g, Phys p, StageBufs32 b) {
  const int64_t slot = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (slot < (int64_t)g.nc2 * g.nc3 * 2 * g.ng) x1_ghost_revision32(g, p, b, slot);
}

// (0) Warp 0 stages the U' and scalar slabs of columns col0 .. col0+C-1 (they
// are consecutive in every variable plane) into the staging planes: the
// aligned interiors by bulk copies completing on `bar`, the ragged ends by
// plain loads (visible after the next CTA barrier).
template <int NS>
__device__ __forceinline__ void x1_32_stage(const Geo& g, const StageBufs32& b, int C,
                                            int64_t col0, float* smf, int nc1max,
                                            uint64_t* bar) {
  constexpr int NV = 5 + NS;
  if (threadIdx.x >= 32) return;
  const X1Smem L(nc1max, NV, C);
  const int64_t ncol = (int64_t)g.nc2 * g.nc3;
  const int64_t nslab = std::min<int64_t>(C, ncol - col0) * g.nc1;
  auto plane = [&](int v) -> const float* {
    return (v < 5 ? b.u + v * g.sv : b.s + (v - 5) * g.sv) + col0 * g.nc1;
  };
  if (threadIdx.x == 0) {
    unsigned bytes = 0;
#pragma unroll
    for (int v = 0; v < NV; ++v) bytes += (unsigned)(bulk_split(plane(v), nslab).body * 4);
    fence_proxy_async_smem();  // earlier reads of the staging planes come first
    mbar_arrive_expect_tx(bar, bytes);
  }
  if (threadIdx.x < 8)
#pragma unroll
    for (int v = 0; v < NV; ++v)
      bulk_stage_slab(smf + L.fo + v * L.ps, plane(v), nslab, bar, threadIdx.x == 0);
}

// One tile after its staging completed, every thread of the CTA (one
// barrier): warp w works column col0 + w.
//   (1) U' -> W' of the column's cells from the staged slabs into shared
//       memory, with W' and the scalar mixing ratios stored; ghost cells take
//       density and pressure from the ghost revision (gravity along x1);
//   (2) the faces in rounds of 32 (face il + 32 k + lane): states and flux in
//       registers; the flux difference of cell f takes face f+1 from the next
//       lane (a shuffle), lane 31 that of the next round's lane 0 one round
//       later; then du or the RK combination (finalize32).
// The staging planes are free after (1): on return from x1_32_convert the
// caller may stage the next tile while x1_32_faces runs.
template <int NS>
__device__ __forceinline__ void x1_32_convert(const Geo& g, const Phys& p, const StageBufs32& b,
                                              int C, int64_t col0, float* smf, int nc1max) {
  constexpr int NV = 5 + NS;
  const int nc1 = g.nc1, ng = g.ng, il = g.il, iu = g.iu;
  const X1Smem L(nc1max, NV, C);
  float* sw = smf;                        // [C][NV][nc1]
  float* sr = sw + (size_t)C * NV * nc1;  // [C][nc1]
  const float* st = smf + L.fo;           // staging planes
  const int64_t ncol = (int64_t)g.nc2 * g.nc3;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, c = tid >> 5;
  const int lgC = __ffs(C) - 1;
  const int64_t sv = g.sv;
  const float gm1 = (float)(p.gammad - 1.);
  const bool revise = p.grav1 != 0.;
  int sbase[NV];  // float offset in the staging planes of each variable's element 0
#pragma unroll
  for (int v = 0; v < NV; ++v)
    sbase[v] = (int)(v * L.ps) +
               bulk_phase((v < 5 ? b.u + v * sv : b.s + (v - 5) * sv) + col0 * nc1);
  auto convert = [&](int cc, int i, bool ghost) {
    const int64_t off = (col0 + cc) * nc1 + i;
    const int e = cc * nc1 + i;
    float uc[5], wc[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) uc[v] = st[sbase[v] + e];
    cons2prim_pert(uc, wc, b.rbf[i], gm1);
    float* base = sw + (size_t)cc * NV * nc1;
    if (ghost && revise) {  // density and pressure from the ghost revision
      wc[IDN] = b.w[IDN * sv + off];
      wc[IPR] = b.w[IPR * sv + off];
#pragma unroll
      for (int v = IVX; v <= IVZ; ++v) b.w[v * sv + off] = wc[v];
    } else {
#pragma unroll
      for (int v = 0; v < 5; ++v) b.w[v * sv + off] = wc[v];
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) base[v * nc1 + i] = wc[v];
    sr[(size_t)cc * nc1 + i] = b.rbf[i] + wc[IDN];
#pragma unroll
    for (int n = 0; n < NS; ++n) {
      float rr = fdiv(st[sbase[5 + n] + e], b.rbf[i] + uc[IDN]);
      base[(5 + n) * nc1 + i] = rr;
      b.R[n * sv + off] = rr;
    }
  };
  if (col0 + c < ncol)
    for (int i = il + lane; i <= iu; i += 32) convert(c, i, false);
  for (int idx = tid; idx < 2 * ng * C; idx += nt) {  // ghost cells, 2 ng per column
    const int cc = idx & (C - 1), k = idx >> lgC;
    if (col0 + cc < ncol) convert(cc, k < ng ? k : iu + 1 + (k - ng), true);
  }
  __syncthreads();
}

template <int NS, int FP>
__device__ __forceinline__ void x1_32_faces(const Geo& g, const Phys& p, const StageBufs32& b,
                                            int C, int last, int64_t col0, const float* smf) {
  constexpr int NV = 5 + NS;
  const int nc1 = g.nc1, il = g.il, iu = g.iu;
  const int lane = threadIdx.x & 31, c = threadIdx.x >> 5;
  const int64_t ncol = (int64_t)g.nc2 * g.nc3;
  auto interior = [&](int cc) {
    const int64_t col = col0 + cc;
    if (col >= ncol) return false;
    const int j = umod(col, g.nc2), k = udiv(col, g.nc2);
    return j >= g.jl && j <= g.ju && k >= g.kl && k <= g.ku;
  };
  const int64_t sv = g.sv;
  const float gamma = (float)p.gammad;
  const bool revise = p.grav1 != 0.;
  const int ptype = (p.r1_shock) ? p.r1_type : interp2_of(p.r1_type);
  const float A1 = (float)g.A1;
  // face f of tile column cc; the stencil f-3 .. f+2 stays inside the column (ng >= 3)
  auto face = [&](int cc, int f, float* F) {
    const float* base = smf + (size_t)cc * NV * nc1 + f - 3;
    const float* rho = smf + (size_t)C * NV * nc1 + (size_t)cc * nc1 + f - 3;
    float L[NV], R[NV];
    float pl, pr;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      float q[6];
#pragma unroll
      for (int s6 = 0; s6 < 6; ++s6) q[s6] = v == IDN ? rho[s6] : base[v * nc1 + s6];
      if (v == IPR) {
        sweep_face_states<FP>(ptype, p.r1_scale != 0, v, q, pl, pr);
        pl += b.offL[f];
        pr += b.offR[f];
      } else if (v < 5) {
        int typ = (p.r1_shock || v == IDN) ? p.r1_type : interp2_of(p.r1_type);
        sweep_face_states<FP>(typ, p.r1_scale != 0, v, q, L[v], R[v]);
      } else {
        sweep_face_states<FP>(p.rs_type, p.rs_scale != 0, v, q, L[v], R[v]);
        L[v] = L[v] < 0.f ? 0.f : L[v];
        R[v] = R[v] < 0.f ? 0.f : R[v];
      }
    }
    if (revise) {
      if (f == il) {
        pl = pr;
        L[IDN] = R[IDN];
      }
      if (f == iu + 1) {
        pr = pl;
        R[IDN] = L[IDN];
      }
    }
    const float pfv = (float)b.pf[f];
    L[IPR] = pfv + pl;
    R[IPR] = pfv + pr;
    if (p.disable1) {
#pragma unroll
      for (int v = 0; v < 5; ++v) F[v] = 0.f;
    } else {
      sweep_riemann<FP>(p.riemann, L, R, pl, pr, pfv, IVX, gamma, F);
    }
#pragma unroll
    for (int n = 0; n < NS; ++n) F[5 + n] = F[IDN] > 0.f ? F[IDN] * L[5 + n] : F[IDN] * R[5 + n];
  };
  const float* wcol = smf + (size_t)c * NV * nc1;
  auto finish = [&](int i, const float* d) {
    const int64_t off = (col0 + c) * nc1 + i;
    if (last) {
      float wc[5];
#pragma unroll
      for (int v = 0; v < 5; ++v) wc[v] = wcol[v * nc1 + i];
      finalize32<NS>(g, p, b, off, i, d, wc);
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) b.D[v * sv + off] = d[v];
    }
  };
  // faces il .. iu+1 in rounds of 32 (face f0 + lane); the flux difference
  // of cell f takes face f+1 from the next lane, lane 31 that of the next
  // round's lane 0 one round later
  if (!interior(c)) return;  // the whole warp
  float Fkeep[NV];  // lane 31: its face of the previous round
#pragma unroll
  for (int v = 0; v < NV; ++v) Fkeep[v] = 0.f;
  for (int f0 = il; f0 <= iu + 1; f0 += 32) {
    const int f = f0 + lane;
    float F[NV];
    if (f <= iu + 1) {
      face(c, f, F);
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) F[v] = 0.f;
    }
    float Fn[NV];  // lanes 0 .. 30: face f + 1; lane 31: this round's first face
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const float dn = __shfl_down_sync(0xffffffffu, F[v], 1);
      const float f0v = __shfl_sync(0xffffffffu, F[v], 0);
      Fn[v] = lane < 31 ? dn : f0v;
    }
    // this lane's cell: f (lanes 0 .. 30), the previous round's last (lane 31)
    const int i = lane < 31 ? f : f0 - 1;
    if (i >= il && i <= iu) {
      float d[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) d[v] = A1 * Fn[v] - A1 * (lane < 31 ? F[v] : Fkeep[v]);
      finish(i, d);
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) Fkeep[v] = F[v];
  }
}

// one tile per CTA: stage, convert, faces
template <int NS, int FP>
__global__ void __launch_bounds__(512, 2) k_x1_32(Geo g, Phys p, StageBufs32 b, int C, int last) {
  extern __shared__ __align__(16) float smf[];
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  __syncthreads();
  const int64_t col0 = (int64_t)blockIdx.x * C;
  x1_32_stage<NS>(g, b, C, col0, smf, g.nc1, &bar);
  const bool ok = threadIdx.x >= 32 || mbar_wait(&bar, 0, &snapb_x1_bulk_timeout);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x < 32) mbar_wait(&bar, 0, &snapb_x1_bulk_timeout);  // copies in flight
    return;
  }
  x1_32_convert<NS>(g, p, b, C, col0, smf, g.nc1);
  x1_32_faces<NS, FP>(g, p, b, C, last, col0, smf);
}

// ---------------------------------------------------------------------------
// x2 / x3 marching sweeps (reference constant along the sweep)
// ---------------------------------------------------------------------------
// One thread's work: line tid (x1 cell x other horizontal index) and face
// segment seg of the sweep axis.
template <int NS, int AX, int FP>
__device__ __forceinline__ void march32_line(const Geo& g, const Phys& p, const StageBufs32& b,
                                             int seglen, int first, int last, int64_t tid,
                                             int seg) {
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
  if (tid >= (int64_t)ni * no) return;
  const int i = g.il + umod(tid, ni);
  const int o = olo + udiv(tid, ni);
  const int f0 = lo + seg * seglen;
  if (f0 > hi) return;
  const int f1 = min(f0 + seglen, hi + 1);
  const int64_t base = i + o * ost;
  const int64_t sv = g.sv;
  const int ivx = AX == 2 ? IVY : IVZ;
  const float A = (float)(AX == 2 ? g.A2 : g.A3);
  const int disabled = AX == 2 ? p.disable2 : p.disable3;
  const int ncax = AX == 2 ? g.nc2 : g.nc3;
  const float rref = b.rbf[i], pref = b.pbf[i];
  const float gamma = (float)p.gammad;

  // six-cell window of the face's stencil plus one cell loaded a face ahead
  // (slot 6), so a load's latency overlaps the previous face's arithmetic
  float q[NV][7];
  auto load = [&](int cell, int slot) {
    cell = min(max(cell, 0), ncax - 1);
    int64_t off = base + cell * st;
#pragma unroll
    for (int v = 0; v < 5; ++v) q[v][slot] = b.w[v * sv + off];
#pragma unroll
    for (int n = 0; n < NS; ++n) q[5 + n][slot] = b.R[n * sv + off];
  };
#pragma unroll
  for (int t = 0; t < 6; ++t) load(f0 - 3 + t, t);

  float Fp[NV];
  for (int f = f0; f <= f1; ++f) {
    load(f + 3, 6);
    // the running sums of the cell this face closes, fetched before the
    // face's arithmetic
    float dprev[NV];
    if (f > f0 && !first) {
      const int64_t off = base + (int64_t)(f - 1) * st;
#pragma unroll
      for (int v = 0; v < NV; ++v) dprev[v] = b.D[v * sv + off];
    }
    float L[NV], R[NV], F[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      if (v < 5) {
        int typ = (p.r23_shock || v == IDN) ? p.r23_type : interp2_of(p.r23_type);
        sweep_face_states<FP>(typ, p.r23_scale != 0, v, q[v], L[v], R[v]);
      } else {
        sweep_face_states<FP>(p.rs_type, p.rs_scale != 0, v, q[v], L[v], R[v]);
        L[v] = L[v] < 0.f ? 0.f : L[v];
        R[v] = R[v] < 0.f ? 0.f : R[v];
      }
    }
    float pl = L[IPR], pr = R[IPR];
    L[IDN] += rref;
    R[IDN] += rref;
    L[IPR] += pref;
    R[IPR] += pref;
    if (disabled) {
#pragma unroll
      for (int v = 0; v < 5; ++v) F[v] = 0.f;
    } else {
      sweep_riemann<FP>(p.riemann, L, R, pl, pr, pref, ivx, gamma, F);
    }
#pragma unroll
    for (int n = 0; n < NS; ++n) F[5 + n] = F[IDN] > 0.f ? F[IDN] * L[5 + n] : F[IDN] * R[5 + n];
    if (f > f0) {
      const int64_t off = base + (int64_t)(f - 1) * st;
      float d[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        d[v] = A * F[v] - A * Fp[v];
        if (!first) d[v] = dprev[v] + d[v];
      }
      if (last) {
        float wc[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) wc[v] = q[v][2];
        finalize32<NS>(g, p, b, off, i, d, wc);
      } else {
#pragma unroll
        for (int v = 0; v < NV; ++v) b.D[v * sv + off] = d[v];
      }
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      Fp[v] = F[v];
#pragma unroll
      for (int t = 0; t < 6; ++t) q[v][t] = q[v][t + 1];
    }
  }
}

template <int NS, int AX, int FP>
__global__ void __launch_bounds__(128) k_march32(Geo g, Phys p, StageBufs32 b, int seglen,
                                                 int first, int last) {
  march32_line<NS, AX, FP>(g, p, b, seglen, first, last,
                       (int64_t)blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// boundary fills of perturbation arrays: as k_bc, plus the x1 offset of the
// reference between the source and the ghost layer (rho, and E or p)
// ---------------------------------------------------------------------------
struct AxisBC32 {
  int n, ng, lo_type, hi_type;
};

__device__ __forceinline__ int bc_map32(const AxisBC32& a, int i, bool& flip) {
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

// ghost cell t = (i, j, k) of the shell from its image inside the block
__device__ __forceinline__ void bc32_cell(int nc1, int nc2, int64_t sv, AxisBC32 a1,
                                          AxisBC32 a2, AxisBC32 a3, float* var, int nv,
                                          int kind, const double* rb, const double* pb,
                                          double igm1, int64_t t, int i, int j, int k) {
  bool f1, f2, f3;
  int si = bc_map32(a1, i, f1), sj = bc_map32(a2, j, f2), sk = bc_map32(a3, k, f3);
  if (si == i && sj == j && sk == k) return;
  int64_t src = ((int64_t)sk * nc2 + sj) * nc1 + si;
  bool flip = kind != SNAPB_SCALAR;
  // A thread's source cell is never its target, so the loads of a group of
  // variables are issued before its stores: the compiler cannot see that the
  // stores miss the sources and would otherwise wait for one load per
  // variable.
  constexpr int kGroup = 8;
  for (int v0 = 0; v0 < nv; v0 += kGroup) {
    float xs[kGroup];
#pragma unroll
    for (int q = 0; q < kGroup; ++q)
      if (v0 + q < nv) xs[q] = var[(v0 + q) * sv + src];
#pragma unroll
    for (int q = 0; q < kGroup; ++q) {
      const int v = v0 + q;
      if (v >= nv) break;
      double x = xs[q];
      if (flip && ((v == IVX && f1) || (v == IVY && f2) || (v == IVZ && f3))) x = -x;
      if (kind != SNAPB_SCALAR && si != i) {
        if (v == IDN) x += rb[si] - rb[i];
        if (v == IPR) x += (pb[si] - pb[i]) * (kind == SNAPB_CONSERVED ? igm1 : 1.0);
      }
      var[v * sv + t] = (float)x;
    }
  }
}

__global__ void k_bc32(Geo g, AxisBC32 a1, AxisBC32 a2, AxisBC32 a3, float* var, int nv,
                       int kind, const double* rb, const double* pb, double igm1) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= bc_shell_slots(g)) return;
  int i, j, k;
  const int64_t t = bc_shell_cell(g, s, i, j, k);
  bc32_cell(g.nc1, g.nc2, g.sv, a1, a2, a3, var, nv, kind, rb, pb, igm1, t, i, j, k);
}

// conversions between the FP64 state and the FP32 perturbation
__global__ void k_to_pert(int64_t n, int nc1, int kind, double igm1, const double* in,
                          const double* rb, const double* pb, float* out) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int i = umod(t, nc1);
  out[IDN * n + t] = (float)(in[IDN * n + t] - rb[i]);
  out[IVX * n + t] = (float)in[IVX * n + t];
  out[IVY * n + t] = (float)in[IVY * n + t];
  out[IVZ * n + t] = (float)in[IVZ * n + t];
  double pref = kind == SNAPB_CONSERVED ? pb[i] * igm1 : pb[i];
  out[IPR * n + t] = (float)(in[IPR * n + t] - pref);
}

__global__ void k_from_pert(int64_t n, int nc1, int kind, double igm1, const float* in,
                            const double* rb, const double* pb, double* out) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int i = umod(t, nc1);
  out[IDN * n + t] = (double)in[IDN * n + t] + rb[i];
  out[IVX * n + t] = in[IVX * n + t];
  out[IVY * n + t] = in[IVY * n + t];
  out[IVZ * n + t] = in[IVZ * n + t];
  double pref = kind == SNAPB_CONSERVED ? pb[i] * igm1 : pb[i];
  out[IPR * n + t] = (double)in[IPR * n + t] + pref;
}

// CFL limit from w' (full state formed in FP64)
__device__ __forceinline__ double warp_min32(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x = fmin(x, __shfl_xor_sync(0xffffffffu, x, o));
  return x;
}

__global__ void k_cfl32(Geo g, double gammad, int use1, int use2, int use3, const float* w,
                        const float* rbf, const float* pbf, unsigned long long* slots) {
  const int ni = g.iu - g.il + 1, nj = g.ju - g.jl + 1, nk = g.ku - g.kl + 1;
  const int64_t n = (int64_t)ni * nj * nk;
  const float gamma = (float)gammad;
  float a[3] = {0.f, 0.f, 0.f};
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    int i = g.il + umod(t, ni);
    int j = g.jl + umod(udiv(t, ni), nj);
    int k = g.kl + udiv(t, (int64_t)ni * nj);
    int64_t o = (int64_t)k * g.s3 + (int64_t)j * g.s2 + i;
    cfl32_speeds(w, g.sv, o, rbf[i], pbf[i], gamma, a);
  }
  double m1, m2, m3;
  cfl32_limits(g, use1, use2, use3, a, m1, m2, m3);
  __shared__ double red[3][32];
  m1 = warp_min32(m1);
  m2 = warp_min32(m2);
  m3 = warp_min32(m3);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][wid] = m1;
    red[1][wid] = m2;
    red[2][wid] = m3;
  }
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    m1 = lane < nw ? red[0][lane] : 1.7e308;
    m2 = lane < nw ? red[1][lane] : 1.7e308;
    m3 = lane < nw ? red[2][lane] : 1.7e308;
    m1 = warp_min32(m1);
    m2 = warp_min32(m2);
    m3 = warp_min32(m3);
    if (lane == 0) {
      atomicMin(&slots[0], (unsigned long long)__double_as_longlong(m1));
      atomicMin(&slots[1], (unsigned long long)__double_as_longlong(m2));
      atomicMin(&slots[2], (unsigned long long)__double_as_longlong(m3));
    }
  }
}

// ---------------------------------------------------------------------------
// persistent batched kernels: every CTA pulls (member, tile) items
// ---------------------------------------------------------------------------
// Persistent batched x1 sweep (CTA of 32 C threads, C the ensemble's tile
// width): tiles are taken from the queue one ahead, so warp 0 stages the next
// tile's slabs by bulk copies while the current tile's faces are computed.
template <int NS, int FP>
__global__ void __launch_bounds__(512, 2) k_x1_32_batch(const Member32* __restrict__ mem, Phys p,
                                                        WorkQueue q, int stage, int last,
                                                        int nc1max) {
  extern __shared__ __align__(16) float smf[];
  __shared__ Member32 s_mem[2];  // descriptors of the current and the next tile's member
  __shared__ uint64_t bar;       // completion of a tile's bulk copies
  __shared__ unsigned long long s_item;
  const int tid = threadIdx.x;
  // Thread 0 claims work items one tile ahead of their use: the claim of the
  // item after next is issued while the next one is being staged, so the
  // atomic's latency overlaps a whole tile.
  unsigned long long ahead = 0;
  if (tid == 0) {
    mbar_init(&bar, 1);
    s_item = atomicAdd(q.counter, 1ULL);
    ahead = atomicAdd(q.counter, 1ULL);
  }
  __syncthreads();
  int m;
  int64_t tile;
  if (!queue_find(q, (int64_t)s_item, m, tile)) return;
  if (tid < 32) {
    load_member_warp(s_mem[0], mem, m);
    if (tid == 0) set_stage32(s_mem[0].b, stage);
    __syncwarp();
    x1_32_stage<NS>(s_mem[0].g, s_mem[0].b, s_mem[0].x1_cols, tile * s_mem[0].x1_cols, smf,
                    nc1max, &bar);
  }
  __syncthreads();
  int buf = 0;
  unsigned parity = 0;
  while (true) {
    const Member32& cur = s_mem[buf];
    const int C = cur.x1_cols;
    const int64_t col0 = tile * C;
    bool ok = true;
    if (tid < 32) ok = mbar_wait(&bar, parity, &snapb_x1_bulk_timeout);
    if (tid == 0) s_item = ahead;  // the next item, claimed a tile ago
    if (__syncthreads_or(!ok)) {
      if (tid < 32) mbar_wait(&bar, parity, &snapb_x1_bulk_timeout);  // copies in flight
      return;
    }
    int nm;
    int64_t ntile;
    const bool more = queue_find(q, (int64_t)s_item, nm, ntile);
    // the next tile's descriptor: the current one when the member is the same
    const int nbuf = more && nm != m ? buf ^ 1 : buf;
    x1_32_convert<NS>(cur.g, p, cur.b, C, col0, smf, nc1max);  // (ends with a CTA barrier)
    if (more && tid < 32) {  // stage the next tile while this one's faces run
      Member32& nxt = s_mem[nbuf];
      if (nbuf != buf) {
        load_member_warp(nxt, mem, nm);
        if (tid == 0) set_stage32(nxt.b, stage);
        __syncwarp();
      }
      x1_32_stage<NS>(nxt.g, nxt.b, nxt.x1_cols, ntile * nxt.x1_cols, smf, nc1max, &bar);
      if (tid == 0) ahead = atomicAdd(q.counter, 1ULL);  // the item after next
    }
    x1_32_faces<NS, FP>(cur.g, p, cur.b, C, last, col0, smf);
    if (!more) return;
    __syncthreads();  // this tile's rows are read; the next descriptor is in place
    buf = nbuf;
    m = nm;
    parity ^= 1;
    tile = ntile;
  }
}

// the x1 ghost revision of every member, kRevisionItem slots per tile
__global__ void __launch_bounds__(256) k_x1_ghost_revision32_batch(const Member32* __restrict__ mem,
                                                                   Phys p, WorkQueue q) {
  int m;
  int64_t tile;
  while (queue_next(q, m, tile)) {
    const Geo& g = mem[m].g;
    const int64_t n = (int64_t)g.nc2 * g.nc3 * 2 * g.ng, s0 = tile * kRevisionItem;
    for (int64_t slot = s0 + threadIdx.x; slot < min(s0 + kRevisionItem, n); slot += blockDim.x)
      x1_ghost_revision32(g, p, mem[m].b, slot);
  }
}

template <int NS, int AX, int FP>
__global__ void __launch_bounds__(128, 6) k_march32_batch(const Member32* __restrict__ mem, Phys p,
                                                       WorkQueue q, int stage, int first,
                                                       int last) {
  int m;
  int64_t tile;
  while (queue_next(q, m, tile)) {
    const Geo g = mem[m].g;
    StageBufs32 b = mem[m].b;
    set_stage32(b, stage);
    const int seglen = AX == 2 ? mem[m].seglen2 : mem[m].seglen3;
    const int nseg = AX == 2 ? mem[m].nseg2 : mem[m].nseg3;
    const int64_t blk = tile / nseg;
    const int seg = (int)(tile - blk * nseg);
    march32_line<NS, AX, FP>(g, p, b, seglen, first, last, blk * blockDim.x + threadIdx.x, seg);
  }
}

// boundary fill over the ghost shell only (bc_shell_cell, common.cuh)
__global__ void __launch_bounds__(256) k_bc32_batch(const Member32* __restrict__ mem, Phys p,
                                                    WorkQueue q, int kind, double igm1) {
  int m;
  int64_t tile;
  while (queue_next(q, m, tile)) {
    const Geo& g = mem[m].g;
    const Member32& mb = mem[m];
    AxisBC32 a1{g.nc1, g.ng, mb.bc[0], mb.bc[1]};
    AxisBC32 a2{g.nc2, g.ng, mb.bc[2], mb.bc[3]};
    AxisBC32 a3{g.nc3, g.ng, mb.bc[4], mb.bc[5]};
    float* var = kind == SNAPB_SCALAR ? mb.b.s : mb.b.u;
    const int nv = kind == SNAPB_SCALAR ? p.nscalar : 5;
    const int64_t n = bc_shell_slots(g), s0 = tile * kShellItem;
    for (int64_t slot = s0 + threadIdx.x; slot < min(s0 + kShellItem, n); slot += blockDim.x) {
      int i, j, k;
      const int64_t t = bc_shell_cell(g, slot, i, j, k);
      bc32_cell(g.nc1, g.nc2, g.sv, a1, a2, a3, var, nv, kind, mb.b.rb, mb.b.pb, igm1, t, i, j,
                k);
    }
  }
}

// Face profile of the FP32 sweeps along `axis` (sweep_face_states, pert.cuh):
// 1, 2, 3 for the default reconstruction with LMARS, HLLC, Roe; 0 otherwise.
int face_profile32(const Phys& p, int axis) {
  const int typ = axis == 1 ? p.r1_type : p.r23_type;
  const int shock = axis == 1 ? p.r1_shock : p.r23_shock;
  const int scale = axis == 1 ? p.r1_scale : p.r23_scale;
  if (typ != SNAPB_RECON_WENO5 || shock || scale) return 0;
  if (p.nscalar > 0 && (p.rs_type != SNAPB_RECON_WENO5 || p.rs_scale)) return 0;
  switch (p.riemann) {
    case SNAPB_RIEMANN_LMARS: return 1;
    case SNAPB_RIEMANN_HLLC: return 2;
    case SNAPB_RIEMANN_ROE: return 3;
  }
  return 0;
}

// f(NS, FP) with the scalar count and the face profile as compile-time constants
template <class F>
static cudaError_t with_ns_profile(int ns, int fp, F&& f) {
#define SNAPB_NF(NS, FP) \
  case NS * 4 + FP:      \
    return f(std::integral_constant<int, NS>{}, std::integral_constant<int, FP>{});
  if (ns < 0 || ns > 3 || fp < 0 || fp > 3) return cudaErrorInvalidValue;
  switch (ns * 4 + fp) {
    SNAPB_NF(0, 0) SNAPB_NF(0, 1) SNAPB_NF(0, 2) SNAPB_NF(0, 3)
    SNAPB_NF(1, 0) SNAPB_NF(1, 1) SNAPB_NF(1, 2) SNAPB_NF(1, 3)
    SNAPB_NF(2, 0) SNAPB_NF(2, 1) SNAPB_NF(2, 2) SNAPB_NF(2, 3)
    SNAPB_NF(3, 0) SNAPB_NF(3, 1) SNAPB_NF(3, 2) SNAPB_NF(3, 3)
  }
#undef SNAPB_NF
  return cudaErrorInvalidValue;
}

cudaError_t launch_x1_32_batch(const Member32* mem, const Phys& p, const WorkQueue& q,
                               int stage, bool last, const PersistGrid& pg, size_t smem, int C,
                               int nc1max, cudaStream_t st) {
  const int nt = 32 * C;  // one warp per column of a tile
  return with_ns_profile(p.nscalar, face_profile32(p, 1), [&](auto ns, auto fp) {
    constexpr int NS = decltype(ns)::value, FP = decltype(fp)::value;
    raise_smem_limit(k_x1_32_batch<NS, FP>, 200 * 1024);
    const int grid = persistent_grid(k_x1_32_batch<NS, FP>, nt, smem, pg);
    k_x1_32_batch<NS, FP><<<grid, nt, smem, st>>>(mem, p, q, stage, last ? 1 : 0, nc1max);
    return cudaGetLastError();
  });
}

cudaError_t launch_x1_ghost_revision32_batch(const Member32* mem, const Phys& p,
                                             const WorkQueue& q, const PersistGrid& pg,
                                             cudaStream_t st) {
  k_x1_ghost_revision32_batch<<<persistent_grid(k_x1_ghost_revision32_batch, 256, 0, pg), 256, 0,
                                st>>>(mem, p, q);
  return cudaGetLastError();
}

cudaError_t launch_march32_batch(int axis, const Member32* mem, const Phys& p,
                                 const WorkQueue& q, int stage, bool first, bool last,
                                 const PersistGrid& pg, cudaStream_t st) {
  return with_ns_profile(p.nscalar, face_profile32(p, axis), [&](auto ns, auto fp) {
    constexpr int NS = decltype(ns)::value, FP = decltype(fp)::value;
    if (axis == 2)
      k_march32_batch<NS, 2, FP><<<persistent_grid(k_march32_batch<NS, 2, FP>, 128, 0, pg), 128,
                                   0, st>>>(mem, p, q, stage, first, last);
    else
      k_march32_batch<NS, 3, FP><<<persistent_grid(k_march32_batch<NS, 3, FP>, 128, 0, pg), 128,
                                   0, st>>>(mem, p, q, stage, first, last);
    return cudaGetLastError();
  });
}

cudaError_t launch_bc32_batch(const Member32* mem, const Phys& p, const WorkQueue& q, int kind,
                              double igm1, const PersistGrid& pg, cudaStream_t st) {
  k_bc32_batch<<<persistent_grid(k_bc32_batch, 256, 0, pg), 256, 0, st>>>(mem, p, q, kind, igm1);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// launchers (called from capi32.cu)
// ---------------------------------------------------------------------------
cudaError_t launch_ref32(const Geo& g, const Phys& p, const double* rb, const double* pb,
                         double* rbw, double* pbw, const StageBufs32& b, cudaStream_t st) {
  int n = g.nc1 + 1;
  k_ref32<<<(n + 127) / 128, 128, 0, st>>>(g, p, rb, pb, rbw, pbw, b);
  k_ref32_residual<<<(n + 127) / 128, 128, 0, st>>>(g, p, b);
  return cudaGetLastError();
}

// columns per x1 tile: a power of two (one warp per column), 8 by default
// (the fastest measured) within about 96 KB of shared memory
int x1_columns_pow2(int c) {
  c = std::max(1, std::min(c, 16));  // CTAs of at most 512 threads
  while (c & (c - 1)) c &= c - 1;
  return c;
}
int x1_columns_per_cta32(const Geo& g, int nvt) {
  size_t per = x1_smem32_per_column(g, nvt);
  return x1_columns_pow2((int)std::min<size_t>(8, std::max<size_t>(1, (96 * 1024) / per)));
}

cudaError_t launch_x1_ghost_revision32(const Geo& g, const Phys& p, const StageBufs32& b,
                                       cudaStream_t st) {
  if (p.grav1 == 0.) return cudaSuccess;
  const int64_t n = (int64_t)g.nc2 * g.nc3 * 2 * g.ng;
  k_x1_ghost_revision32<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, p, b);
  return cudaGetLastError();
}

template <int NS, int FP>
static cudaError_t launch_x1_32t(const Geo& g, const Phys& p, const StageBufs32& b, bool last,
                                 cudaStream_t st) {
  const int nvt = 5 + NS;
  int C = x1_columns_per_cta32(g, nvt);
  size_t smem = x1_smem32_bytes(g.nc1, nvt, C);
  if (smem > 200 * 1024) return cudaErrorInvalidConfiguration;
  raise_smem_limit(k_x1_32<NS, FP>, 200 * 1024);
  cudaError_t e = launch_x1_ghost_revision32(g, p, b, st);
  if (e != cudaSuccess) return e;
  int64_t ncol = (int64_t)g.nc2 * g.nc3;
  k_x1_32<NS, FP><<<(unsigned)((ncol + C - 1) / C), 32 * C, smem, st>>>(g, p, b, C,
                                                                      last ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_x1_32(const Geo& g, const Phys& p, const StageBufs32& b, bool last,
                         cudaStream_t st) {
  return with_ns_profile(p.nscalar, face_profile32(p, 1), [&](auto ns, auto fp) {
    return launch_x1_32t<decltype(ns)::value, decltype(fp)::value>(g, p, b, last, st);
  });
}

template <int NS, int AX, int FP>
static cudaError_t launch_march32_t(const Geo& g, const Phys& p, const StageBufs32& b,
                                    bool first, bool last, cudaStream_t st) {
  int ni = g.iu - g.il + 1;
  int no = AX == 2 ? g.ku - g.kl + 1 : g.ju - g.jl + 1;
  int n = AX == 2 ? g.nx2 : g.nx3;
  int seglen = 32;
  int64_t threads = (int64_t)ni * no;
  while (seglen > 8 && threads * ((n + seglen - 1) / seglen) < 148LL * 1024 * 2) seglen /= 2;
  dim3 grid((unsigned)((threads + 127) / 128), (unsigned)((n + seglen - 1) / seglen));
  k_march32<NS, AX, FP><<<grid, 128, 0, st>>>(g, p, b, seglen, first ? 1 : 0, last ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_march32(int axis, const Geo& g, const Phys& p, const StageBufs32& b,
                           bool first, bool last, cudaStream_t st) {
  return with_ns_profile(p.nscalar, face_profile32(p, axis), [&](auto ns, auto fp) {
    constexpr int NS = decltype(ns)::value, FP = decltype(fp)::value;
    return axis == 2 ? launch_march32_t<NS, 2, FP>(g, p, b, first, last, st)
                     : launch_march32_t<NS, 3, FP>(g, p, b, first, last, st);
  });
}

cudaError_t launch_bc32(const Geo& g, const snapb_hydro_config& c, float* var, int nv, int kind,
                        const double* rb, const double* pb, cudaStream_t st) {
  AxisBC32 a1{g.nc1, g.ng, c.bc[0], c.bc[1]};
  AxisBC32 a2{g.nc2, g.ng, c.bc[2], c.bc[3]};
  AxisBC32 a3{g.nc3, g.ng, c.bc[4], c.bc[5]};
  const int64_t n = bc_shell_slots_host(g);
  if (n == 0) return cudaSuccess;
  k_bc32<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, a1, a2, a3, var, nv, kind, rb, pb,
                                                     1.0 / (c.gammad - 1.0));
  return cudaGetLastError();
}

cudaError_t launch_to_pert(const Geo& g, const Phys& p, int kind, const double* in,
                           const double* rb, const double* pb, float* out, cudaStream_t st) {
  k_to_pert<<<(unsigned)((g.sv + 255) / 256), 256, 0, st>>>(g.sv, g.nc1, kind,
                                                            1.0 / (p.gammad - 1.0), in, rb, pb,
                                                            out);
  return cudaGetLastError();
}

cudaError_t launch_from_pert(const Geo& g, const Phys& p, int kind, const float* in,
                             const double* rb, const double* pb, double* out, cudaStream_t st) {
  k_from_pert<<<(unsigned)((g.sv + 255) / 256), 256, 0, st>>>(g.sv, g.nc1, kind,
                                                              1.0 / (p.gammad - 1.0), in, rb, pb,
                                                              out);
  return cudaGetLastError();
}

cudaError_t launch_cfl32(const Geo& g, const Phys& p, const float* w, const float* rbf,
                         const float* pbf, unsigned long long* slots, cudaStream_t st) {
  int scheme = p.implicit_scheme;
  int use1 = g.nc1 > 1, use2 = g.nc2 > 1, use3 = g.nc3 > 1;
  if (scheme != 0) {
    use1 = use1 && (!(scheme & 1) || (g.nc3 == 1 && g.nc2 == 1));
    use2 = use2 && !((scheme >> 1) & 1);
    use3 = use3 && !((scheme >> 2) & 1);
  }
  int64_t n = (int64_t)(g.iu - g.il + 1) * (g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
  k_cfl32<<<blocks, 256, 0, st>>>(g, p.gammad, use1, use2, use3, w, rbf, pbf, slots);
  return cudaGetLastError();
}

}  // namespace snapb

extern "C" int snapb_bulk_copy_timeouts(void) {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, snapb::snapb_x1_bulk_timeout, sizeof(int)) != cudaSuccess)
    return -1;
  if (v) {
    const int z = 0;
    if (cudaMemcpyToSymbol(snapb::snapb_x1_bulk_timeout, &z, sizeof(int)) != cudaSuccess)
      return -1;
  }
  return v;
}
