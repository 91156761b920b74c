// vic_cr.cu — vertically implicit correction (VIC) of one RK stage of the FP32
// perturbation form, 3x3 blocks, by block cyclic reduction: one CTA per x1
// column (x1 is the vertical axis), the column's whole system in shared
// memory, everything in one kernel.
//
// Per column (nl layers, one thread per layer and phase):
//   (1) the full primitives of cells -1 .. nl (FP64 reference + FP32
//       perturbation, rounded to FP32 as the blocks take them) and the flux
//       Jacobian J of each cell, then |A| = R |Lambda| R^-1 at the Roe
//       average of each face, all in FP32 and in parallel over the column;
//   (2) the blocks of each layer, a_i (diagonal), b_i (below), c_i (above),
//       assembled in FP32 exactly as the column sweep of vic.cu assembles
//       them (the reference's vic_assemble), then widened to FP64, with the
//       right-hand side du_i / dt in FP64;
//   (3) block cyclic reduction in FP64: at stride s the equations i with
//       i % 2s == s are eliminated from their neighbours i +- s (3x3 cofactor
//       inverses, as the reference's 3x3 solve), until equation 0 alone is
//       left; then the solutions are filled in back down the strides;
//   (4) the MS-VIC column sums (sum (rho V)^2 and B_dry, FP64 block
//       reductions) and, per cell, the mass redistribution, the scalar mass
//       fix and the RK combination (or du), as the finish kernel of vic.cu.
// Nothing of the solve goes through HBM: the kernel reads w', du, u, u0 (and
// the scalars) once, coalesced along x1, and writes u (and u0, s, r).
//
// Block cyclic reduction eliminates the same block-tridiagonal system as the
// reference's block-Thomas sweep (ForwardSweep,
// src/implicit/forward_sweep_impl.h:20-109, then the back substitution of
// src/implicit/vic_redistribute_impl.h:26-106); its operation order differs,
// so the two agree up to FP64 rounding.  Blocks: vic_assemble_partial_impl
// (src/implicit/vic_assemble_partial_impl.h:29-111) and the flux
// decomposition (src/implicit/flux_decomposition_impl.h:133-245).
#include <algorithm>

#include "block_cr.cuh"
#include "kernels.cuh"
#include "vic_blocks.cuh"
#include "vic_common.cuh"

namespace snapb {

namespace {

constexpr int kCrThreads = 128;
constexpr int kCrMaxLayers = 256;  // longest column the solver takes

// Shared-memory plan of one column with nl layers: FP32 block-formation
// buffers, then the FP64 system (b, a, c blocks and right-hand sides, the
// solution overwriting the right-hand side) and the reduction scratch.
struct CrPlan {
  int nl;
  __host__ __device__ int nc() const { return nl + 2; }  // cells -1 .. nl
  __host__ __device__ size_t floats() const {
    return (size_t)nc() * (5 + 9) + (size_t)(nl + 1) * 9;  // W, J per cell; |A| per face
  }
  __host__ __device__ size_t dbl_offset() const { return ((floats() * 4 + 15) / 16) * 16; }
  __host__ __device__ size_t bytes() const {
    return dbl_offset() + ((size_t)nl * 30 + 2 * (kCrThreads / 32)) * sizeof(double);
  }
};

// One column of the FP32 form, the whole CTA.  b's stage fields are set.
template <int NS>
__device__ __forceinline__ void vic_cr_column(const Geo& g, const Phys& p, const StageBufs32& b,
                                              int64_t col, char* smem) {
  constexpr int N = 3;
  const CrPlan P{g.nx1};
  const int nl = P.nl, nc = P.nc(), tid = threadIdx.x, nt = blockDim.x;
  const int64_t sv = g.sv, cb = column_base(g, col);
  float* wf = reinterpret_cast<float*>(smem);  // [5][nc]  full primitives, cell i at i + 1
  float* Jf = wf + 5 * nc;                     // [nc][9]  J of cell i at i + 1
  float* Af = Jf + 9 * nc;                     // [nl+1][9] |A| of face f (cells f-1, f)
  double* Bl = reinterpret_cast<double*>(smem + P.dbl_offset());  // [nl][9] below (x_{i-s})
  double* Dg = Bl + 9 * nl;                                       // [nl][9] diagonal
  double* Ab = Dg + 9 * nl;                                       // [nl][9] above (x_{i+s})
  double* R = Ab + 9 * nl;                                        // [nl][3] rhs, then x
  double* red = R + 3 * nl;
  const double dt = *b.dt, V = g.vol;
  const double gm1c = p.gammad - 1.;
  const double gm1f = 0.5 * (p.gammad + p.gammad) - 1.;

  // (1) cells: full primitives and J; sum (rho V)^2 over the layers
  double sa2 = 0.;
  for (int t = tid; t < nc; t += nt) {
    const int i = t - 1;
    float fw[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const double x = vic_w(b, sv, v, cb + i, g.il + i);
      fw[v] = (float)x;
      wf[v * nc + t] = fw[v];
      if (v == IDN && i >= 0 && i < nl) {
        const double ai = x * V;
        sa2 += ai * ai;
      }
    }
    float J[N][N];
    jac_block<N, float>((float)gm1c, fw, J);
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
      for (int q = 0; q < N; ++q) Jf[t * 9 + r * 3 + q] = J[r][q];
  }
  __syncthreads();
  for (int f = tid; f <= nl; f += nt) {  // faces: |A| at the Roe average of cells f-1, f
    float wl[5], wr[5], A[N][N];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      wl[v] = wf[v * nc + f];
      wr[v] = wf[v * nc + f + 1];
    }
    absA_block<N, float>((float)gm1f, wl, wr, A);
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
      for (int q = 0; q < N; ++q) Af[f * 9 + r * 3 + q] = A[r][q];
  }
  __syncthreads();

  // (2) layer blocks, assembled in FP32 as the column sweep does, widened
  {
    const float Aa = (float)g.A1, hiv = (float)(0.5 / g.vol), idt = (float)(1. / dt),
                grav = (float)p.grav1;
    for (int i = tid; i < nl; i += nt) {
      const float* Am = Af + i * 9;        // face below
      const float* Ap = Af + (i + 1) * 9;  // face above
      const float* Jp = Jf + i * 9;        // cell i - 1
      const float* Jn = Jf + (i + 2) * 9;  // cell i + 1
      float af[9], bf[9], cf[9];
#pragma unroll
      for (int r = 0; r < N; ++r)
#pragma unroll
        for (int q = 0; q < N; ++q) {
          float phi = 0.f;
          if (r == 1 && q == 0) phi = grav;
          if (r == 2 && q == 1) phi = grav;
          const int k = r * 3 + q;
          af[k] = (Am[k] * Aa + Ap[k] * Aa) * hiv - phi;
          bf[k] = -(Am[k] + Jp[k]) * Aa * hiv;
          cf[k] = -(Ap[k] - Jn[k]) * Aa * hiv;
        }
#pragma unroll
      for (int r = 0; r < N; ++r) af[r * 3 + r] += idt;
      if (i == 0) {
#pragma unroll
        for (int k = 0; k < 9; ++k) af[k] += bf[k] * ((k % 3) == 1 ? -1.f : 1.f);
      }
      if (i == nl - 1) {
#pragma unroll
        for (int k = 0; k < 9; ++k) af[k] += cf[k] * ((k % 3) == 1 ? -1.f : 1.f);
      }
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        Dg[i * 9 + k] = (double)af[k];
        Bl[i * 9 + k] = i == 0 ? 0. : (double)bf[k];       // no layer below the first
        Ab[i * 9 + k] = i == nl - 1 ? 0. : (double)cf[k];  // none above the last
      }
#pragma unroll
      for (int r = 0; r < N; ++r) R[i * 3 + r] = vic_d(b, sel<N>(r) * sv + cb + i) / dt;
    }
  }
  __syncthreads();

  // (3) block cyclic reduction, FP64
  block_cr3_solve(Bl, Dg, Ab, R, nl);

  // (4) column sums, then every cell of the column
  double bdry = 0.;
  for (int i = tid; i < nl; i += nt) bdry += (vic_d(b, IDN * sv + cb + i) - R[i * 3]) * 1. * V;
  cta_sum2(sa2, bdry, red);
  const bool du_only = b.vic_du_only, first = b.stage == 0;
  for (int i = tid; i < nl; i += nt) {
    const int64_t off = cb + i;
    const int xi = g.il + i;
    const double rhok = vic_full(b, (double)b.w[IDN * sv + off], IDN, xi);
    const double etk = vic_d(b, IDN * sv + off);
    const double ai = rhok * g.vol;
    const double fix = R[i * 3] - etk;
    double du[5];
    du[IDN] = etk + fix * 1. + rhok * ai * bdry / sa2;
    du[IVX] = R[i * 3 + 1];
    du[IVY] = vic_d(b, IVY * sv + off);
    du[IVZ] = vic_d(b, IVZ * sv + off);
    du[IPR] = R[i * 3 + 2];
    if (b.M) b.M[IDN * sv + off] = fix;
    if (du_only) {
#pragma unroll
      for (int v = 0; v < 5; ++v) vic_set_d(b, v * sv + off, du[v]);
      continue;
    }
    double unew_rho = 0.;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const int64_t o = v * sv + off;
      const double uo = b.u[o], u0o = first ? 0. : (double)b.u0[o];
      const double un = vic_rk_from(b.u, b.u0, o, first, uo, u0o, b.wgt0, b.wgt1, b.wgt2, du[v]);
      if (v == IDN) unew_rho = vic_full_rho(b, un, xi);
    }
#pragma unroll
    for (int n = 0; n < NS; ++n) {
      const int64_t o = n * sv + off;
      const double so = b.s[o], s0o = first ? 0. : (double)b.s0[o];
      const double ds = vic_d(b, (5 + n) * sv + off) + fix * (double)b.r[o];
      const double sn = vic_rk_from(b.s, b.s0, o, first, so, s0o, b.wgt0, b.wgt1, b.wgt2, ds);
      b.r[o] = sn / unew_rho;
    }
  }
}

template <int NS>
__global__ void __launch_bounds__(kCrThreads, 4) k_vic_cr32(Geo g, Phys p, StageBufs32 b) {
  extern __shared__ __align__(16) char cr_smem[];
  vic_cr_column<NS>(g, p, b, blockIdx.x, cr_smem);
}

template <int NS>
__global__ void __launch_bounds__(kCrThreads, 4) k_vic_cr32_batch(const Member32* __restrict__ mem,
                                                                  Phys p, WorkQueue q, int stage) {
  extern __shared__ __align__(16) char cr_smem[];
  __shared__ Member32 s_mem;  // the member's descriptor, read as the column needs its fields
  int m;
  int64_t tile;
  while (queue_next(q, m, tile)) {  // (starts with a barrier: the last column is done)
    load_member(s_mem, mem, m);
    if (threadIdx.x == 0) set_stage32(s_mem.b, stage);
    __syncthreads();
    vic_cr_column<NS>(s_mem.g, p, s_mem.b, tile, cr_smem);
  }
}

// (the limit is set once per kernel, so to the cap rather than to the first
// column height's plan)
template <class K>
void allow_smem(K kernel, size_t bytes) {
  if (bytes > 48 * 1024) raise_smem_limit(kernel, 200 * 1024);
}

}  // namespace

// the solver applies to the FP32 form with 3x3 blocks and columns of at most
// kCrMaxLayers layers
bool vic_cr_applies(const Geo& g, const Phys& p) {
  return p.implicit_scheme != 0 && vic_n(p) == 3 && g.nx1 >= 1 && g.nx1 <= kCrMaxLayers &&
         p.nscalar <= 3;
}

size_t vic_cr_smem_bytes(int nl) { return CrPlan{nl}.bytes(); }

cudaError_t launch_vic_cr32(const Geo& g, const Phys& p, const StageBufs32& b, cudaStream_t st) {
  const int64_t ncol = (int64_t)(g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  const size_t smem = vic_cr_smem_bytes(g.nx1);
#define SNAPB_CR(NS)                                                         \
  case NS:                                                                   \
    allow_smem(k_vic_cr32<NS>, vic_cr_smem_bytes(kCrMaxLayers));             \
    k_vic_cr32<NS><<<(unsigned)ncol, kCrThreads, smem, st>>>(g, p, b);       \
    break;
  switch (p.nscalar) {
    SNAPB_CR(0)
    SNAPB_CR(1)
    SNAPB_CR(2)
    SNAPB_CR(3)
    default: return cudaErrorInvalidValue;
  }
#undef SNAPB_CR
  return cudaGetLastError();
}

cudaError_t launch_vic_cr32_batch(const Member32* mem, const Phys& p, const WorkQueue& q,
                                  int stage, const PersistGrid& pg, int max_layers,
                                  cudaStream_t st) {
  const size_t smem = vic_cr_smem_bytes(max_layers);
#define SNAPB_CRB(NS)                                                                       \
  case NS:                                                                                  \
    allow_smem(k_vic_cr32_batch<NS>, vic_cr_smem_bytes(kCrMaxLayers));                      \
    k_vic_cr32_batch<NS><<<persistent_grid(k_vic_cr32_batch<NS>, kCrThreads, smem, pg),      \
                           kCrThreads, smem, st>>>(mem, p, q, stage);                       \
    break;
  switch (p.nscalar) {
    SNAPB_CRB(0)
    SNAPB_CRB(1)
    SNAPB_CRB(2)
    SNAPB_CRB(3)
    default: return cudaErrorInvalidValue;
  }
#undef SNAPB_CRB
  return cudaGetLastError();
}

}  // namespace snapb
