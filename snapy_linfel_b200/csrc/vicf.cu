// vicf.cu — vertically implicit correction (VIC) of one RK stage as one fused
// kernel, a variant of the column + finish pair of vic.cu.
//
// One kernel per solve: k_vicf, one CTA per tile of 32 x1 columns (x1 is the
// vertical axis; a tile's column index sits on the lanes), or its persistent
// batched form k_vicf_batch over the tiles of many ensemble members.  Per tile:
//   (1) producer warps form the blocks of each layer from the state — a_i,
//       b_i, c_i and the right-hand side du_i / dt, with the Roe-averaged
//       |A| = R |Lambda| R^-1 at the layer's two faces and the flux
//       Jacobians J of the cells below and above — into a double-buffered
//       ring of chunks in shared memory;
//   (2) two elimination warps work the block-tridiagonal system from both
//       ends at once (a twisted block factorisation): warp 0 eliminates
//       upwards from the bottom layer, as the reference's forward sweep
//       does, warp 1 downwards from the top layer; at the middle layer
//       m = nl / 2 the two reduced systems meet and that layer is solved
//       first.  Each chain is half as long as one sweep over the column;
//   (3) both warps back-substitute outwards from the middle layer and
//       accumulate the MS-VIC column sums;
//   (4) the whole CTA applies the mass redistribution, the scalar mass fix
//       and the RK combination (or leaves du) to the tile's cells, its
//       inputs staged through shared memory by cp.async.
// (1) and (2) overlap: the producers fill chunk c+1 while the elimination
// warps consume chunk c, with one CTA barrier per chunk (no other
// synchronisation).  The reduced blocks and partial solutions (N*N + N
// doubles per cell) are written by (2) and read back by (3) inside the same
// CTA a short time later, so with a few tiles in flight per SM they are
// served by L2 rather than HBM.  Every elimination step is FP64.
//
// Reference: ImplicitHydroImpl::forward (src/implicit/implicit_hydro.cpp:99-189),
// vic_assemble_partial_impl (src/implicit/vic_assemble_partial_impl.h:29-111),
// vic_assemble_full_impl (src/implicit/vic_assemble_full_impl.h:16-106),
// ForwardSweep (src/implicit/forward_sweep_impl.h:20-109), ludcmp/lubksb
// (src/math/ludcmp.h:24-76, src/math/lubksb.h:124-147),
// vic_backward_reduce / vic_redistribute_cell (src/implicit/vic_redistribute_impl.h:26-106),
// flux Jacobian and Roe eigenvectors (src/implicit/flux_decomposition_impl.h:133-245).
// The reference eliminates each column bottom-up only; the twisted order
// gives the same solution up to rounding.
#include <cstring>
#include <mutex>
#include <type_traits>
#include <utility>
#include <string>

#include "kernels.cuh"
#include "ring.cuh"
#include "vic_blocks.cuh"
#include "vic_common.cuh"

namespace snapb {
namespace fused {


// Tile shape and shared-memory plan of the fused kernel for N x N blocks.
template <int N>
struct VicCfg {
  static constexpr int TC = 32;               // columns per tile (lane = column)
  static constexpr int K = N == 3 ? 2 : 1;    // layers per chunk at each end
  static constexpr int PW = N == 3 ? 2 : 1;   // producer warps per end
  static constexpr int NT = (2 + 2 * PW) * 32;
  static constexpr int NN = N * N;
  static constexpr int RE = 3 * NN + N;       // ring entry: a, b, c, rhs
  static constexpr int ES = NN + N;           // scratch record: reduced block, partial solution
  static constexpr int BD = N == 3 ? 4 : 2;   // back-substitution prefetch depth (layers)
  static constexpr int BE = ES + 2;           // back ring entry: record, du[IDN], w[IDN]
  static constexpr size_t ring_bytes = (size_t)2 * 2 * K * RE * TC * sizeof(double);
  static constexpr size_t back_bytes = (size_t)2 * BD * BE * 32 * sizeof(double);
  // fixed area after the shared region: the top chain's last reduced block and
  // partial solution [ES][TC], the middle solution [N][TC], the column sums
  // [4][TC] and the column offsets [TC] (int64)
  static constexpr size_t fixed_bytes = ((size_t)(ES + N + 4) * TC + TC) * sizeof(double);
};

// Finish staging: per sub-tile of TL layers, the solution rows [N][TC][TL+1]
// (doubles) and the cell inputs [elem][TC][TL] in the stored precision T:
// w[IDN], the du rows the solve does not replace, u, u0, and per scalar s,
// s0, r and its du row.
template <int N, int NS, class T>
struct VicFin {
  static constexpr int TC = VicCfg<N>::TC;
  static constexpr int DR = N == 3 ? 3 : 1;   // du rows read: IDN (+ IVY, IVZ)
  static constexpr int elems = 1 + DR + 10 + 4 * NS;
  static constexpr size_t bytes_for(int tl) {
    return (size_t)N * TC * (tl + 1) * sizeof(double) + (size_t)elems * TC * tl * sizeof(T);
  }
  static constexpr int TL = bytes_for(16) <= 64 * 1024 ? 16 : 8;
  static constexpr size_t bytes = bytes_for(TL);
};

template <class B>
using StoredT = std::remove_pointer_t<decltype(std::declval<B>().u)>;

template <int N, int NS, class T>
constexpr size_t vic_smem_bytes() {
  using C = VicCfg<N>;
  size_t r = C::ring_bytes;
  if (C::back_bytes > r) r = C::back_bytes;
  if (VicFin<N, NS, T>::bytes > r) r = VicFin<N, NS, T>::bytes;
  r = (r + 15) & ~(size_t)15;
  return r + C::fixed_bytes;
}

// Scratch: per tile of TC columns, [nl][N*N+N][TC] doubles (column fastest,
// so a warp's stores and loads of one element are one 256-byte line).
size_t scratch_bytes(const Geo& g, const Phys& p) {
  if (p.implicit_scheme == 0) return 0;
  const int N = vic_n(p);
  const int64_t ncol = (int64_t)(g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  const int64_t tiles = (ncol + 31) / 32;
  return (size_t)(tiles * 32 * (int64_t)g.nx1 * (N * N + N)) * sizeof(double);
}

// Block construction per form: the FP64 plain form in FP64; the FP32
// perturbation form forms |A| and J in FP32 from the full states (only the
// elimination and the balance terms stay FP64 there) and widens them.
template <int N>
__device__ __forceinline__ void absA_of(const StageBufs&, double gm1, const double* wl,
                                        const double* wr, double (&A)[N][N]) {
  absA_block<N>(gm1, wl, wr, A);
}
template <int N>
__device__ __forceinline__ void jac_of(const StageBufs&, double gm1, const double* w,
                                       double (&J)[N][N]) {
  jac_block<N>(gm1, w, J);
}
template <int N>
__device__ __forceinline__ void absA_of(const StageBufs32&, double gm1, const double* wl,
                                        const double* wr, double (&A)[N][N]) {
  float fl[5], fr[5], F[N][N];
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    fl[v] = (float)wl[v];
    fr[v] = (float)wr[v];
  }
  absA_block<N, float>((float)gm1, fl, fr, F);
#pragma unroll
  for (int r = 0; r < N; ++r)
#pragma unroll
    for (int q = 0; q < N; ++q) A[r][q] = (double)F[r][q];
}
template <int N>
__device__ __forceinline__ void jac_of(const StageBufs32&, double gm1, const double* w,
                                       double (&J)[N][N]) {
  float fw[5], F[N][N];
#pragma unroll
  for (int v = 0; v < 5; ++v) fw[v] = (float)w[v];
  jac_block<N, float>((float)gm1, fw, F);
#pragma unroll
  for (int r = 0; r < N; ++r)
#pragma unroll
    for (int q = 0; q < N; ++q) J[r][q] = (double)F[r][q];
}

// ---------------------------------------------------------------------------
// (1) the blocks of layer i of one column (cb: the column's (k, j, il)
// offset), written to out[e * TC], e = a (N*N), b (N*N), c (N*N), rhs (N):
//   a_i = (|A|_{i-1/2} + |A|_{i+1/2}) A / (2V) - Phi + I / dt,
//   b_i = -(|A|_{i-1/2} + J_{i-1}) A / (2V),  c_i = -(|A|_{i+1/2} - J_{i+1}) A / (2V),
// with the reflecting-wall fix a += b diag(1,-1,1,..) at the bottom layer and
// a += c diag(..) at the top one, rhs = du_i / dt
// (vic_assemble_partial_impl.h:29-111, forward_sweep_impl.h:31-47).
// ---------------------------------------------------------------------------
template <int N, class B>
__device__ __forceinline__ void vic_layer_blocks(const Geo& g, const Phys& p, const B& b,
                                                 int64_t cb, int i, int nl, double dt,
                                                 double* out) {
  constexpr int NN = N * N, TC = VicCfg<N>::TC;
  const int64_t sv = g.sv;
  const double gm1c = p.gammad - 1.;
  const double gm1f = 0.5 * (p.gammad + p.gammad) - 1.;
  const double Aa = g.A1, hiv = 0.5 / g.vol, idt = 1. / dt, grav = p.grav1;
  double wm[5], wc[5], wp[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    wm[v] = vic_w(b, sv, v, cb + i - 1, g.il + i - 1);
    wc[v] = vic_w(b, sv, v, cb + i, g.il + i);
    wp[v] = vic_w(b, sv, v, cb + i + 1, g.il + i + 1);
  }
  double Am[N][N], Ap[N][N], J[N][N], bb[N][N], cc[N][N];
  absA_of<N>(b, gm1f, wm, wc, Am);
  jac_of<N>(b, gm1c, wm, J);
#pragma unroll
  for (int r = 0; r < N; ++r)
#pragma unroll
    for (int q = 0; q < N; ++q) bb[r][q] = -(Am[r][q] + J[r][q]) * Aa * hiv;
  absA_of<N>(b, gm1f, wc, wp, Ap);
  jac_of<N>(b, gm1c, wp, J);
#pragma unroll
  for (int r = 0; r < N; ++r)
#pragma unroll
    for (int q = 0; q < N; ++q) cc[r][q] = -(Ap[r][q] - J[r][q]) * Aa * hiv;
#pragma unroll
  for (int r = 0; r < N; ++r)
#pragma unroll
    for (int q = 0; q < N; ++q) {
      double phi = 0.;
      if (r == 1 && q == 0) phi = grav;
      if (N == 3 && r == 2 && q == 1) phi = grav;
      if (N == 5 && r == IPR && q == IVX) phi = grav;
      double a = (Am[r][q] * Aa + Ap[r][q] * Aa) * hiv - phi;
      if (r == q) a += idt;
      if (i == 0) a += bb[r][q] * (q == 1 ? -1. : 1.);
      if (i == nl - 1) a += cc[r][q] * (q == 1 ? -1. : 1.);
      out[(r * N + q) * TC] = a;
      out[(NN + r * N + q) * TC] = bb[r][q];
      out[(2 * NN + r * N + q) * TC] = cc[r][q];
    }
#pragma unroll
  for (int r = 0; r < N; ++r) out[(3 * NN + r) * TC] = vic_d(b, sel<N>(r) * sv + cb + i) / dt;
}

// X -= L Y (N x N) and y -= L z (N) with L, Y, z in registers
template <int N>
__device__ __forceinline__ void vic_eliminate(double (&X)[N][N], double (&y)[N],
                                              const double (&L)[N][N], const double (&Y)[N][N],
                                              const double (&z)[N]) {
#pragma unroll
  for (int r = 0; r < N; ++r) {
    double bd = 0.;
#pragma unroll
    for (int q = 0; q < N; ++q) {
      double t = 0.;
#pragma unroll
      for (int kk = 0; kk < N; ++kk) t += L[r][kk] * Y[kk][q];
      X[r][q] -= t;
      bd += L[r][q] * z[q];
    }
    y[r] = y[r] - bd;
  }
}

// ---------------------------------------------------------------------------
// (4) finish of layers [i0, i0 + TL) of the tile: redistribution, scalar mass
// fix, RK combination (or du), all inputs of the sub-tile fetched by cp.async
// first (the solution rows along columns, the cell values along x1).
// ---------------------------------------------------------------------------
template <int N, int NS, class B>
__device__ __forceinline__ void vic_finish_subtile(const Geo& g, const B& b, const double* S,
                                                   const double* zs, const int64_t* cbs,
                                                   int64_t col0, int64_t ncol, int i0,
                                                   double* sm) {
  using C = VicCfg<N>;
  using F = VicFin<N, NS, StoredT<B>>;
  using T = StoredT<B>;
  constexpr int TC = C::TC, ES = C::ES, NN = C::NN, TL = F::TL, DR = F::DR;
  const int nl = g.nx1;
  const int64_t sv = g.sv;
  double* dl = sm;                                             // [N][TC][TL+1]
  T* cell = reinterpret_cast<T*>(dl + (size_t)N * TC * (TL + 1));  // [elem][TC][TL]
  auto DL = [&](int r, int c, int s) -> double& { return dl[((size_t)r * TC + c) * (TL + 1) + s]; };
  auto CE = [&](int e, int c, int s) -> T* { return cell + ((size_t)e * TC + c) * TL + s; };
  const bool du_only = b.vic_du_only, first = b.stage == 0;
  const int eRHO = 0, eDU = 1, eU = 1 + DR, eU0 = eU + 5, eS = eU0 + 5;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int idx = tid; idx < N * TC * TL; idx += nt) {
    const int c = idx % TC, rest = idx / TC;
    const int s = rest % TL, r = rest / TL;
    const int i = i0 + s;
    if (col0 + c < ncol && i < nl)
      cp_async_bytes8(&DL(r, c, s), S + ((int64_t)i * ES + NN + r) * TC + c);
  }
  const int ne = du_only ? eU : (first ? eU0 : eS);  // u0 is the stage input at stage 0
  for (int idx = tid; idx < ne * TC * TL; idx += nt) {
    const int s = idx % TL, rest = idx / TL;
    const int c = rest % TC, e = rest / TC;
    const int i = i0 + s;
    if (col0 + c >= ncol || i >= nl) continue;
    const int64_t off = cbs[c] + i;
    const T* src;
    if (e == eRHO) src = b.w + IDN * sv + off;
    else if (e < eU) src = b.D + (e == eDU ? IDN : (e == eDU + 1 ? IVY : IVZ)) * sv + off;
    else if (e < eU0) src = b.u + (e - eU) * sv + off;
    else src = b.u0 + (e - eU0) * sv + off;
    cp_async_elem(CE(e, c, s), src);
  }
  if (!du_only) {
    for (int idx = tid; idx < 4 * NS * TC * TL; idx += nt) {
      const int s = idx % TL, rest = idx / TL;
      const int c = rest % TC, q = rest / TC;
      const int n = q / 4, kind = q % 4;
      const int i = i0 + s;
      if (col0 + c >= ncol || i >= nl || (kind == 1 && first)) continue;
      const int64_t o = n * sv + cbs[c] + i;
      const T* src = kind == 0 ? b.s + o
                               : (kind == 1 ? b.s0 + o : (kind == 2 ? b.r + o : b.D + 5 * sv + o));
      cp_async_elem(CE(eS + q, c, s), src);
    }
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  for (int idx = tid; idx < TC * TL; idx += nt) {
    const int s = idx % TL, c = idx / TL;
    const int i = i0 + s;
    if (col0 + c >= ncol || i >= nl) continue;
    const int64_t off = cbs[c] + i;
    const int xi = g.il + i;
    const double sum_a2 = zs[c] + zs[2 * TC + c];
    const double b_dry = zs[TC + c] + zs[3 * TC + c];
    const double rhok = vic_full(b, (double)*CE(eRHO, c, s), IDN, xi);
    const double etk = *CE(eDU, c, s);
    const double ai = rhok * g.vol;
    const double fix = DL(0, c, s) - etk;
    double du[5];
    du[IDN] = etk + fix * 1. + rhok * ai * b_dry / sum_a2;
    if constexpr (N == 3) {
      du[IVX] = DL(1, c, s);
      du[IVY] = *CE(eDU + 1, c, s);
      du[IVZ] = *CE(eDU + 2, c, s);
      du[IPR] = DL(2, c, s);
    } else {
#pragma unroll
      for (int v = 1; v < 5; ++v) du[v] = DL(v, c, s);
    }
    if (b.M) b.M[IDN * sv + off] = fix;
    if (du_only) {
#pragma unroll
      for (int v = 0; v < 5; ++v) vic_set_d(b, v * sv + off, du[v]);
      continue;
    }
    double unew_rho = 0.;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const double uo = *CE(eU + v, c, s), u0o = first ? 0. : (double)*CE(eU0 + v, c, s);
      const double un = vic_rk_from(b.u, b.u0, v * sv + off, first, uo, u0o, b.wgt0, b.wgt1,
                                    b.wgt2, du[v]);
      if (v == IDN) unew_rho = vic_full_rho(b, un, xi);
    }
#pragma unroll
    for (int n = 0; n < NS; ++n) {
      const int64_t o = n * sv + off;
      const double so = *CE(eS + 4 * n, c, s);
      const double s0o = first ? 0. : (double)*CE(eS + 4 * n + 1, c, s);
      const double ro = *CE(eS + 4 * n + 2, c, s), dso = *CE(eS + 4 * n + 3, c, s);
      const double ds = dso + fix * ro;
      const double sn = vic_rk_from(b.s, b.s0, o, first, so, s0o, b.wgt0, b.wgt1, b.wgt2, ds);
      b.r[o] = sn / unew_rho;
    }
  }
  __syncthreads();  // the staging area is refilled by the next sub-tile
}

// ---------------------------------------------------------------------------
// One tile: columns [tile * TC, tile * TC + TC) of the block, whole CTA
// (VicCfg<N>::NT threads).  sm: dynamic shared memory of vic_smem_bytes().
// ---------------------------------------------------------------------------
template <int N, int NS, class B>
__device__ __forceinline__ void vic_tile(const Geo& g, const Phys& p, const B& b, int64_t tile,
                                         double* sm) {
  using C = VicCfg<N>;
  constexpr int TC = C::TC, K = C::K, PW = C::PW, NN = C::NN, RE = C::RE, ES = C::ES;
  constexpr int BD = C::BD, BE = C::BE;
  constexpr size_t region = (vic_smem_bytes<N, NS, StoredT<B>>() - C::fixed_bytes) / sizeof(double);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nl = g.nx1;
  const int64_t sv = g.sv;
  const int64_t ncol = (int64_t)(g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  const int64_t col0 = tile * TC;
  double* S = b.vic + tile * (int64_t)nl * ES * TC;  // this tile's records [nl][ES][TC]
  double* ring = sm;                                 // [2 buf][2 end][K][RE][TC]
  double* midb = sm + region;                        // [ES][TC]
  double* xmid = midb + (size_t)ES * TC;             // [N][TC]
  double* zs = xmid + (size_t)N * TC;                // [4][TC]: sum_a2, b_dry per chain
  int64_t* cbs = reinterpret_cast<int64_t*>(zs + 4 * TC);  // [TC]
  if (tid < TC) cbs[tid] = col0 + tid < ncol ? column_base(g, col0 + tid) : 0;
  __syncthreads();
  const int m = nl / 2;                      // middle layer; the bottom end owns 0..m
  const int nch = (m + 1 + K - 1) / K;       // chunks (the top end has nl-1-m <= m+1 layers)
  const double dt = *b.dt;
  const bool colok = col0 + lane < ncol;
  auto RG = [&](int buf, int end, int k) -> double* {
    return ring + ((size_t)((buf * 2 + end) * K + k) * RE) * TC + lane;
  };
  auto produce = [&](int ch) {
    const int pw = warp - 2, end = pw / PW, ph = pw % PW;
    if (!colok) return;
    const int64_t cb = cbs[lane];
#pragma unroll
    for (int k = ph; k < K; k += PW) {
      const int j = ch * K + k;
      const int i = end == 0 ? j : nl - 1 - j;
      if (end == 0 ? (j > m) : (i <= m)) continue;
      vic_layer_blocks<N, B>(g, p, b, cb, i, nl, dt, RG(ch & 1, end, k));
    }
  };
  // (1) + (2): chunk ch is consumed while chunk ch + 1 is formed
  double rb[N][N], rd[N];  // last reduced block and partial solution of this chain
  if (warp >= 2) produce(0);
  __syncthreads();
  for (int ch = 0; ch < nch; ++ch) {
    if (warp < 2) {
      if (colok) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
          const int j = ch * K + k;
          const int i = warp == 0 ? j : nl - 1 - j;
          if (warp == 0 ? (i >= m) : (i <= m)) continue;
          const double* src = RG(ch & 1, warp, k);
          double a[N][N], bb[N][N], cc[N][N], r[N];
#pragma unroll
          for (int x = 0; x < N; ++x) {
#pragma unroll
            for (int q = 0; q < N; ++q) {
              a[x][q] = src[(x * N + q) * TC];
              bb[x][q] = src[(NN + x * N + q) * TC];
              cc[x][q] = src[(2 * NN + x * N + q) * TC];
            }
            r[x] = src[(3 * NN + x) * TC];
          }
          if (warp == 0) {
            // bottom-up (ForwardSweep): a'_i = (a_i - b_i a'_{i-1})^-1 c_i
            if (i > 0) vic_eliminate<N>(a, r, bb, rb, rd);
            block_solve<N>(a, cc, r);
#pragma unroll
            for (int x = 0; x < N; ++x)
#pragma unroll
              for (int q = 0; q < N; ++q) rb[x][q] = cc[x][q];
          } else {
            // top-down: b'_i = (a_i - c_i b'_{i+1})^-1 b_i
            if (i < nl - 1) vic_eliminate<N>(a, r, cc, rb, rd);
            block_solve<N>(a, bb, r);
#pragma unroll
            for (int x = 0; x < N; ++x)
#pragma unroll
              for (int q = 0; q < N; ++q) rb[x][q] = bb[x][q];
          }
          double* rec = S + (int64_t)i * ES * TC + lane;
#pragma unroll
          for (int x = 0; x < N; ++x) {
            rd[x] = r[x];
            rec[(NN + x) * TC] = r[x];
#pragma unroll
            for (int q = 0; q < N; ++q) rec[(x * N + q) * TC] = rb[x][q];
          }
        }
      }
    } else if (ch + 1 < nch) {
      produce(ch + 1);
    }
    __syncthreads();
  }
  // the middle layer: its row couples both reduced systems
  if (warp == 1 && colok && m < nl - 1) {
#pragma unroll
    for (int x = 0; x < N; ++x) {
      midb[(NN + x) * TC + lane] = rd[x];
#pragma unroll
      for (int q = 0; q < N; ++q) midb[(x * N + q) * TC + lane] = rb[x][q];
    }
  }
  __syncthreads();
  if (warp == 0 && colok) {
    const double* src = RG((m / K) & 1, 0, m % K);  // chunk nch-1, never overwritten
    double a[N][N], bb[N][N], cc[N][N], r[N], z[N][N];
#pragma unroll
    for (int x = 0; x < N; ++x) {
#pragma unroll
      for (int q = 0; q < N; ++q) {
        a[x][q] = src[(x * N + q) * TC];
        bb[x][q] = src[(NN + x * N + q) * TC];
        cc[x][q] = src[(2 * NN + x * N + q) * TC];
        z[x][q] = 0.;
      }
      r[x] = src[(3 * NN + x) * TC];
    }
    if (m > 0) vic_eliminate<N>(a, r, bb, rb, rd);
    if (m < nl - 1) {
      double tb[N][N], td[N];
#pragma unroll
      for (int x = 0; x < N; ++x) {
        td[x] = midb[(NN + x) * TC + lane];
#pragma unroll
        for (int q = 0; q < N; ++q) tb[x][q] = midb[(x * N + q) * TC + lane];
      }
      vic_eliminate<N>(a, r, cc, tb, td);
    }
    block_solve<N>(a, z, r);
    double* rec = S + (int64_t)m * ES * TC + lane;
#pragma unroll
    for (int x = 0; x < N; ++x) {
      rd[x] = r[x];
      rec[(NN + x) * TC] = r[x];
      xmid[x * TC + lane] = r[x];
    }
  }
  __syncthreads();
  // (3) back substitution outwards from the middle, with the column sums
  // sum (rho V)^2 and B_dry = sum (du[IDN] - delta_0) V of each chain; each
  // layer's record, du[IDN] and w[IDN] arrive BD layers ahead through a
  // per-thread cp.async ring (in the shared region, the chunks being spent)
  if (warp < 2) {
    double sa2 = 0., bdry = 0.;
    if (colok) {
      const int64_t cb = cbs[lane];
      const int dir = warp == 0 ? -1 : 1;
      const int ifirst = warp == 0 ? m : m + 1;
      const int cnt = warp == 0 ? m + 1 : nl - 1 - m;
      double* br = sm + (size_t)warp * BD * BE * 32;
      auto slot_at = [&](int slot, int e) { return br + ((size_t)(slot * BE + e) * 32 + lane); };
      auto fetch = [&](int t, int slot) {
        if (t < cnt) {
          const int i = ifirst + dir * t;
          const double* rec = S + (int64_t)i * ES * TC + lane;
#pragma unroll
          for (int e = 0; e < ES; ++e) cp_async_bytes8(slot_at(slot, e), rec + e * TC);
          cp_async_elem(slot_at(slot, ES), b.D + IDN * sv + cb + i);
          cp_async_elem(slot_at(slot, ES + 1), b.w + IDN * sv + cb + i);
        }
        cp_async_commit();
      };
#pragma unroll
      for (int t = 0; t < BD; ++t) fetch(t, t);
      double xp[N];
#pragma unroll
      for (int x = 0; x < N; ++x) xp[x] = warp == 0 ? rd[x] : xmid[x * TC + lane];
      const double V = g.vol;
      for (int t = 0, slot = 0; t < cnt; ++t) {
        cp_async_wait<BD - 1>();  // the group of step t has landed
        const int i = ifirst + dir * t;
        double cur[ES];
#pragma unroll
        for (int e = 0; e < ES; ++e) cur[e] = *slot_at(slot, e);
        const double du0 = ring_elem(slot_at(slot, ES), b.D);
        const double rho = vic_full(b, ring_elem(slot_at(slot, ES + 1), b.w), IDN, g.il + i);
        fetch(t + BD, slot);  // the slot's values are in registers: refill it
        slot = slot + 1 == BD ? 0 : slot + 1;
        double x[N];
        if (warp == 0 && t == 0) {
#pragma unroll
          for (int r = 0; r < N; ++r) x[r] = xp[r];  // the middle layer itself
        } else {
#pragma unroll
          for (int r = 0; r < N; ++r) {
            double s = 0.;
#pragma unroll
            for (int q = 0; q < N; ++q) s += cur[r * N + q] * xp[q];
            x[r] = cur[NN + r] - s;
          }
          double* rec = S + (int64_t)i * ES * TC + lane;
#pragma unroll
          for (int r = 0; r < N; ++r) rec[(NN + r) * TC] = x[r];
        }
        const double ai = rho * V;
        sa2 += ai * ai;
        bdry += (du0 - x[0]) * 1. * V;
#pragma unroll
        for (int r = 0; r < N; ++r) xp[r] = x[r];
      }
      cp_async_wait<0>();
    }
    zs[(2 * warp) * TC + lane] = sa2;
    zs[(2 * warp + 1) * TC + lane] = bdry;
  }
  __syncthreads();
  // (4) the tile's cells
  using F = VicFin<N, NS, StoredT<B>>;
  for (int i0 = 0; i0 < nl; i0 += F::TL)
    vic_finish_subtile<N, NS, B>(g, b, S, zs, cbs, col0, ncol, i0, sm);
}

template <int N, int NS, class B>
__global__ void __launch_bounds__(VicCfg<N>::NT, N == 3 ? 2 : 1) k_vicf(Geo g, Phys p, B b) {
  extern __shared__ __align__(16) double vic_smem[];
  vic_tile<N, NS, B>(g, p, b, (int64_t)blockIdx.x, vic_smem);
}

template <int N, int NS, class B>
static cudaError_t launch_vic_ns(const Geo& g, const Phys& p, const B& b, cudaStream_t st) {
  const int64_t ncol = (int64_t)(g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  const int64_t tiles = (ncol + VicCfg<N>::TC - 1) / VicCfg<N>::TC;
  constexpr size_t smem = vic_smem_bytes<N, NS, StoredT<B>>();
  raise_smem_limit(k_vicf<N, NS, B>, smem);
  k_vicf<N, NS, B><<<(unsigned)tiles, VicCfg<N>::NT, smem, st>>>(g, p, b);
  return cudaGetLastError();
}

template <int N, class B>
static cudaError_t launch_vic_n(const Geo& g, const Phys& p, const B& b, cudaStream_t st) {
  switch (p.nscalar) {
    case 0: return launch_vic_ns<N, 0, B>(g, p, b, st);
    case 1: return launch_vic_ns<N, 1, B>(g, p, b, st);
    case 2: return launch_vic_ns<N, 2, B>(g, p, b, st);
    case 3: return launch_vic_ns<N, 3, B>(g, p, b, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace fused

cudaError_t launch_vicf(const Geo& g, const Phys& p, const StageBufs& b, cudaStream_t st) {
  using namespace fused;
  if (vic_n(p) == 5) return launch_vic_n<5>(g, p, b, st);
  return launch_vic_n<3>(g, p, b, st);
}

cudaError_t launch_vicf32(const Geo& g, const Phys& p, const StageBufs32& b, cudaStream_t st) {
  using namespace fused;
  if (vic_n(p) == 5) return launch_vic_n<5>(g, p, b, st);
  return launch_vic_n<3>(g, p, b, st);
}

namespace fused {

// ---- persistent batched variant (ensemble members, FP32 form) ----
// Work items: the 32-column tiles of every member.  Each member's result is
// bit-identical to snapb_stage_f32 on that member alone (same tile function).
template <int N, int NS>
__global__ void __launch_bounds__(VicCfg<N>::NT, N == 3 ? 2 : 1)
    k_vicf_batch(const Member32* __restrict__ mem, Phys p, WorkQueue q, int stage) {
  // the member's descriptor is read from shared memory as the tile needs its
  // fields rather than held in registers
  __shared__ Member32 s_mem;
  extern __shared__ __align__(16) double vic_smem[];
  int m;
  int64_t tile;
  while (queue_next(q, m, tile)) {  // (starts with a barrier: the last tile is done)
    load_member(s_mem, mem, m);
    if (threadIdx.x == 0) set_stage32(s_mem.b, stage);
    __syncthreads();
    vic_tile<N, NS, StageBufs32>(s_mem.g, p, s_mem.b, tile, vic_smem);
  }
}

template <int N, int NS>
static cudaError_t launch_vic_batch_ns(const Member32* mem, const Phys& p, const WorkQueue& q,
                                       int stage, const PersistGrid& pg, cudaStream_t st) {
  constexpr size_t smem = vic_smem_bytes<N, NS, float>();
  raise_smem_limit(k_vicf_batch<N, NS>, smem);
  const int grid = persistent_grid(k_vicf_batch<N, NS>, VicCfg<N>::NT, smem, pg);
  k_vicf_batch<N, NS><<<grid, VicCfg<N>::NT, smem, st>>>(mem, p, q, stage);
  return cudaGetLastError();
}

}  // namespace fused

cudaError_t launch_vicf_batch(const Member32* mem, const Phys& p, const WorkQueue& q, int stage,
                              const PersistGrid& pg, cudaStream_t st) {
  using namespace fused;
#define SNAPB_VB(NV)                                                          \
  switch (p.nscalar) {                                                        \
    case 0: return launch_vic_batch_ns<NV, 0>(mem, p, q, stage, pg, st);      \
    case 1: return launch_vic_batch_ns<NV, 1>(mem, p, q, stage, pg, st);      \
    case 2: return launch_vic_batch_ns<NV, 2>(mem, p, q, stage, pg, st);      \
    case 3: return launch_vic_batch_ns<NV, 3>(mem, p, q, stage, pg, st);      \
    default: return cudaErrorInvalidValue;                                    \
  }
  if (vic_n(p) == 5) {
    SNAPB_VB(5)
  }
  SNAPB_VB(3)
#undef SNAPB_VB
}

int vicf_tile_columns() { return fused::VicCfg<3>::TC; }

size_t vicf_scratch_bytes(const Geo& g, const Phys& p) { return fused::scratch_bytes(g, p); }

}  // namespace snapb


