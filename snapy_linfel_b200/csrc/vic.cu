// vic.cu — vertically implicit correction (VIC) of one RK stage, FP64.
//
// Two kernels per solve:
//   k_vic_column    one thread per x1 column (x1 is the vertical axis): the
//                   blocks are formed on the fly while the column is swept —
//                   the Roe-averaged |A| = R |Lambda| R^-1 once per interface
//                   (the reference forms it twice, once per neighbouring cell)
//                   and the flux Jacobian once per cell, a layer ahead of the
//                   elimination that consumes them (formed in the iteration
//                   that eliminates the layer below, so the two independent
//                   dependency chains interleave) — then the block-Thomas
//                   elimination, back substitution and the MS-VIC column
//                   sums.  Only the reduced blocks and the partial solutions
//                   go through HBM;
//   k_vic_finish    per cell: mass redistribution, scalar mass fix and the RK
//                   combination (or du), with delta transposed through shared
//                   memory.
// Every workspace array is laid out with the column index fastest, so the
// sequential sweep's loads and stores are coalesced across a warp's columns.
//
// Reference: ImplicitHydroImpl::forward (src/implicit/implicit_hydro.cpp:99-189),
// vic_assemble_partial_impl (src/implicit/vic_assemble_partial_impl.h:29-111),
// vic_assemble_full_impl (src/implicit/vic_assemble_full_impl.h:16-106),
// ForwardSweep (src/implicit/forward_sweep_impl.h:20-109), ludcmp/lubksb
// (src/math/ludcmp.h:24-76, src/math/lubksb.h:124-147),
// vic_backward_reduce / vic_redistribute_cell (src/implicit/vic_redistribute_impl.h:26-106),
// flux Jacobian and Roe eigenvectors (src/implicit/flux_decomposition_impl.h:133-245).
#include <cstdlib>
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

// ---------------------------------------------------------------------------
// Scratch layout (doubles, column index fastest so that the threads of a warp,
// one column each, read consecutive addresses):
//   S [nl][N*N+N][ncol]  the reduced blocks a'_i then the partial solutions
//                        delta_i (back-substituted in place)
//   Z [2][ncol]          per-column sums: sum (rho V)^2 and B_dry
// ---------------------------------------------------------------------------

size_t vic_column_scratch_bytes(const Geo& g, const Phys& p) {
  if (p.implicit_scheme == 0) return 0;
  int N = vic_n(p);
  int64_t ncol = (int64_t)(g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  int64_t nl = g.nx1;
  int64_t es = N * N + N;
  return (size_t)(nl * es * ncol + 2 * ncol) * sizeof(double);
}

// workspace share of the implicit solve: room for either variant (the column
// + finish pair here, or the fused kernel of vicf.cu)
size_t vic_scratch_bytes(const Geo& g, const Phys& p) {
  const size_t a = vic_column_scratch_bytes(g, p), b = vicf_scratch_bytes(g, p);
  return a > b ? a : b;
}

// Few columns (2-D domains, thin 3-D ones) leave most of the GPU idle with one
// thread per column: the blocks |A| (per face) and J (per cell) are then
// formed by a fully parallel kernel first, so the sequential sweep only
// eliminates.  Scratch T [nl+2][2 N*N][ncol]: index t holds |A| of the face
// between cells t-1 and t, and J of cell t-1.
constexpr int64_t kSplitMaxCols = 8192;

bool vic_split(const Geo& g, const Phys& p) {
  const int64_t ncol = (int64_t)(g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  return p.implicit_scheme != 0 && ncol <= kSplitMaxCols;
}

size_t vic_blocks_bytes(const Geo& g, const Phys& p) {
  if (!vic_split(g, p)) return 0;
  int N = vic_n(p);
  int64_t ncol = (int64_t)(g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  return (size_t)((int64_t)(g.nx1 + 2) * 2 * N * N * ncol) * sizeof(double);
}

constexpr int kTC = 32;           // columns per tile
constexpr int kFinThreads = 256;  // threads of a finish CTA

// Back substitution: the reduced block, partial solution and du[IDN] of a
// layer are fetched kBackDepth<N> layers ahead into a per-thread ring in
// shared memory by asynchronous copies (cp.async), so the short recurrence
// does not wait a memory latency per layer and holds no extra registers.
// Ring layout [slot][element][thread] (element ES = du[IDN]), doubles.
constexpr int kFwdDepth = 4;  // layers of the forward sweep in flight

template <int N>
struct BackRing {
  static constexpr int depth = N == 3 ? 4 : 2;
  static constexpr int elems = N * N + N + 1;
};
template <int N>
constexpr size_t back_ring_bytes(int threads) {
  return (size_t)threads * BackRing<N>::depth * BackRing<N>::elems * sizeof(double);
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
// Precision of the blocks (|A|, J and the assembled a, b, c) per form: FP64
// for the FP64 plain form, FP32 for the FP32 perturbation form, whose states
// are FP32.  The elimination, the back substitution and the scratch stay FP64
// in both forms: the assembled blocks are widened before they enter it.
template <class B>
struct BlockPrec {
  using T = double;
};
template <>
struct BlockPrec<StageBufs32> {
  using T = float;
};
template <int N>
__device__ __forceinline__ void absA_of(const StageBufs32&, double gm1, const double* wl,
                                        const double* wr, float (&A)[N][N]) {
  float fl[5], fr[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    fl[v] = (float)wl[v];
    fr[v] = (float)wr[v];
  }
  absA_block<N, float>((float)gm1, fl, fr, A);
}
template <int N>
__device__ __forceinline__ void jac_of(const StageBufs32&, double gm1, const double* w,
                                       float (&J)[N][N]) {
  float fw[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) fw[v] = (float)w[v];
  jac_block<N, float>((float)gm1, fw, J);
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
// the same from full states already rounded to FP32
template <int N>
__device__ __forceinline__ void absA_of(const StageBufs32&, double gm1, const float* wl,
                                        const float* wr, float (&A)[N][N]) {
  absA_block<N, float>((float)gm1, wl, wr, A);
}
template <int N>
__device__ __forceinline__ void jac_of(const StageBufs32&, double gm1, const float* w,
                                       float (&J)[N][N]) {
  jac_block<N, float>((float)gm1, w, J);
}

// One layer of the block-Thomas forward elimination: a_i, b_i, c_i from |A|
// at the layer's lower / upper faces (Am, Ap) and J of the cells below /
// above (Jp, Jn); the previous reduced block and partial solution (ap, dp)
// are eliminated, and c (reduced block) and rhs (partial solution) return the
// new ones.  Used by the split sweep; the fused sweep (vic_column) spells out
// the same arithmetic inline.
template <int N, class BT>
__device__ __forceinline__ void vic_layer(const BT (&Am)[N][N], const BT (&Ap)[N][N],
                                          const BT (&Jp)[N][N], const BT (&Jn)[N][N],
                                          const double (&ap)[N][N], const double (&dp)[N],
                                          double (&rhs)[N], double (&c)[N][N], int i, int nl,
                                          double Aa, double hiv, double idt, double grav) {
  double a[N][N], bb[N][N];
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
  block_solve<N>(a, c, rhs);
}

// Back substitution delta_i -= a'_i delta_{i+1} and the MS-VIC column sums
// (sum (rho V)^2 from the forward sweep, B_dry accumulated here); the inputs
// of each layer arrive through the thread's shared-memory ring.
template <int N, class B>
__device__ __forceinline__ void vic_back(const B& b, double* S, double* Z, int64_t ncol,
                                         int64_t sv, int64_t cb, int nl, const double (&dp)[N],
                                         double sum_a2, double V) {
  constexpr int ES = VicDims<N>::ES;
  constexpr int DB = BackRing<N>::depth, RE = BackRing<N>::elems;
  extern __shared__ double vic_ring[];
  const int nt = blockDim.x, lane = threadIdx.x;
  auto Sat = [&](int i, int e) -> double& { return S[((int64_t)i * ES + e) * ncol]; };
  cp_async_wait<0>();  // the forward ring is drained before its memory is reused
  auto ring = [&](int slot, int e) { return vic_ring + ((size_t)(slot * RE + e) * nt + lane); };
  auto fetch = [&](int i, int slot) {
    if (i >= 0) {
#pragma unroll
      for (int e = 0; e < ES; ++e) cp_async_bytes8(ring(slot, e), &Sat(i, e));
      cp_async_elem(ring(slot, ES), b.D + IDN * sv + cb + i);
    }
    cp_async_commit();
  };
  double dn[N];
#pragma unroll
  for (int r = 0; r < N; ++r) dn[r] = dp[r];
  double b_dry = (vic_d(b, IDN * sv + cb + nl - 1) - dn[0]) * 1. * V;
#pragma unroll
  for (int k = 0; k < DB; ++k) fetch(nl - 2 - k, k);
  for (int i = nl - 2, slot = 0; i >= 0; --i) {
    cp_async_wait<DB - 1>();  // the group of layer i has landed
    double cur[ES];
#pragma unroll
    for (int e = 0; e < ES; ++e) cur[e] = *ring(slot, e);
    const double dcur = ring_elem(ring(slot, ES), b.D);
    double d[N];
#pragma unroll
    for (int r = 0; r < N; ++r) {
      double t = 0.;
#pragma unroll
      for (int q = 0; q < N; ++q) t += cur[r * N + q] * dn[q];
      d[r] = cur[N * N + r] - t;
    }
    b_dry += (dcur - d[0]) * 1. * V;
    fetch(i - DB, slot);  // the slot's values are consumed: refill it
    slot = slot + 1 == DB ? 0 : slot + 1;
#pragma unroll
    for (int r = 0; r < N; ++r) {
      dn[r] = d[r];
      Sat(i, N * N + r) = d[r];
    }
  }
  cp_async_wait<0>();
  Z[0] = sum_a2;
  Z[ncol] = b_dry;
}

// (1) one thread per column: blocks formed a layer ahead of the
// block-Thomas elimination, back substitution and the column sums.  Loads of
// a layer's w and du go 32 columns apart across a warp; the next layers of
// each column sit in the same 32-byte sectors, which stay in L1.
template <int N, class B>
__device__ __forceinline__ void vic_column(const Geo& g, const Phys& p, const B& b, int64_t col) {
  constexpr int ES = VicDims<N>::ES;
  using BT = typename BlockPrec<B>::T;  // precision of the blocks and their assembly
  const int64_t ncol = (int64_t)(g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  if (col >= ncol) return;
  const int nl = g.nx1;
  const int64_t sv = g.sv;
  const int64_t cb = column_base(g, col);
  double* S = b.vic + col;
  double* Z = S + (int64_t)nl * ES * ncol;
  auto Sat = [&](int i, int e) -> double& { return S[((int64_t)i * ES + e) * ncol]; };
  // full primitives of a cell in the block precision, with the full density
  // in FP64 beside them (the column sum)
  auto load_w = [&](int i, BT* w, double& rho) {
    rho = vic_w(b, sv, IDN, cb + i, g.il + i);
    w[IDN] = (BT)rho;
#pragma unroll
    for (int v = 1; v < 5; ++v) w[v] = (BT)vic_w(b, sv, v, cb + i, g.il + i);
  };
  const double gm1c = p.gammad - 1.;
  const double gm1f = 0.5 * (p.gammad + p.gammad) - 1.;
  const double dt = *b.dt, idtd = 1. / dt;
  const double V = g.vol;
  const BT Aa = (BT)g.A1, hiv = (BT)(0.5 / g.vol), idt = (BT)(1. / dt), grav = (BT)p.grav1;
  // Forward sweep inputs of iteration i — w of cell i+2 (for the blocks of
  // layer i+1) and the rows of du at layer i — arrive kFwdDepth iterations
  // ahead through the same per-thread shared-memory ring as the back
  // substitution, layout [slot][element][thread].  The blocks of layer i+1
  // (|A| at its upper face, J of the cell above it) are formed in iteration i,
  // beside the elimination of layer i that does not depend on them, so the
  // two dependency chains interleave.
  constexpr int DF = kFwdDepth, FE = 5 + N;
  static_assert(DF * FE <= BackRing<N>::depth * BackRing<N>::elems, "ring too small");
  extern __shared__ double vic_ring[];
  const int nt = blockDim.x, lane = threadIdx.x;
  auto fring = [&](int slot, int e) { return vic_ring + ((size_t)(slot * FE + e) * nt + lane); };
  auto ffetch = [&](int i, int slot) {
    if (i < nl) {
      const int L = min(i + 2, nl);  // cell nl is the ghost above the column
#pragma unroll
      for (int v = 0; v < 5; ++v) cp_async_elem(fring(slot, v), b.w + v * sv + cb + L);
#pragma unroll
      for (int r = 0; r < N; ++r)
        cp_async_elem(fring(slot, 5 + r), b.D + sel<N>(r) * sv + cb + i);
    }
    cp_async_commit();
  };
#pragma unroll
  for (int k = 0; k < DF; ++k) ffetch(k, k);
  BT wc[5], wn[5], wn2[5];
  double rc, rn, rn2;
  BT Am[N][N], Jp[N][N], Jc[N][N], Ap[N][N], Jn[N][N];
  // (the first elimination step uses no previous layer: zeros keep it branch-free)
  double ap[N][N] = {}, dp[N] = {};
  load_w(-1, wn, rn);
  jac_of<N>(b, gm1c, wn, Jp);
  load_w(0, wc, rc);
  absA_of<N>(b, gm1f, wn, wc, Am);
  jac_of<N>(b, gm1c, wc, Jc);
  load_w(min(1, nl), wn, rn);  // cell 1 (the ghost cell nl when nl = 1)
  absA_of<N>(b, gm1f, wc, wn, Ap);
  jac_of<N>(b, gm1c, wn, Jn);
  double sum_a2 = 0.;
  for (int i = 0, fslot = 0; i < nl; ++i) {
    double rhs[N];
    cp_async_wait<DF - 1>();  // the group of iteration i has landed
    {
      const int xi = g.il + min(i + 2, nl);
      rn2 = vic_full(b, (double)ring_stored(fring(fslot, IDN), b.w), IDN, xi);
      wn2[IDN] = (BT)rn2;
#pragma unroll
      for (int v = 1; v < 5; ++v) wn2[v] = vic_full_blk(b, ring_stored(fring(fslot, v), b.w), v, xi);
    }
#pragma unroll
    for (int r = 0; r < N; ++r) rhs[r] = ring_elem(fring(fslot, 5 + r), b.D) * idtd;
    // blocks of layer i+1 (unused after the last layer)
    BT Apn[N][N], Jnn[N][N];
    absA_of<N>(b, gm1f, wn, wn2, Apn);
    jac_of<N>(b, gm1c, wn2, Jnn);
    double ai = rc * V;
    sum_a2 += ai * ai;
    // assembly in the block precision, then widened for the elimination
    BT af[N][N], bf[N][N], cf[N][N];
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
      for (int q = 0; q < N; ++q) {
        BT phi = BT(0);
        if (r == 1 && q == 0) phi = grav;
        if (N == 3 && r == 2 && q == 1) phi = grav;
        if (N == 5 && r == IPR && q == IVX) phi = grav;
        af[r][q] = (Am[r][q] * Aa + Ap[r][q] * Aa) * hiv - phi;
        bf[r][q] = -(Am[r][q] + Jp[r][q]) * Aa * hiv;
        cf[r][q] = -(Ap[r][q] - Jn[r][q]) * Aa * hiv;
      }
#pragma unroll
    for (int r = 0; r < N; ++r) af[r][r] += idt;
    // boundary folds of the first and last layers, branch-free (weight 0
    // elsewhere, which adds an exact zero)
    const BT f0 = i == 0 ? BT(1) : BT(0), f1 = i == nl - 1 ? BT(1) : BT(0);
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
      for (int q = 0; q < N; ++q) {
        af[r][q] += bf[r][q] * (q == 1 ? -f0 : f0);
        af[r][q] += cf[r][q] * (q == 1 ? -f1 : f1);
      }
    double a[N][N], bb[N][N], c[N][N];
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
      for (int q = 0; q < N; ++q) {
        a[r][q] = (double)af[r][q];
        bb[r][q] = (double)bf[r][q];
        c[r][q] = (double)cf[r][q];
      }
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
    block_solve<N>(a, c, rhs);
    // the slot's values are consumed (the solve depends on them): refill it
    ffetch(i + DF, fslot);
    fslot = fslot + 1 == DF ? 0 : fslot + 1;
#pragma unroll
    for (int r = 0; r < N; ++r) {
      dp[r] = rhs[r];
      __stcs(&Sat(i, N * N + r), rhs[r]);
#pragma unroll
      for (int q = 0; q < N; ++q) {
        ap[r][q] = c[r][q];
        __stcs(&Sat(i, r * N + q), c[r][q]);
      }
    }
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
      for (int q = 0; q < N; ++q) {
        Am[r][q] = Ap[r][q];
        Jp[r][q] = Jc[r][q];
        Jc[r][q] = Jn[r][q];
        Ap[r][q] = Apn[r][q];
        Jn[r][q] = Jnn[r][q];
      }
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      wc[v] = wn[v];
      wn[v] = wn2[v];
    }
    rc = rn;
    rn = rn2;
  }
  // back substitution: delta_i -= a'_i delta_{i+1}; B_dry accumulated on the
  // way, the inputs of each layer arriving through the shared-memory ring.
  constexpr int DB = BackRing<N>::depth, RE = BackRing<N>::elems;
  cp_async_wait<0>();  // the forward ring is drained before its memory is reused
  auto ring = [&](int slot, int e) { return vic_ring + ((size_t)(slot * RE + e) * nt + lane); };
  auto fetch = [&](int i, int slot) {
    if (i >= 0) {
#pragma unroll
      for (int e = 0; e < ES; ++e) cp_async_bytes8(ring(slot, e), &Sat(i, e));
      cp_async_elem(ring(slot, ES), b.D + IDN * sv + cb + i);
    }
    cp_async_commit();
  };
  double dn[N];
#pragma unroll
  for (int r = 0; r < N; ++r) dn[r] = dp[r];
  double b_dry = (vic_d(b, IDN * sv + cb + nl - 1) - dn[0]) * 1. * V;
#pragma unroll
  for (int k = 0; k < DB; ++k) fetch(nl - 2 - k, k);
  for (int i = nl - 2, slot = 0; i >= 0; --i) {
    cp_async_wait<DB - 1>();  // the group of layer i has landed
    double cur[ES];
#pragma unroll
    for (int e = 0; e < ES; ++e) cur[e] = *ring(slot, e);
    const double dcur = ring_elem(ring(slot, ES), b.D);
    double d[N];
#pragma unroll
    for (int r = 0; r < N; ++r) {
      double t = 0.;
#pragma unroll
      for (int q = 0; q < N; ++q) t += cur[r * N + q] * dn[q];
      d[r] = cur[N * N + r] - t;
    }
    b_dry += (dcur - d[0]) * 1. * V;
    fetch(i - DB, slot);  // the slot's values are consumed: refill it
    slot = slot + 1 == DB ? 0 : slot + 1;
#pragma unroll
    for (int r = 0; r < N; ++r) {
      dn[r] = d[r];
      Sat(i, N * N + r) = d[r];
    }
  }
  cp_async_wait<0>();
  Z[0] = sum_a2;
  Z[ncol] = b_dry;
}

// ---- split sweep (few columns): blocks first, then the elimination ----
template <int N>
struct PreRing {
  static constexpr int elems = 2 * N * N + N + 1;  // A_{i+1}, J_{i+2}, du rows, rho
};
template <int N>
constexpr size_t pre_ring_bytes(int threads) {
  return (size_t)threads * sizeof(double) *
         (kFwdDepth * PreRing<N>::elems > BackRing<N>::depth * BackRing<N>::elems
              ? kFwdDepth * PreRing<N>::elems
              : BackRing<N>::depth * BackRing<N>::elems);
}

// one thread per (column, t), t in [0, nl+1], column fastest (coalesced stores)
template <int N>
__global__ void __launch_bounds__(256) k_vic_blocks(Geo g, Phys p, StageBufs b) {
  constexpr int NN = N * N;
  const int64_t ncol = (int64_t)(g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  const int nl = g.nx1;
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= ncol * (nl + 2)) return;
  const int64_t col = idx - (int64_t)udiv(idx, ncol) * ncol;
  const int t = udiv(idx, ncol);
  const int64_t sv = g.sv, cb = column_base(g, col);
  const double gm1c = p.gammad - 1.;
  const double gm1f = 0.5 * (p.gammad + p.gammad) - 1.;
  double wl[5], wr[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) wl[v] = b.w[v * sv + cb + t - 1];
  double* out = b.vicT + (int64_t)t * 2 * NN * ncol + col;
  double J[N][N];
  jac_of<N>(b, gm1c, wl, J);
#pragma unroll
  for (int r = 0; r < N; ++r)
#pragma unroll
    for (int q = 0; q < N; ++q) out[(NN + r * N + q) * ncol] = J[r][q];
  if (t <= nl) {
#pragma unroll
    for (int v = 0; v < 5; ++v) wr[v] = b.w[v * sv + cb + t];
    double A[N][N];
    absA_of<N>(b, gm1f, wl, wr, A);
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
      for (int q = 0; q < N; ++q) out[(r * N + q) * ncol] = A[r][q];
  }
}

// the elimination of one column from the precomputed blocks
template <int N>
__global__ void __launch_bounds__(128) k_vic_column_pre(Geo g, Phys p, StageBufs b) {
  constexpr int ES = VicDims<N>::ES, NN = N * N, DF = kFwdDepth, FE = PreRing<N>::elems;
  const int64_t ncol = (int64_t)(g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  const int64_t col = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncol) return;
  const int nl = g.nx1;
  const int64_t sv = g.sv;
  const int64_t cb = column_base(g, col);
  double* S = b.vic + col;
  double* Z = S + (int64_t)nl * ES * ncol;
  auto Sat = [&](int i, int e) -> double& { return S[((int64_t)i * ES + e) * ncol]; };
  const double* T = b.vicT + col;
  auto Tat = [&](int t, int e) { return T + ((int64_t)t * 2 * NN + e) * ncol; };
  extern __shared__ double vic_ring[];
  const int nt = blockDim.x, lane = threadIdx.x;
  auto fring = [&](int slot, int e) { return vic_ring + ((size_t)(slot * FE + e) * nt + lane); };
  auto ffetch = [&](int i, int slot) {  // layer i: A_{i+1}, J_{i+2}, du rows and rho of cell i
    if (i < nl) {
#pragma unroll
      for (int e = 0; e < NN; ++e) cp_async_bytes8(fring(slot, e), Tat(i + 1, e));
#pragma unroll
      for (int e = 0; e < NN; ++e) cp_async_bytes8(fring(slot, NN + e), Tat(i + 2, NN + e));
#pragma unroll
      for (int r = 0; r < N; ++r)
        cp_async_bytes8(fring(slot, 2 * NN + r), b.D + sel<N>(r) * sv + cb + i);
      cp_async_bytes8(fring(slot, 2 * NN + N), b.w + IDN * sv + cb + i);
    }
    cp_async_commit();
  };
#pragma unroll
  for (int k = 0; k < DF; ++k) ffetch(k, k);
  const double dt = *b.dt;
  const double Aa = g.A1, hiv = 0.5 / g.vol, idt = 1. / dt, grav = p.grav1, V = g.vol;
  double Am[N][N], Jp[N][N], Jc[N][N], ap[N][N], dp[N];
#pragma unroll
  for (int r = 0; r < N; ++r)
#pragma unroll
    for (int q = 0; q < N; ++q) {
      Am[r][q] = *Tat(0, r * N + q);
      Jp[r][q] = *Tat(0, NN + r * N + q);
      Jc[r][q] = *Tat(1, NN + r * N + q);
      ap[r][q] = 0.;
    }
#pragma unroll
  for (int r = 0; r < N; ++r) dp[r] = 0.;
  double sum_a2 = 0.;
  for (int i = 0, fslot = 0; i < nl; ++i) {
    double Ap[N][N], Jn[N][N], rhs[N];
    cp_async_wait<DF - 1>();  // the group of layer i has landed
#pragma unroll
    for (int r = 0; r < N; ++r) {
      rhs[r] = *fring(fslot, 2 * NN + r) / dt;
#pragma unroll
      for (int q = 0; q < N; ++q) {
        Ap[r][q] = *fring(fslot, r * N + q);
        Jn[r][q] = *fring(fslot, NN + r * N + q);
      }
    }
    const double ai = *fring(fslot, 2 * NN + N) * V;
    sum_a2 += ai * ai;
    double c[N][N];
    vic_layer<N>(Am, Ap, Jp, Jn, ap, dp, rhs, c, i, nl, Aa, hiv, idt, grav);
    ffetch(i + DF, fslot);  // the slot's values are consumed: refill it
    fslot = fslot + 1 == DF ? 0 : fslot + 1;
#pragma unroll
    for (int r = 0; r < N; ++r) {
      dp[r] = rhs[r];
      __stcs(&Sat(i, NN + r), rhs[r]);
#pragma unroll
      for (int q = 0; q < N; ++q) {
        ap[r][q] = c[r][q];
        __stcs(&Sat(i, r * N + q), c[r][q]);
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
  vic_back<N>(b, S, Z, ncol, sv, cb, nl, dp, sum_a2, V);
}

// the ring of a 128-thread CTA exceeds the default 48 KB of dynamic shared
// memory (raise_smem_limit, kernels.cuh)
template <class K>
static void allow_ring_smem(K kernel, size_t bytes) {
  raise_smem_limit(kernel, bytes);
}

template <int N, class B>
__global__ void __launch_bounds__(128) k_vic_column(Geo g, Phys p, B b) {
  vic_column<N, B>(g, p, b, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}

// (3) redistribution + RK combination (or du), tiles of 32 columns x 32
// layers: delta is transposed through shared memory so that the state
// arrays are read and written along x1.
// one tile: columns col0 .. col0+kTC-1, layers i0 .. i0+kTL-1 (whole CTA)
// Shared memory of one finish tile: the back-substituted solution rows
// [N][kTC][kTL+1] (doubles), the column sums and offsets, the layers'
// reference densities, then the tile's cell inputs [element][kTC][kTL] in the
// stored precision T: w'[IDN], the du rows the solve does not replace, and
// (RK update) u, u0, and per scalar s, s0, r and its du row.
template <int N, int NS>
struct FinSmem {
  static constexpr int TL = 16;  // layers per staged tile
  static constexpr int du_rows = N == 3 ? 3 : 1;           // IDN (+ IVY, IVZ)
  static constexpr int elems = 1 + du_rows + 10 + 4 * NS;  // upper bound
  static constexpr size_t head = ((size_t)N * kTC * (TL + 1) + 3 * kTC + TL) * sizeof(double);
};
template <int N, int NS, class T>
constexpr size_t finish_smem_bytes() {
  return FinSmem<N, NS>::head + (size_t)FinSmem<N, NS>::elems * kTC * FinSmem<N, NS>::TL * sizeof(T);
}

// Views of a staged tile's shared memory, in the order above (the reference
// densities are used by the FP32 form only).
template <int N, int NS, class T>
struct FinTile {
  static constexpr int kTL = FinSmem<N, NS>::TL;
  double *dl, *zs, *rbs;
  int64_t* cbs;
  T* cell;
  __device__ __forceinline__ explicit FinTile(double* base) {
    dl = base;
    zs = dl + (size_t)N * kTC * (kTL + 1);
    cbs = reinterpret_cast<int64_t*>(zs + 2 * kTC);
    rbs = reinterpret_cast<double*>(cbs + kTC);
    cell = reinterpret_cast<T*>(rbs + kTL);
  }
  __device__ __forceinline__ double& DL(int r, int c, int s) const {
    return dl[((size_t)r * kTC + c) * (kTL + 1) + s];
  }
  __device__ __forceinline__ T* CE(int e, int c, int s) const {
    return cell + ((size_t)e * kTC + c) * kTL + s;
  }
};

// One tile, columns col0 .. col0+kTC-1, layers i0 .. i0+kTL-1 (whole CTA), in
// two halves.  The issue half fetches every input of the tile with cp.async
// (coalesced: the solution rows along columns, the cell values along x1) and
// commits them as one group, so all of a tile's loads are in flight together
// without holding registers; after the caller's wait and CTA barrier the
// compute half finishes the tile's cells from shared memory.
template <int N, int NS, class B>
__device__ __forceinline__ void vic_finish_issue(const Geo& g, const B& b, int64_t col0, int i0) {
  constexpr int ES = VicDims<N>::ES, kTL = FinSmem<N, NS>::TL;
  constexpr bool kPert = std::is_same_v<B, StageBufs32>;
  using T = std::remove_pointer_t<decltype(b.u)>;  // stored precision (FP32 / FP64)
  const int nl = g.nx1;
  const int64_t ncol = (int64_t)(g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  const int64_t sv = g.sv;
  const double* S = b.vic;
  const double* Z = S + (int64_t)nl * ES * ncol;
  extern __shared__ double fin_smem[];
  const FinTile<N, NS, T> t(fin_smem);
  const bool du_only = b.vic_du_only, first = b.stage == 0;
  constexpr int DR = FinSmem<N, NS>::du_rows;
  const int eRHO = 0, eDU = 1, eU = 1 + DR, eU0 = eU + 5, eS = eU0 + 5;
  const int tid = threadIdx.x;
  if (tid < 2 * kTC) {  // column sums (1 past the last column)
    const int c = tid % kTC, k = tid / kTC;
    if (col0 + c < ncol)
      cp_async_bytes8(&t.zs[k * kTC + c], Z + k * ncol + col0 + c);
    else
      t.zs[k * kTC + c] = 1.;
    if (k == 0) t.cbs[c] = col0 + c < ncol ? column_base(g, col0 + c) : 0;
  }
  if constexpr (kPert)
    if (tid < kTL && i0 + tid < nl) cp_async_bytes8(&t.rbs[tid], b.rb + g.il + i0 + tid);
  // Each thread copies the same CPT cells of every element: their offsets are
  // formed once, and the element loops pick one source array per pass.
  constexpr int CPT = kTC * kTL / kFinThreads;
  static_assert(CPT * kFinThreads == kTC * kTL, "finish tile and CTA shape");
  {  // solution rows, columns fastest (S is [layer][element][column])
    int64_t soff[CPT];
    bool sok[CPT];
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
      const int idx = tid + j * kFinThreads, c = idx % kTC, s = idx / kTC;
      sok[j] = col0 + c < ncol && i0 + s < nl;
      soff[j] = ((int64_t)(i0 + s) * ES + N * N) * ncol + col0 + c;
    }
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
      for (int j = 0; j < CPT; ++j) {
        const int idx = tid + j * kFinThreads;
        if (sok[j]) cp_async_bytes8(&t.DL(r, idx % kTC, idx / kTC), S + soff[j] + (int64_t)r * ncol);
      }
  }
  // cell inputs, layers fastest (the state arrays run along x1)
  int64_t goff[CPT];
  bool gok[CPT];
#pragma unroll
  for (int j = 0; j < CPT; ++j) {
    const int idx = tid + j * kFinThreads, s = idx % kTL, c = idx / kTL;
    gok[j] = col0 + c < ncol && i0 + s < nl;
    goff[j] = gok[j] ? column_base(g, col0 + c) + i0 + s : 0;
  }
  auto stage_elem = [&](int e, const T* base) {
    T* dst = t.CE(e, 0, 0);
#pragma unroll
    for (int j = 0; j < CPT; ++j)
      if (gok[j]) cp_async_elem(dst + tid + j * kFinThreads, base + goff[j]);
  };
  stage_elem(eRHO, b.w + IDN * sv);
  stage_elem(eDU, b.D + IDN * sv);
  if constexpr (N == 3) {
    stage_elem(eDU + 1, b.D + IVY * sv);
    stage_elem(eDU + 2, b.D + IVZ * sv);
  }
  if (!du_only) {
    for (int v = 0; v < 5; ++v) {
      stage_elem(eU + v, b.u + v * sv);
      if (!first) stage_elem(eU0 + v, b.u0 + v * sv);  // u0 is the stage input at stage 0
    }
    for (int n = 0; n < NS; ++n) {
      stage_elem(eS + 4 * n, b.s + n * sv);
      if (!first) stage_elem(eS + 4 * n + 1, b.s0 + n * sv);
      stage_elem(eS + 4 * n + 2, b.r + n * sv);
      stage_elem(eS + 4 * n + 3, b.D + (5 + n) * sv);
    }
  }
  cp_async_commit();
}

template <int N, int NS, class B>
__device__ __forceinline__ void vic_finish_compute(const Geo& g, const Phys& p, const B& b,
                                                   int64_t col0, int i0) {
  constexpr int kTL = FinSmem<N, NS>::TL, DR = FinSmem<N, NS>::du_rows;
  constexpr bool kPert = std::is_same_v<B, StageBufs32>;
  using T = std::remove_pointer_t<decltype(b.u)>;
  const int nl = g.nx1;
  const int64_t ncol = (int64_t)(g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  const int64_t sv = g.sv;
  extern __shared__ double fin_smem[];
  const FinTile<N, NS, T> t(fin_smem);
  const bool du_only = b.vic_du_only, first = b.stage == 0;
  (void)p;
  // element slots; per scalar n: s, s0, r, its du row at eS + 4 n
  const int eRHO = 0, eDU = 1, eU = 1 + DR, eU0 = eU + 5, eS = eU0 + 5;
  for (int idx = threadIdx.x; idx < kTC * kTL; idx += blockDim.x) {
    const int s = idx % kTL, c = idx / kTL;
    const int i = i0 + s;
    if (col0 + c >= ncol || i >= nl) continue;
    const int64_t off = t.cbs[c] + i;
    double rhok = (double)*t.CE(eRHO, c, s);  // full density
    if constexpr (kPert) rhok += t.rbs[s];
    const double etk = *t.CE(eDU, c, s);
    double ai = rhok * g.vol;
    double fix = t.DL(0, c, s) - etk;
    double du[5];
    du[IDN] = etk + fix * 1. + rhok * ai * t.zs[kTC + c] / t.zs[c];
    if constexpr (N == 3) {
      du[IVX] = t.DL(1, c, s);
      du[IVY] = *t.CE(eDU + 1, c, s);
      du[IVZ] = *t.CE(eDU + 2, c, s);
      du[IPR] = t.DL(2, c, s);
    } else {
#pragma unroll
      for (int v = 1; v < 5; ++v) du[v] = t.DL(v, c, s);
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
      const double uo = *t.CE(eU + v, c, s), u0o = first ? 0. : (double)*t.CE(eU0 + v, c, s);
      double un = vic_rk_from(b.u, b.u0, v * sv + off, first, uo, u0o, b.wgt0, b.wgt1, b.wgt2,
                              du[v]);
      if (v == IDN) {
        unew_rho = un;  // full density of the new state
        if constexpr (kPert) unew_rho += t.rbs[s];
      }
    }
#pragma unroll
    for (int n = 0; n < NS; ++n) {
      const int64_t o = n * sv + off;
      const double so = *t.CE(eS + 4 * n, c, s);
      const double s0o = first ? 0. : (double)*t.CE(eS + 4 * n + 1, c, s);
      const double ro = *t.CE(eS + 4 * n + 2, c, s), dso = *t.CE(eS + 4 * n + 3, c, s);
      double ds = dso + fix * ro;
      double sn = vic_rk_from(b.s, b.s0, o, first, so, s0o, b.wgt0, b.wgt1, b.wgt2, ds);
      b.r[o] = sn / unew_rho;
    }
  }
}

template <int N, int NS, class B>
__device__ __forceinline__ void vic_finish_tile_staged(const Geo& g, const Phys& p, const B& b,
                                                       int64_t col0, int i0) {
  vic_finish_issue<N, NS, B>(g, b, col0, i0);
  cp_async_wait<0>();
  __syncthreads();
  vic_finish_compute<N, NS, B>(g, p, b, col0, i0);
}

// Register variant (scalars, or FP64 state: the staged inputs would not fit
// in 48 KB of shared memory and would cut the resident CTAs): each thread
// issues the loads of its cells before any store.
template <int N, int NS, class B, int NT, int kTL>
__device__ __forceinline__ void vic_finish_tile_regs(const Geo& g, const Phys& p, const B& b,
                                                int64_t col0, int i0) {
  constexpr int ES = VicDims<N>::ES;
  const int nl = g.nx1;
  const int64_t ncol = (int64_t)(g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  const int64_t sv = g.sv;
  const double* S = b.vic;
  const double* Z = S + (int64_t)nl * ES * ncol;
  __shared__ double dl[N][kTC][kTL + 1];
  __shared__ double zs[2][kTC];
  __shared__ int64_t cbs[kTC];  // (k, j, il) offsets of the tile's columns
  const int tid = threadIdx.x;
  for (int idx = tid; idx < N * kTC * kTL; idx += blockDim.x) {
    int c = idx % kTC, rest = idx / kTC;
    int s = rest % kTL, r = rest / kTL;
    int64_t col = col0 + c;
    int i = i0 + s;
    dl[r][c][s] = (col < ncol && i < nl) ? S[((int64_t)i * ES + N * N + r) * ncol + col] : 0.;
  }
  if (tid < 2 * kTC) {
    int c = tid % kTC, k = tid / kTC;
    zs[k][c] = col0 + c < ncol ? Z[k * ncol + col0 + c] : 1.;
    if (k == 0) cbs[c] = col0 + c < ncol ? column_base(g, col0 + c) : 0;
  }
  __syncthreads();
  // (2) each thread's kTC kTL / NT cells: every load first (no store in
  // between, so they are all in flight together), then the arithmetic and
  // the stores.  Cells are distinct, so the order is the sequential one's.
  constexpr int IT = kTC * kTL / NT, NSA = NS > 0 ? NS : 1;
  using T = std::remove_pointer_t<decltype(b.u)>;  // stored precision (FP32 / FP64)
  T rho[IT], et[IT], dvy[IT], dvz[IT], uo[IT][5], u0o[IT][5];
  T so[IT][NSA], s0o[IT][NSA], ro[IT][NSA], dso[IT][NSA];
  int64_t offs[IT];
  bool ok[IT];
  const bool du_only = b.vic_du_only, first = b.stage == 0;
#pragma unroll
  for (int k = 0; k < IT; ++k) {
    const int idx = tid + k * NT;
    const int s = idx % kTL, c = idx / kTL;
    const int64_t col = col0 + c;
    const int i = i0 + s;
    ok[k] = col < ncol && i < nl;
    if (!ok[k]) continue;
    const int64_t off = cbs[c] + i;
    offs[k] = off;
    rho[k] = b.w[IDN * sv + off];
    et[k] = b.D[IDN * sv + off];
    if constexpr (N == 3) {
      dvy[k] = b.D[IVY * sv + off];
      dvz[k] = b.D[IVZ * sv + off];
    }
    if (!du_only) {
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        uo[k][v] = b.u[v * sv + off];
        if (!first) u0o[k][v] = b.u0[v * sv + off];
      }
#pragma unroll
      for (int n = 0; n < NS; ++n) {
        const int64_t o = n * sv + off;
        so[k][n] = b.s[o];
        if (!first) s0o[k][n] = b.s0[o];
        ro[k][n] = b.r[o];
        dso[k][n] = b.D[(5 + n) * sv + off];
      }
    }
  }
#pragma unroll
  for (int k = 0; k < IT; ++k) {
    if (!ok[k]) continue;
    const int idx = tid + k * NT;
    const int s = idx % kTL, c = idx / kTL;
    const int64_t off = offs[k];
    const int xi = g.il + i0 + s;
    const double rhok = vic_full(b, (double)rho[k], IDN, xi), etk = et[k];
    double ai = rhok * g.vol;
    double fix = dl[0][c][s] - etk;
    double du[5];
    du[IDN] = etk + fix * 1. + rhok * ai * zs[1][c] / zs[0][c];
    if constexpr (N == 3) {
      du[IVX] = dl[1][c][s];
      du[IVY] = dvy[k];
      du[IVZ] = dvz[k];
      du[IPR] = dl[2][c][s];
    } else {
#pragma unroll
      for (int v = 1; v < 5; ++v) du[v] = dl[v][c][s];
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
      double un = vic_rk_from(b.u, b.u0, v * sv + off, first, uo[k][v], u0o[k][v], b.wgt0,
                              b.wgt1, b.wgt2, du[v]);
      if (v == IDN) unew_rho = vic_full_rho(b, un, xi);
    }
#pragma unroll
    for (int n = 0; n < NS; ++n) {
      const int64_t o = n * sv + off;
      double ds = (double)dso[k][n] + fix * (double)ro[k][n];
      double sn = vic_rk_from(b.s, b.s0, o, first, so[k][n], s0o[k][n], b.wgt0, b.wgt1,
                              b.wgt2, ds);
      b.r[o] = sn / unew_rho;
    }
  }
}

// Which finish variant a form takes, and its launch shape.
template <int N, int NS, class T>
struct FinCfg {
  static constexpr bool staged = finish_smem_bytes<N, NS, T>() <= 48 * 1024;
  static constexpr int threads = kFinThreads;
  static constexpr int layers = staged ? FinSmem<N, NS>::TL : 32;  // tile height
  static constexpr int min_ctas = staged ? 4 : 2;  // register budget of the batched kernel
  // one-block kernel: two resident CTAs for FP32 state (its register
  // variant sits just above 128 registers uncapped, which would leave one);
  // FP64 state keeps the compiler's budget (capping it spills)
  static constexpr int min_ctas_single = staged ? 4 : (sizeof(T) == 4 ? 2 : 1);
  static constexpr size_t smem = staged ? finish_smem_bytes<N, NS, T>() : 0;
};
template <class B>
using StoredT = std::remove_pointer_t<decltype(std::declval<B>().u)>;

template <int N, int NS, class B>
__device__ __forceinline__ void vic_finish_tile(const Geo& g, const Phys& p, const B& b,
                                                int64_t col0, int i0) {
  using C = FinCfg<N, NS, StoredT<B>>;
  if constexpr (C::staged)
    vic_finish_tile_staged<N, NS, B>(g, p, b, col0, i0);
  else
    vic_finish_tile_regs<N, NS, B, C::threads, C::layers>(g, p, b, col0, i0);
}

template <int N, int NS, class B>
__global__ void __launch_bounds__(FinCfg<N, NS, StoredT<B>>::threads,
                                  FinCfg<N, NS, StoredT<B>>::min_ctas_single) k_vic_finish(Geo g, Phys p, B b) {
  vic_finish_tile<N, NS, B>(g, p, b, (int64_t)blockIdx.x * kTC,
                            (int)blockIdx.y * FinCfg<N, NS, StoredT<B>>::layers);
}

template <int N, class B>
static cudaError_t launch_vic_n(const Geo& g, const Phys& p, const B& b, cudaStream_t st) {
  const int64_t ncol = (int64_t)(g.ju - g.jl + 1) * (g.ku - g.kl + 1);
  const int nl = g.nx1;
  // small column counts: narrower CTAs spread the sequential sweeps over more SMs
  int bs = ncol >= 148 * 128 ? 128 : (ncol >= 148 * 64 ? 64 : 32);
  bool split = false;
  if constexpr (std::is_same_v<B, StageBufs>) split = b.vicT != nullptr;
  if constexpr (std::is_same_v<B, StageBufs>) {
    if (split) {
      const int64_t nb = ncol * (nl + 2);
      k_vic_blocks<N><<<(unsigned)((nb + 255) / 256), 256, 0, st>>>(g, p, b);
      allow_ring_smem(k_vic_column_pre<N>, pre_ring_bytes<N>(128));
      k_vic_column_pre<N><<<(unsigned)((ncol + bs - 1) / bs), bs, pre_ring_bytes<N>(bs), st>>>(
          g, p, b);
    }
  }
  if (!split) {
    allow_ring_smem(k_vic_column<N, B>, back_ring_bytes<N>(128));
    k_vic_column<N, B><<<(unsigned)((ncol + bs - 1) / bs), bs, back_ring_bytes<N>(bs), st>>>(
        g, p, b);
  }
  using T = std::remove_pointer_t<decltype(b.u)>;
#define SNAPB_VF(NS)                                                   \
  case NS: {                                                           \
    using FC = FinCfg<N, NS, T>;                                       \
    dim3 gf((unsigned)((ncol + kTC - 1) / kTC),                        \
            (unsigned)((nl + FC::layers - 1) / FC::layers));           \
    if (FC::smem) allow_ring_smem(k_vic_finish<N, NS, B>, FC::smem);   \
    k_vic_finish<N, NS, B><<<gf, FC::threads, FC::smem, st>>>(g, p, b); \
  } break;
  switch (p.nscalar) {
    SNAPB_VF(0)
    SNAPB_VF(1)
    SNAPB_VF(2)
    SNAPB_VF(3)
    default: return cudaErrorInvalidValue;
  }
#undef SNAPB_VF
  return cudaGetLastError();
}

// Variant of the implicit solve, from the environment (read at every launch):
// the column + finish pair by default; SNAPB_VIC_KERNEL=fused selects the
// fused kernel of vicf.cu, =cr block cyclic reduction (vic_cr.cu, FP32 form,
// where it applies).
static const char* vic_kernel_env() {
  const char* v = std::getenv("SNAPB_VIC_KERNEL");
  return v ? v : "";
}
static bool vic_fused_selected() { return std::strcmp(vic_kernel_env(), "fused") == 0; }
static bool vic_cr_selected() { return std::strcmp(vic_kernel_env(), "cr") == 0; }

cudaError_t launch_vic_column(const Geo& g, const Phys& p, const StageBufs& b,
                              cudaStream_t st) {
  if (vic_n(p) == 5) return launch_vic_n<5>(g, p, b, st);
  return launch_vic_n<3>(g, p, b, st);
}

cudaError_t launch_vic(const Geo& g, const Phys& p, const StageBufs& b, cudaStream_t st) {
  if (vic_fused_selected()) return launch_vicf(g, p, b, st);
  return launch_vic_column(g, p, b, st);
}

cudaError_t launch_vic32(const Geo& g, const Phys& p, const StageBufs32& b, cudaStream_t st) {
  if (vic_fused_selected()) return launch_vicf32(g, p, b, st);
  if (vic_cr_selected() && vic_cr_applies(g, p)) return launch_vic_cr32(g, p, b, st);
  if (vic_n(p) == 5) return launch_vic_n<5>(g, p, b, st);
  return launch_vic_n<3>(g, p, b, st);
}

// ---- persistent batched variants (ensemble members, FP32 form) ----
// V selects the register budget: 0 = compiler's choice, 1 = at least 3 CTAs of
// 128 threads per SM (~168 registers), 2 = 4 CTAs (128 registers, some spill)
template <int N, int V>
__global__ void __launch_bounds__(128, V == 0 ? 1 : (V == 1 ? 3 : 4))
    k_vic_column_batch(const Member32* __restrict__ mem, Phys p, WorkQueue q, int stage) {
  // The member's descriptor is read from shared memory as the sweep needs its
  // fields instead of being copied into registers (~50 of them) for the tile
  // (for the sweeps of stage32.cu the compiler hoists those reads and spills).
  __shared__ Member32 s_mem;
  int m;
  int64_t tile;
  while (queue_next(q, m, tile)) {  // (starts with a barrier: the last tile is done)
    load_member(s_mem, mem, m);
    const int64_t col = tile * s_mem.vic_cols + threadIdx.x;
    if ((int)threadIdx.x < s_mem.vic_cols) vic_column<N, StageBufs32>(s_mem.g, p, s_mem.b, col);
  }
  (void)stage;
}

// Batched finish.  Staged tiles run as a pipeline: while a tile's inputs are
// in flight, warp 0 claims the next work item and, when it belongs to another
// member, copies that member's descriptor into the second descriptor buffer,
// so the only latency between two tiles of a CTA is the tile's own loads.
template <int N, int NS>
__global__ void __launch_bounds__(FinCfg<N, NS, float>::threads,
                                  FinCfg<N, NS, float>::min_ctas) k_vic_finish_batch(const Member32* __restrict__ mem,
                                                          Phys p, WorkQueue q, int stage) {
  using FC = FinCfg<N, NS, float>;
  constexpr int TLY = FC::layers;
  // descriptors of the current and the next tile's member, read as needed
  // (see the column kernel)
  __shared__ Member32 s_mem[2];
  if constexpr (!FC::staged) {
    int m;
    int64_t tile;
    while (queue_next(q, m, tile)) {  // (starts with a barrier: the last tile is done)
      load_member(s_mem[0], mem, m);
      if (threadIdx.x == 0) set_stage32(s_mem[0].b, stage);
      __syncthreads();
      const int nlb = (s_mem[0].g.nx1 + TLY - 1) / TLY;
      const int64_t cb = tile / nlb;
      const int lb = (int)(tile - cb * nlb);
      vic_finish_tile<N, NS, StageBufs32>(s_mem[0].g, p, s_mem[0].b, cb * kTC, lb * TLY);
    }
  } else {
    __shared__ unsigned long long s_item;
    const int tid = threadIdx.x;
    if (tid == 0) s_item = atomicAdd(q.counter, 1ULL);
    __syncthreads();
    int m;
    int64_t tile;
    if (!queue_find(q, (int64_t)s_item, m, tile)) return;
    if (tid < 32) {
      load_member_warp(s_mem[0], mem, m);
      if (tid == 0) set_stage32(s_mem[0].b, stage);
    }
    __syncthreads();
    int buf = 0;
    while (true) {
      const Member32& cur = s_mem[buf];
      const int nlb = (cur.g.nx1 + TLY - 1) / TLY;
      const int64_t cb = tile / nlb;
      const int lb = (int)(tile - cb * nlb);
      vic_finish_issue<N, NS, StageBufs32>(cur.g, cur.b, cb * kTC, lb * TLY);
      if (tid < 32) {  // the next item, and its member's descriptor if that changes
        unsigned long long it = 0;
        if (tid == 0) it = atomicAdd(q.counter, 1ULL);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (tid == 0) s_item = it;
        int nm;
        int64_t nt;
        if (queue_find(q, (int64_t)it, nm, nt) && nm != m) {
          const int* src = reinterpret_cast<const int*>(mem + nm);
          int* dst = reinterpret_cast<int*>(&s_mem[buf ^ 1]);
          for (int k = tid; k < (int)(sizeof(Member32) / sizeof(int)); k += 32)
            cp_async_bytes4(dst + k, src + k);
        }
        cp_async_commit();
      }
      cp_async_wait<0>();
      __syncthreads();  // the tile's inputs, the next item and its descriptor are in place
      int nm;
      int64_t ntile;
      const bool more = queue_find(q, (int64_t)s_item, nm, ntile);
      const int nbuf = more && nm != m ? buf ^ 1 : buf;
      if (tid == 0 && nbuf != buf) set_stage32(s_mem[nbuf].b, stage);
      vic_finish_compute<N, NS, StageBufs32>(cur.g, p, cur.b, cb * kTC, lb * TLY);
      if (!more) return;
      __syncthreads();  // the tile's shared memory is free; s_item is read
      buf = nbuf;
      m = nm;
      tile = ntile;
    }
  }
}

template <int N, int V>
static void launch_vcb(const Member32* mem, const Phys& p, const WorkQueue& q, int stage,
                       const PersistGrid& pg, int block, cudaStream_t st) {
  const size_t smem = back_ring_bytes<N>(block);
  allow_ring_smem(k_vic_column_batch<N, V>, back_ring_bytes<N>(128));
  k_vic_column_batch<N, V><<<persistent_grid(k_vic_column_batch<N, V>, block, smem, pg), block,
                             smem, st>>>(mem, p, q, stage);
}

cudaError_t launch_vic_column_batch(const Member32* mem, const Phys& p, const WorkQueue& q,
                                    int stage, const PersistGrid& pg, int block, int variant,
                                    cudaStream_t st) {
  const bool five = vic_n(p) == 5;
  switch (variant) {
    case 1: five ? launch_vcb<5, 1>(mem, p, q, stage, pg, block, st)
                 : launch_vcb<3, 1>(mem, p, q, stage, pg, block, st); break;
    case 2: five ? launch_vcb<5, 2>(mem, p, q, stage, pg, block, st)
                 : launch_vcb<3, 2>(mem, p, q, stage, pg, block, st); break;
    default: five ? launch_vcb<5, 0>(mem, p, q, stage, pg, block, st)
                  : launch_vcb<3, 0>(mem, p, q, stage, pg, block, st);
  }
  return cudaGetLastError();
}

// finish tile height of the FP32 form (the batched plan sizes its tiles with it)
template <int N>
static int finish_layers32(int nscalar) {
  switch (nscalar) {
    case 0: return FinCfg<N, 0, float>::layers;
    case 1: return FinCfg<N, 1, float>::layers;
    case 2: return FinCfg<N, 2, float>::layers;
    default: return FinCfg<N, 3, float>::layers;
  }
}
int vic_finish_layers32(const Phys& p) {
  return vic_n(p) == 5 ? finish_layers32<5>(p.nscalar) : finish_layers32<3>(p.nscalar);
}

cudaError_t launch_vic_finish_batch(const Member32* mem, const Phys& p, const WorkQueue& q,
                                    int stage, const PersistGrid& pg, cudaStream_t st) {
  static_assert(kTC == kVicFinishCols, "finish tile shape");
#define SNAPB_VFB(N, NS)                                                                  \
  {                                                                                       \
    using FC = FinCfg<N, NS, float>;                                                      \
    if (FC::smem) allow_ring_smem(k_vic_finish_batch<N, NS>, FC::smem);                   \
    k_vic_finish_batch<N, NS><<<persistent_grid(k_vic_finish_batch<N, NS>, FC::threads,   \
                                                FC::smem, pg),                            \
                                FC::threads, FC::smem, st>>>(mem, p, q, stage);           \
  }
  if (vic_n(p) == 5) {
    switch (p.nscalar) {
      case 0: SNAPB_VFB(5, 0); break;
      case 1: SNAPB_VFB(5, 1); break;
      case 2: SNAPB_VFB(5, 2); break;
      case 3: SNAPB_VFB(5, 3); break;
      default: return cudaErrorInvalidValue;
    }
  } else {
    switch (p.nscalar) {
      case 0: SNAPB_VFB(3, 0); break;
      case 1: SNAPB_VFB(3, 1); break;
      case 2: SNAPB_VFB(3, 2); break;
      case 3: SNAPB_VFB(3, 3); break;
      default: return cudaErrorInvalidValue;
    }
  }
#undef SNAPB_VFB
  return cudaGetLastError();
}

}  // namespace snapb

// ---------------------------------------------------------------------------
// Implicit correction without any allocation.
//
// Some callers cannot allocate device memory when they need this solve: code
// running inside a CUDA-graph capture or a stream-ordered region where
// cudaMalloc would break the capture, embedded hosts whose memory is fully
// pre-partitioned, and foreign-language callers that hold no allocator handle
// (no torch, no CUDA context helper).  For them the solve's scratch lives in
// a fixed array in the library's own device global memory instead of the
// caller's workspace.  Every GPU that loads the library holds this array
// (kNoAllocScratchBytes) until the process exits.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB
static __device__ __align__(256) double
    g_noalloc_vic_scratch[kNoAllocScratchBytes / sizeof(double)];

// Device address of g_noalloc_vic_scratch on the current device.  In host code
// the array's name only stands in for the symbol, so the address is looked up
// with cudaGetSymbolAddress once per device (with that device current) and
// cached for the life of the process.  The cache is not invalidated by
// cudaDeviceReset; the header tells callers not to use this entry point after
// resetting a device in the same process.
cudaError_t noalloc_scratch(double** out) {
  static std::mutex mu;
  static double* addr[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_vic_scratch);
    if (e != cudaSuccess) return e;
    addr[dev] = static_cast<double*>(p);
  }
  *out = addr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" int snapb_implicit_correction_noalloc(const snapb_hydro_config* cfg, const double* dt,
                                                 double* du, const double* w, double* mass_corr,
                                                 void* stream) {
  using namespace snapb;
  if (const char* e = internal_check_config(cfg))
    return internal_fail(SNAPB_ERR_ARG, std::string("implicit_correction_noalloc: ") + e);
  if (cfg->implicit_scheme == 0) return SNAPB_OK;  // null operation
  if (!dt || !du || !w)
    return internal_fail(SNAPB_ERR_ARG, "implicit_correction_noalloc: null pointer");
  Geo g = make_geo(*cfg);
  Phys p = make_phys(*cfg);
  p.nscalar = 0;
  size_t need = vic_column_scratch_bytes(g, p);
  if (need > kNoAllocScratchBytes)
    return internal_fail(SNAPB_ERR_ARG,
                         "implicit_correction_noalloc: the column solve needs " +
                             std::to_string(need) + " bytes of scratch (nx1 * columns * (N*N+N) * 8)"
                             " but the built-in buffer holds " +
                             std::to_string(kNoAllocScratchBytes) +
                             " bytes; use snapb_implicit_correction with a workspace");
  double* scratch = nullptr;
  cudaError_t e = noalloc_scratch(&scratch);
  if (e != cudaSuccess)
    return internal_fail(SNAPB_ERR_CUDA, std::string("implicit_correction_noalloc: symbol address: ") +
                                             cudaGetErrorString(e));
  // The solve writes every scratch entry before it reads it, so nothing has
  // to be cleared between calls.
  StageBufs b;
  std::memset(&b, 0, sizeof(b));
  b.dt = dt;
  b.w = const_cast<double*>(w);
  b.D = du;
  b.M = mass_corr;
  b.vic = scratch;
  b.vic_du_only = 1;
  e = launch_vic_column(g, p, b, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess)
    return internal_fail(SNAPB_ERR_CUDA, std::string("implicit_correction_noalloc: ") +
                                             cudaGetErrorString(e));
  return SNAPB_OK;
}
