// vic_blocks.cuh — the local blocks of the vertically implicit system,
// templated on the scalar type (double, or the Dual of dual.cuh in the
// adjoint): the x1 flux Jacobian dF/dU of a cell and |A| = R |Lambda| R^-1 at
// the Roe average of an interface
// (src/implicit/flux_decomposition_impl.h:133-245), and the block solve of
// the elimination (src/math/ludcmp.h:24-76, src/math/lubksb.h:124-147).
#pragma once

#include "common.cuh"

namespace snapb {

// rows / columns of the 5x5 system kept by the N-block form: N = 3 keeps
// (IDN, IVX, IPR), N = 5 keeps everything
template <int N>
__device__ __forceinline__ int sel(int r) {
  if constexpr (N == 3) return r == 2 ? IPR : r;
  return r;
}

// N x N block of the x1 flux Jacobian dF/dU at primitive state w
template <int N, class T>
__device__ __forceinline__ void jac_block(T gm1, const T* w, T (&J)[N][N]) {
  T v1 = w[IVX], v2 = w[IVY], v3 = w[IVZ], rho = w[IDN], pres = w[IPR];
  T s2 = v1 * v1 + v2 * v2 + v3 * v3;
  T hp = fdiv(fdiv(gm1 + T(1), gm1) * pres, rho);
  T c1 = ((gm1 - T(1)) * s2 / T(2) - hp) * v1;
  T c2 = hp + s2 / T(2) - gm1 * v1 * v1;
  T full[5][5] = {{T(0.), T(1.), T(0.), T(0.), T(0.)},
                  {gm1 * s2 / T(2) - v1 * v1, (T(2.) - gm1) * v1, -gm1 * v2, -gm1 * v3, gm1},
                  {-v1 * v2, v2, v1, T(0.), T(0.)},
                  {-v1 * v3, v3, T(0.), v1, T(0.)},
                  {c1, c2, -gm1 * v2 * v1, -gm1 * v3 * v1, (gm1 + T(1)) * v1}};
#pragma unroll
  for (int r = 0; r < N; ++r)
#pragma unroll
    for (int q = 0; q < N; ++q) J[r][q] = full[sel<N>(r)][sel<N>(q)];
}

// N x N block of |A| = R |Lambda| R^-1 at the Roe average of (wl, wr)
template <int N, class T>
__device__ __forceinline__ void absA_block(T gm1, const T* wl, const T* wr, T (&A)[N][N]) {
  T sdl = sqrt(wl[IDN]), sdr = sqrt(wr[IDN]);
  T isd = fdiv(T(1.0), sdl + sdr);
  T r = sdl * sdr;
  T u = (sdl * wl[IVX] + sdr * wr[IVX]) * isd;
  T v = (sdl * wl[IVY] + sdr * wr[IVY]) * isd;
  T w = (sdl * wl[IVZ] + sdr * wr[IVZ]) * isd;
  T el = fdiv(wl[IPR], gm1) + T(0.5) * wl[IDN] * (sqr(wl[IVX]) + sqr(wl[IVY]) + sqr(wl[IVZ]));
  T er = fdiv(wr[IPR], gm1) + T(0.5) * wr[IDN] * (sqr(wr[IVX]) + sqr(wr[IVY]) + sqr(wr[IVZ]));
  T hbar = (fdiv(el + wl[IPR], sdl) + fdiv(er + wr[IPR], sdr)) * isd;
  T p = fdiv((hbar - T(0.5) * (u * u + v * v + w * w)) * gm1, gm1 + T(1.)) * r;
  T cs = sqrt(fdiv(p * (gm1 + T(1.)), r));
  T lam[5] = {fabs(u - cs), fabs(u), fabs(u + cs), fabs(u), fabs(u)};
  T ke = T(0.5) * (u * u + v * v + w * w);
  T hp = fdiv(fdiv(gm1 + T(1.), gm1) * p, r);
  T h = hp + ke;
  T i2chp = fdiv(T(1.), T(2.) * cs * hp), ihp = fdiv(T(1.), hp), i2hp = T(0.5) * ihp;
  T R[5][5] = {{T(1.), T(1.), T(1.), T(0.), T(0.)},
               {u - cs, u, u + cs, T(0.), T(0.)},
               {v, v, v, T(1.), T(0.)},
               {w, w, w, T(0.), T(1.)},
               {h - u * cs, ke, h + u * cs, v, w}};
  T Ri[5][5] = {{(cs * ke + u * hp) * i2chp, (-hp - cs * u) * i2chp, -v * i2hp, -w * i2hp, i2hp},
                {(hp - ke) * ihp, u * ihp, v * ihp, w * ihp, -ihp},
                {(cs * ke - u * hp) * i2chp, (hp - cs * u) * i2chp, -v * i2hp, -w * i2hp, i2hp},
                {-v, T(0.), T(1.), T(0.), T(0.)},
                {-w, T(0.), T(0.), T(1.), T(0.)}};
#pragma unroll
  for (int a = 0; a < N; ++a)
#pragma unroll
    for (int b = 0; b < N; ++b) {
      int ra = sel<N>(a), cb = sel<N>(b);
      T s = T(0.);
#pragma unroll
      for (int k = 0; k < 5; ++k) s += (R[ra][k] * lam[k]) * Ri[k][cb];
      A[a][b] = s;
    }
}


// cofactor inverse of a 3 x 3 block
template <class T>
__device__ __forceinline__ void inverse3(const T (&M)[3][3], T (&inv)[3][3]) {
  auto cof = [&](int i, int j) {
    int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
    return M[i1][j1] * M[i2][j2] - M[i1][j2] * M[i2][j1];
  };
  T c00 = cof(0, 0), c10 = cof(1, 0), c20 = cof(2, 0);
  T det = c00 * M[0][0] + c10 * M[1][0] + c20 * M[2][0];
  T id = T(1) / det;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) inv[i][j] = cof(j, i) * id;
}

// [C | rhs] <- inv [C | rhs] for a 3 x 3 inverse
template <class T>
__device__ __forceinline__ void apply_inverse3(const T (&inv)[3][3], T (&C)[3][3], T (&rhs)[3]) {
  T x[3], X[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    x[i] = inv[i][0] * rhs[0] + inv[i][1] * rhs[1] + inv[i][2] * rhs[2];
#pragma unroll
    for (int j = 0; j < 3; ++j)
      X[i][j] = inv[i][0] * C[0][j] + inv[i][1] * C[1][j] + inv[i][2] * C[2][j];
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    rhs[i] = x[i];
#pragma unroll
    for (int j = 0; j < 3; ++j) C[i][j] = X[i][j];
  }
}

// X = M^-1 [C | rhs] for an N x N block: cofactor inverse for N = 3,
// LU with implicit-scaling partial pivoting (Crout) for N = 5
template <int N, class T>
__device__ __forceinline__ void block_solve(T (&M)[N][N], T (&C)[N][N], T (&rhs)[N]) {
  if constexpr (N == 3) {
    T inv[3][3];
    inverse3(M, inv);
    apply_inverse3(inv, C, rhs);
  } else {
    T vv[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
      T big = T(0);
#pragma unroll
      for (int j = 0; j < N; ++j) big = fmax(big, fabs(M[i][j]));
      vv[i] = T(1) / big;
    }
    int indx[N];
#pragma unroll
    for (int j = 0; j < N; ++j) {
#pragma unroll
      for (int i = 0; i < j; ++i) {
        T s = M[i][j];
#pragma unroll
        for (int k = 0; k < i; ++k) s -= M[i][k] * M[k][j];
        M[i][j] = s;
      }
      T big = T(0);
      int imax = j;
#pragma unroll
      for (int i = j; i < N; ++i) {
        T s = M[i][j];
#pragma unroll
        for (int k = 0; k < j; ++k) s -= M[i][k] * M[k][j];
        M[i][j] = s;
        T d = vv[i] * fabs(s);
        if (d >= big) {
          big = d;
          imax = i;
        }
      }
      // row swap j <-> imax done with selects so the arrays stay in registers
#pragma unroll
      for (int i = j + 1; i < N; ++i) {
        if (i == imax) {
#pragma unroll
          for (int k = 0; k < N; ++k) {
            T t = M[i][k];
            M[i][k] = M[j][k];
            M[j][k] = t;
          }
          T t = vv[i];
          vv[i] = vv[j];
          vv[j] = t;
        }
      }
      indx[j] = imax;
      if (j != N - 1) {
        T d = T(1) / M[j][j];
#pragma unroll
        for (int i = j + 1; i < N; ++i) M[i][j] *= d;
      }
    }
    // forward / back substitution on the N+1 columns [C | rhs]
#pragma unroll
    for (int i = 0; i < N; ++i) {
      int ip = indx[i];
#pragma unroll
      for (int r2 = i + 1; r2 < N; ++r2) {
        if (r2 == ip) {
#pragma unroll
          for (int c = 0; c < N; ++c) {
            T t = C[r2][c];
            C[r2][c] = C[i][c];
            C[i][c] = t;
          }
          T t = rhs[r2];
          rhs[r2] = rhs[i];
          rhs[i] = t;
        }
      }
#pragma unroll
      for (int j = 0; j < i; ++j) {
#pragma unroll
        for (int c = 0; c < N; ++c) C[i][c] -= M[i][j] * C[j][c];
        rhs[i] -= M[i][j] * rhs[j];
      }
    }
#pragma unroll
    for (int i = N - 1; i >= 0; --i) {
#pragma unroll
      for (int j = i + 1; j < N; ++j) {
#pragma unroll
        for (int c = 0; c < N; ++c) C[i][c] -= M[i][j] * C[j][c];
        rhs[i] -= M[i][j] * rhs[j];
      }
      T d = T(1) / M[i][i];
#pragma unroll
      for (int c = 0; c < N; ++c) C[i][c] *= d;
      rhs[i] *= d;
    }
  }
}

}  // namespace snapb
