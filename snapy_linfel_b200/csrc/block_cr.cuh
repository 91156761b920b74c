// block_cr.cuh — block cyclic reduction of a block-tridiagonal system with
// 3 x 3 blocks held in shared memory, solved by one CTA, FP64.
//
// Layer i's equation is Bl_i x_{i-1} + Dg_i x_i + Ab_i x_{i+1} = R_i (Bl_0 and
// Ab_{nl-1} zero).  At stride s the equations i with i % 2s == s are
// eliminated from their neighbours i +- s (3x3 cofactor inverses, the 3x3
// solve of block_solve), until equation 0 alone is left; then the solutions
// are filled in back down the strides.  The solve overwrites the blocks and
// leaves x in R.  It eliminates the same system as a block-Thomas sweep in
// another order, so the two agree up to FP64 rounding.
#pragma once

namespace snapb {

// X = M^-1 (3x3 cofactor inverse, in place), the 3x3 solve of block_solve
__device__ __forceinline__ void inv3_inplace(double* M) {
  auto m = [&](int i, int j) { return M[i * 3 + j]; };
  auto cof = [&](int i, int j) {
    const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
    return m(i1, j1) * m(i2, j2) - m(i1, j2) * m(i2, j1);
  };
  const double c00 = cof(0, 0), c10 = cof(1, 0), c20 = cof(2, 0);
  const double det = c00 * m(0, 0) + c10 * m(1, 0) + c20 * m(2, 0);
  const double id = 1. / det;
  double inv[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) inv[i * 3 + j] = cof(j, i) * id;
#pragma unroll
  for (int k = 0; k < 9; ++k) M[k] = inv[k];
}

// P = -X Y (3x3)
__device__ __forceinline__ void neg_mul33(const double* X, const double* Y, double* P) {
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int q = 0; q < 3; ++q)
      P[r * 3 + q] = -(X[r * 3] * Y[q] + X[r * 3 + 1] * Y[3 + q] + X[r * 3 + 2] * Y[6 + q]);
}
// Z += X Y (3x3), z += X y
__device__ __forceinline__ void add_mul33(const double* X, const double* Y, double* Z) {
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int q = 0; q < 3; ++q)
      Z[r * 3 + q] += X[r * 3] * Y[q] + X[r * 3 + 1] * Y[3 + q] + X[r * 3 + 2] * Y[6 + q];
}
__device__ __forceinline__ void add_mul31(const double* X, const double* y, double* z) {
#pragma unroll
  for (int r = 0; r < 3; ++r) z[r] += X[r * 3] * y[0] + X[r * 3 + 1] * y[1] + X[r * 3 + 2] * y[2];
}

// sum over the CTA (all threads call it); red: 2 doubles per warp of scratch
__device__ __forceinline__ void cta_sum2(double& x, double& y, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    x += __shfl_xor_sync(0xffffffffu, x, o);
    y += __shfl_xor_sync(0xffffffffu, y, o);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0) {
    red[2 * wid] = x;
    red[2 * wid + 1] = y;
  }
  __syncthreads();
  x = 0.;
  y = 0.;
  for (int k = 0; k < nw; ++k) {  // the same order on every thread
    x += red[2 * k];
    y += red[2 * k + 1];
  }
}

// Solve the system of nl layers in place (the whole CTA calls it; it ends
// with a CTA barrier).  Bl, Dg, Ab: [nl][9] row-major blocks; R: [nl][3].
__device__ __forceinline__ void block_cr3_solve(double* Bl, double* Dg, double* Ab, double* R,
                                                int nl) {
  const int tid = threadIdx.x, nt = blockDim.x;
  int s = 1;
  for (; s < nl; s <<= 1) {
    const int s2 = 2 * s;
    for (int j = s + tid * s2; j < nl; j += nt * s2) inv3_inplace(Dg + j * 9);
    __syncthreads();
    for (int i = tid * s2; i < nl; i += nt * s2) {
      double Dn[9], Rn[3];
#pragma unroll
      for (int k = 0; k < 9; ++k) Dn[k] = Dg[i * 9 + k];
#pragma unroll
      for (int r = 0; r < 3; ++r) Rn[r] = R[i * 3 + r];
      const int lo = i - s, hi = i + s;
      if (lo >= 0) {  // eliminate x_lo: alpha = -b_i a_lo^-1
        double al[9], Bn[9];
        neg_mul33(Bl + i * 9, Dg + lo * 9, al);
        add_mul33(al, Ab + lo * 9, Dn);
        add_mul31(al, R + lo * 3, Rn);
#pragma unroll
        for (int k = 0; k < 9; ++k) Bn[k] = 0.;
        add_mul33(al, Bl + lo * 9, Bn);
#pragma unroll
        for (int k = 0; k < 9; ++k) Bl[i * 9 + k] = Bn[k];
      }
      if (hi < nl) {  // eliminate x_hi: beta = -c_i a_hi^-1
        double be[9], Cn[9];
        neg_mul33(Ab + i * 9, Dg + hi * 9, be);
        add_mul33(be, Bl + hi * 9, Dn);
        add_mul31(be, R + hi * 3, Rn);
#pragma unroll
        for (int k = 0; k < 9; ++k) Cn[k] = 0.;
        add_mul33(be, Ab + hi * 9, Cn);
#pragma unroll
        for (int k = 0; k < 9; ++k) Ab[i * 9 + k] = Cn[k];
      }
#pragma unroll
      for (int k = 0; k < 9; ++k) Dg[i * 9 + k] = Dn[k];
#pragma unroll
      for (int r = 0; r < 3; ++r) R[i * 3 + r] = Rn[r];
    }
    __syncthreads();
  }
  if (tid == 0) {  // equation 0 alone: x_0 = a_0^-1 r_0
    inv3_inplace(Dg);
    double x[3] = {0., 0., 0.};
    add_mul31(Dg, R, x);
#pragma unroll
    for (int r = 0; r < 3; ++r) R[r] = x[r];
  }
  __syncthreads();
  for (s >>= 1; s >= 1; s >>= 1) {
    const int s2 = 2 * s;
    for (int j = s + tid * s2; j < nl; j += nt * s2) {
      double t[3], x[3] = {0., 0., 0.}, mb[9];
#pragma unroll
      for (int r = 0; r < 3; ++r) t[r] = R[j * 3 + r];
#pragma unroll
      for (int k = 0; k < 9; ++k) mb[k] = -Bl[j * 9 + k];
      add_mul31(mb, R + (j - s) * 3, t);
      if (j + s < nl) {
#pragma unroll
        for (int k = 0; k < 9; ++k) mb[k] = -Ab[j * 9 + k];
        add_mul31(mb, R + (j + s) * 3, t);
      }
      add_mul31(Dg + j * 9, t, x);
#pragma unroll
      for (int r = 0; r < 3; ++r) R[j * 3 + r] = x[r];
    }
    __syncthreads();
  }
}

}  // namespace snapb
