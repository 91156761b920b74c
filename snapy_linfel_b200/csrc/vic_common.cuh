// vic_common.cuh — state access shared by the implicit-solve kernels
// (vic.cu, vicf.cu, vic_cr.cu): the column offsets, the full primitives of the
// FP64 plain form and of the FP32 perturbation form, du access and the RK
// combination in the stored precision.
#pragma once

#include "kernels.cuh"

namespace snapb {

template <int N>
struct VicDims {
  static constexpr int ES = N * N + N;
};

inline int vic_n(const Phys& p) { return ((p.implicit_scheme >> 3) & 1) ? 5 : 3; }

// (k, j, il) offset of interior column `col`
__device__ __forceinline__ int64_t column_base(const Geo& g, int64_t col) {
  const int nj = g.ju - g.jl + 1;
  const int j = g.jl + umod(col, nj), k = g.kl + udiv(col, nj);
  return (int64_t)k * g.s3 + (int64_t)j * g.s2 + g.il;
}

// ---- state access, FP64 plain form and FP32 perturbation form ----
// full primitive of variable v at offset off, x1 index xi
__device__ __forceinline__ double vic_w(const StageBufs& b, int64_t sv, int v, int64_t off,
                                        int xi) {
  return b.w[v * sv + off];
}
__device__ __forceinline__ double vic_w(const StageBufs32& b, int64_t sv, int v, int64_t off,
                                        int xi) {
  double x = (double)b.w[v * sv + off];
  if (v == IDN) x += b.rb[xi];
  if (v == IPR) x += b.pb[xi];
  return x;
}
// full primitive of variable v at x1 index xi from a stored value x
__device__ __forceinline__ double vic_full(const StageBufs&, double x, int v, int xi) { return x; }
__device__ __forceinline__ double vic_full(const StageBufs32& b, double x, int v, int xi) {
  if (v == IDN) x += b.rb[xi];
  if (v == IPR) x += b.pb[xi];
  return x;
}
// the same in the precision the blocks are formed in: the FP64 plain form's
// value as is; for the FP32 perturbation form the stored velocities as they
// are, density and pressure summed with the reference in FP64 and rounded
__device__ __forceinline__ double vic_full_blk(const StageBufs&, double x, int v, int xi) {
  return x;
}
__device__ __forceinline__ float vic_full_blk(const StageBufs32& b, float x, int v, int xi) {
  if (v == IDN) return (float)((double)x + b.rb[xi]);
  if (v == IPR) return (float)((double)x + b.pb[xi]);
  return x;
}
__device__ __forceinline__ double vic_d(const StageBufs& b, int64_t idx) { return b.D[idx]; }
__device__ __forceinline__ double vic_d(const StageBufs32& b, int64_t idx) {
  return (double)b.D[idx];
}
__device__ __forceinline__ void vic_set_d(const StageBufs& b, int64_t idx, double x) {
  b.D[idx] = x;
}
__device__ __forceinline__ void vic_set_d(const StageBufs32& b, int64_t idx, double x) {
  b.D[idx] = (float)x;
}
// RK combination of one stored value (u' for the FP32 form: the reference
// part of u is constant in time, so the combination is the same), from
// values already loaded (qo = q[o], q0o = q0[o] when stage > 0); the stored
// q keeps the stored precision
__device__ __forceinline__ double vic_rk_from(double* q, double* q0, int64_t o, bool first,
                                              double qo, double q0o, double w0, double w1,
                                              double w2, double d) {
  double q0v = first ? qo : q0o;
  if (first) q0[o] = qo;
  double qn = w0 * q0v + w1 * qo + w2 * d;
  q[o] = qn;
  return qn;
}
__device__ __forceinline__ double vic_rk_from(float* q, float* q0, int64_t o, bool first,
                                              double qo, double q0o, double w0, double w1,
                                              double w2, double d) {
  double q0v = first ? qo : q0o;
  if (first) q0[o] = (float)qo;
  float qn = (float)(w0 * q0v + w1 * qo + w2 * d);
  q[o] = qn;
  return qn;
}
// full density of a stored conserved perturbation
__device__ __forceinline__ double vic_full_rho(const StageBufs&, double u_rho, int) {
  return u_rho;
}
__device__ __forceinline__ double vic_full_rho(const StageBufs32& b, double u_rho, int xi) {
  return u_rho + b.rb[xi];
}

}  // namespace snapb
