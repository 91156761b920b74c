// dual.cuh — forward-mode dual numbers for the local Jacobian-vector products
// inside the adjoint kernels.
//
// Dual x = (v, d): value and one directional derivative.  The templated point
// kernels of common.cuh / vic.cu (reconstruction, Riemann fluxes, flux
// Jacobians, Roe eigen-decompositions) are evaluated with T = Dual to get an
// exact derivative of their outputs along one input direction; the adjoint
// kernels contract those with the incoming cotangents.  Comparisons and
// branch selections use the value only, i.e. every switch (WENO weights are
// smooth; HLLC / Roe wave-speed selections, LMARS upwinding, the pressure
// clamp) is differentiated on its active branch.
#pragma once

#include <cuda_runtime.h>

namespace snapb {

// the double overloads stay visible next to the Dual ones below
using ::fabs;
using ::fmax;
using ::fmin;
using ::pow;
using ::sqrt;

struct Dual {
  double v, d;
  __host__ __device__ Dual() : v(0.), d(0.) {}
  __host__ __device__ Dual(double x) : v(x), d(0.) {}  // NOLINT: constants promote
  __host__ __device__ Dual(double x, double dx) : v(x), d(dx) {}
  __host__ __device__ Dual& operator+=(const Dual& o) {
    v += o.v;
    d += o.d;
    return *this;
  }
  __host__ __device__ Dual& operator-=(const Dual& o) {
    v -= o.v;
    d -= o.d;
    return *this;
  }
  __host__ __device__ Dual& operator*=(const Dual& o) {
    d = d * o.v + v * o.d;
    v *= o.v;
    return *this;
  }
  __host__ __device__ Dual& operator/=(const Dual& o) {
    double iv = 1. / o.v;
    d = (d - v * iv * o.d) * iv;
    v *= iv;
    return *this;
  }
};

__host__ __device__ __forceinline__ Dual operator+(Dual a, const Dual& b) { return a += b; }
__host__ __device__ __forceinline__ Dual operator-(Dual a, const Dual& b) { return a -= b; }
__host__ __device__ __forceinline__ Dual operator*(Dual a, const Dual& b) { return a *= b; }
__host__ __device__ __forceinline__ Dual operator/(Dual a, const Dual& b) { return a /= b; }
__host__ __device__ __forceinline__ Dual operator-(const Dual& a) { return Dual(-a.v, -a.d); }
__host__ __device__ __forceinline__ bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
__host__ __device__ __forceinline__ bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
__host__ __device__ __forceinline__ bool operator<=(const Dual& a, const Dual& b) {
  return a.v <= b.v;
}
__host__ __device__ __forceinline__ bool operator>=(const Dual& a, const Dual& b) {
  return a.v >= b.v;
}
__host__ __device__ __forceinline__ bool operator==(const Dual& a, const Dual& b) {
  return a.v == b.v;
}
__host__ __device__ __forceinline__ bool operator!=(const Dual& a, const Dual& b) {
  return a.v != b.v;
}
__device__ __forceinline__ Dual sqrt(const Dual& a) {
  double s = ::sqrt(a.v);
  return Dual(s, a.d * 0.5 / s);
}
__device__ __forceinline__ Dual fabs(const Dual& a) { return a.v < 0. ? -a : a; }
__device__ __forceinline__ Dual fmax(const Dual& a, const Dual& b) { return a.v >= b.v ? a : b; }
__device__ __forceinline__ Dual fmin(const Dual& a, const Dual& b) { return a.v <= b.v ? a : b; }
// x^e for a constant exponent (x > 0 wherever it is used: pressures, densities)
__device__ __forceinline__ Dual pow(const Dual& x, double e) {
  double y = ::pow(x.v, e);
  return Dual(y, e * y / x.v * x.d);
}

}  // namespace snapb
