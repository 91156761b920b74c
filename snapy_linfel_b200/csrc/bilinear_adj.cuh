// bilinear_adj.cuh — reverse-mode gradients, written by hand, of the two
// bilinear forms the implicit solve's adjoint contracts: y^T |A|(wl, wr) x
// with respect to both primitive states of an interface, and y^T J(w) x with
// respect to a cell's primitive state (the blocks of vic_blocks.cuh:
// absA_block, jac_block; reference src/implicit/flux_decomposition_impl.h:
// 133-245).  One forward evaluation keeps the intermediates and one reverse
// sweep carries the cotangents back, in place of one dual-number evaluation
// of the whole block per input component.  The derivative of |s| is taken
// as +1 at s = 0, as the dual numbers take it.
#pragma once

#include <cmath>

namespace snapb {

// rows / columns of the N-block form (as sel<N> of vic_blocks.cuh)
template <int N>
__host__ __device__ __forceinline__ int sel_rc(int r) {
  if constexpr (N == 3) return r == 2 ? 4 : r;
  return r;
}

// gl += d/dwl, gr += d/dwr of y^T |A|(wl, wr) x (either may be null)
template <int N>
__host__ __device__ __forceinline__ void absA_bilinear_vjp(double gm1, const double* wl,
                                                           const double* wr, const double* y,
                                                           const double* x, double* gl,
                                                           double* gr) {
  // ---- forward, as absA_block ----
  const double rl = wl[0], ul = wl[1], vl = wl[2], zl = wl[3], pl = wl[4];
  const double rr = wr[0], ur = wr[1], vr = wr[2], zr = wr[3], pr = wr[4];
  const double sdl = sqrt(rl), sdr = sqrt(rr);
  const double isd = 1.0 / (sdl + sdr);
  const double r = sdl * sdr;
  const double nu = sdl * ul + sdr * ur, nv = sdl * vl + sdr * vr, nw = sdl * zl + sdr * zr;
  const double u = nu * isd, v = nv * isd, w = nw * isd;
  const double kl = ul * ul + vl * vl + zl * zl, kr = ur * ur + vr * vr + zr * zr;
  const double el = pl / gm1 + 0.5 * rl * kl, er = pr / gm1 + 0.5 * rr * kr;
  const double ql = (el + pl) / sdl, qr = (er + pr) / sdr;
  const double hbar = (ql + qr) * isd;
  const double q2 = u * u + v * v + w * w;
  const double g1 = gm1 + 1.0, c = gm1 / g1;
  const double pb = (hbar - 0.5 * q2) * c;  // p / r
  const double P = pb * r;
  const double cs = sqrt(P * g1 / r);
  const double ke = 0.5 * q2;
  const double hp = g1 / gm1 * P / r;
  const double h = hp + ke;
  const double i2chp = 1.0 / (2.0 * cs * hp), ihp = 1.0 / hp, i2hp = 0.5 * ihp;
  const double lam[5] = {fabs(u - cs), fabs(u), fabs(u + cs), fabs(u), fabs(u)};
  const double R[5][5] = {{1., 1., 1., 0., 0.},
                          {u - cs, u, u + cs, 0., 0.},
                          {v, v, v, 1., 0.},
                          {w, w, w, 0., 1.},
                          {h - u * cs, ke, h + u * cs, v, w}};
  const double Ri[5][5] = {
      {(cs * ke + u * hp) * i2chp, (-hp - cs * u) * i2chp, -v * i2hp, -w * i2hp, i2hp},
      {(hp - ke) * ihp, u * ihp, v * ihp, w * ihp, -ihp},
      {(cs * ke - u * hp) * i2chp, (hp - cs * u) * i2chp, -v * i2hp, -w * i2hp, i2hp},
      {-v, 0., 1., 0., 0.},
      {-w, 0., 0., 1., 0.}};
  // F = sum_k Y_k lam_k X_k, Y_k = sum_a y_a R[ra][k], X_k = sum_b Ri[k][cb] x_b
  double Y[5], X[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    double sy = 0., sx = 0.;
#pragma unroll
    for (int a = 0; a < N; ++a) {
      sy += y[a] * R[sel_rc<N>(a)][k];
      sx += Ri[k][sel_rc<N>(a)] * x[a];
    }
    Y[k] = sy;
    X[k] = sx;
  }
  // ---- reverse ----
  double bR[5][5] = {}, bRi[5][5] = {}, blam[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    blam[k] = Y[k] * X[k];
#pragma unroll
    for (int a = 0; a < N; ++a) {
      bR[sel_rc<N>(a)][k] = y[a] * lam[k] * X[k];
      bRi[k][sel_rc<N>(a)] = Y[k] * lam[k] * x[a];
    }
  }
  double bu = 0., bv = 0., bw = 0., bcs = 0., bh = 0., bke = 0., bhp = 0.;
  double bi2chp = 0., bihp = 0., bi2hp = 0.;
  // R
  bu += bR[1][0] + bR[1][1] + bR[1][2];
  bcs += bR[1][2] - bR[1][0];
  bv += bR[2][0] + bR[2][1] + bR[2][2] + bR[4][3];
  bw += bR[3][0] + bR[3][1] + bR[3][2] + bR[4][4];
  bh += bR[4][0] + bR[4][2];
  bu += (bR[4][2] - bR[4][0]) * cs;
  bcs += (bR[4][2] - bR[4][0]) * u;
  bke += bR[4][1];
  // Ri, rows 0 and 2 (i2chp rows), columns 2..4 of rows 0 and 2 (i2hp)
  {
    const double b0 = bRi[0][0], b1 = bRi[0][1], d0 = bRi[2][0], d1 = bRi[2][1];
    bcs += (b0 + d0) * ke * i2chp - (b1 + d1) * u * i2chp;
    bke += (b0 + d0) * cs * i2chp;
    bu += (b0 - d0) * hp * i2chp - (b1 + d1) * cs * i2chp;
    bhp += (b0 - d0) * u * i2chp + (d1 - b1) * i2chp;
    bi2chp += b0 * (cs * ke + u * hp) + b1 * (-hp - cs * u) + d0 * (cs * ke - u * hp) +
              d1 * (hp - cs * u);
    const double s2 = bRi[0][2] + bRi[2][2], s3 = bRi[0][3] + bRi[2][3];
    bv -= s2 * i2hp;
    bw -= s3 * i2hp;
    bi2hp += -s2 * v - s3 * w + bRi[0][4] + bRi[2][4];
  }
  // Ri row 1 (ihp)
  bhp += bRi[1][0] * ihp;
  bke -= bRi[1][0] * ihp;
  bu += bRi[1][1] * ihp;
  bv += bRi[1][2] * ihp;
  bw += bRi[1][3] * ihp;
  bihp += bRi[1][0] * (hp - ke) + bRi[1][1] * u + bRi[1][2] * v + bRi[1][3] * w - bRi[1][4];
  // Ri rows 3, 4
  bv -= bRi[3][0];
  bw -= bRi[4][0];
  // lam
  {
    const double s0 = (u - cs) < 0. ? -1. : 1., su = u < 0. ? -1. : 1.,
                 s2 = (u + cs) < 0. ? -1. : 1.;
    bu += blam[0] * s0 + (blam[1] + blam[3] + blam[4]) * su + blam[2] * s2;
    bcs += blam[2] * s2 - blam[0] * s0;
  }
  // i2hp = ihp / 2, ihp = 1 / hp, i2chp = 1 / (2 cs hp)
  bihp += 0.5 * bi2hp;
  bhp -= bihp * ihp * ihp;
  bcs -= bi2chp * i2chp / cs;
  bhp -= bi2chp * i2chp / hp;
  // h = hp + ke
  bhp += bh;
  bke += bh;
  // hp = g1 / gm1 P / r,  cs = sqrt(P g1 / r)
  double bP = bhp * g1 / gm1 / r + bcs * g1 / (2.0 * cs * r);
  double br = -bhp * hp / r - bcs * cs / (2.0 * r);
  // ke = q2 / 2, P = (hbar - q2 / 2) c r
  double bq2 = 0.5 * bke - 0.5 * bP * c * r;
  const double bhbar = bP * c * r;
  br += bP * pb;
  bu += 2.0 * u * bq2;
  bv += 2.0 * v * bq2;
  bw += 2.0 * w * bq2;
  // hbar = (ql + qr) isd; u, v, w = n isd
  const double bql = bhbar * isd, bqr = bhbar * isd;
  double bisd = bhbar * (ql + qr) + bu * nu + bv * nv + bw * nw;
  const double bnu = bu * isd, bnv = bv * isd, bnw = bw * isd;
  // ql = (el + pl) / sdl, el = pl / gm1 + rl kl / 2
  const double bel = bql / sdl, ber = bqr / sdr;
  double bsdl = -bql * ql / sdl, bsdr = -bqr * qr / sdr;
  // isd = 1 / (sdl + sdr), r = sdl sdr
  const double bS = -bisd * isd * isd;
  bsdl += bS + br * sdr + bnu * ul + bnv * vl + bnw * zl;
  bsdr += bS + br * sdl + bnu * ur + bnv * vr + bnw * zr;
  if (gl) {
    gl[0] += bel * 0.5 * kl + bsdl / (2.0 * sdl);
    gl[1] += bel * rl * ul + bnu * sdl;
    gl[2] += bel * rl * vl + bnv * sdl;
    gl[3] += bel * rl * zl + bnw * sdl;
    gl[4] += bel / gm1 + bql / sdl;
  }
  if (gr) {
    gr[0] += ber * 0.5 * kr + bsdr / (2.0 * sdr);
    gr[1] += ber * rr * ur + bnu * sdr;
    gr[2] += ber * rr * vr + bnv * sdr;
    gr[3] += ber * rr * zr + bnw * sdr;
    gr[4] += ber / gm1 + bqr / sdr;
  }
}

// gw += d/dw of y^T J(w) x
template <int N>
__host__ __device__ __forceinline__ void jac_bilinear_vjp(double gm1, const double* w,
                                                          const double* y, const double* x,
                                                          double* gw) {
  const double rho = w[0], v1 = w[1], v2 = w[2], v3 = w[3], pres = w[4];
  const double s2 = v1 * v1 + v2 * v2 + v3 * v3;
  const double g1 = gm1 + 1.0;
  const double hp = g1 / gm1 * pres / rho;
  double B[5][5] = {};  // d F / d J_full = y_a x_b on the kept rows and columns
#pragma unroll
  for (int a = 0; a < N; ++a)
#pragma unroll
    for (int b = 0; b < N; ++b) B[sel_rc<N>(a)][sel_rc<N>(b)] = y[a] * x[b];
  double b1 = 0., b2 = 0., b3 = 0., bs2 = 0., bhp = 0.;
  // row 1: gm1 s2/2 - v1^2, (2 - gm1) v1, -gm1 v2, -gm1 v3, gm1
  bs2 += B[1][0] * 0.5 * gm1;
  b1 += -2.0 * v1 * B[1][0] + (2.0 - gm1) * B[1][1];
  b2 -= gm1 * B[1][2];
  b3 -= gm1 * B[1][3];
  // rows 2, 3: -v1 v2, v2, v1; -v1 v3, v3, v1
  b1 += -v2 * B[2][0] + B[2][2] - v3 * B[3][0] + B[3][3];
  b2 += -v1 * B[2][0] + B[2][1];
  b3 += -v1 * B[3][0] + B[3][1];
  // row 4: c1 = ((gm1 - 1) s2/2 - hp) v1, c2 = hp + s2/2 - gm1 v1^2,
  //        -gm1 v2 v1, -gm1 v3 v1, (gm1 + 1) v1
  bs2 += B[4][0] * 0.5 * (gm1 - 1.0) * v1 + 0.5 * B[4][1];
  bhp += -B[4][0] * v1 + B[4][1];
  b1 += B[4][0] * ((gm1 - 1.0) * s2 * 0.5 - hp) - 2.0 * gm1 * v1 * B[4][1] -
        gm1 * v2 * B[4][2] - gm1 * v3 * B[4][3] + g1 * B[4][4];
  b2 -= gm1 * v1 * B[4][2];
  b3 -= gm1 * v1 * B[4][3];
  // s2, hp = g1 / gm1 pres / rho
  b1 += 2.0 * v1 * bs2;
  b2 += 2.0 * v2 * bs2;
  b3 += 2.0 * v3 * bs2;
  gw[0] -= bhp * hp / rho;
  gw[1] += b1;
  gw[2] += b2;
  gw[3] += b3;
  gw[4] += bhp * g1 / gm1 / rho;
}

}  // namespace snapb
