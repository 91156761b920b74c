// Host check of csrc/bilinear_adj.cuh: the hand-written reverse-mode
// gradients of y^T |A|(wl, wr) x and y^T J(w) x against central differences
// of the block formulas, evaluated in long double (the formulas restated here
// from the flux decomposition: Roe average, R |Lambda| R^-1, and the x1 flux
// Jacobian; reference src/implicit/flux_decomposition_impl.h:133-245).
// Prints "worst <N=3> <N=5>": the largest relative error over seeded random
// states (perturbation-scale velocities and pressures near 1e5 Pa), skipping
// samples whose difference stencil straddles a kink of |u|, |u - cs|, |u + cs|.
#define __host__
#define __device__
#define __forceinline__ inline
#include <cmath>
#include <cstdio>
#include <random>

#include "../../snapy_linfel_b200/csrc/bilinear_adj.cuh"

using namespace snapb;
typedef long double LD;

template <int N>
static int sel(int r) {
  return N == 3 ? (r == 2 ? 4 : r) : r;
}

// y^T |A|(wl, wr) x in long double; kink: the smallest |u|, |u -+ cs|
template <int N>
static LD absA_form(LD gm1, const LD* wl, const LD* wr, const double* y, const double* x,
                    LD* kink) {
  LD sdl = sqrtl(wl[0]), sdr = sqrtl(wr[0]);
  LD isd = 1.0L / (sdl + sdr), r = sdl * sdr;
  LD u = (sdl * wl[1] + sdr * wr[1]) * isd, v = (sdl * wl[2] + sdr * wr[2]) * isd,
     w = (sdl * wl[3] + sdr * wr[3]) * isd;
  LD el = wl[4] / gm1 + 0.5L * wl[0] * (wl[1] * wl[1] + wl[2] * wl[2] + wl[3] * wl[3]);
  LD er = wr[4] / gm1 + 0.5L * wr[0] * (wr[1] * wr[1] + wr[2] * wr[2] + wr[3] * wr[3]);
  LD hbar = ((el + wl[4]) / sdl + (er + wr[4]) / sdr) * isd;
  LD p = ((hbar - 0.5L * (u * u + v * v + w * w)) * gm1 / (gm1 + 1.0L)) * r;
  LD cs = sqrtl(p * (gm1 + 1.0L) / r);
  if (kink) *kink = fminl(fabsl(u), fminl(fabsl(u - cs), fabsl(u + cs)));
  LD lam[5] = {fabsl(u - cs), fabsl(u), fabsl(u + cs), fabsl(u), fabsl(u)};
  LD ke = 0.5L * (u * u + v * v + w * w);
  LD hp = (gm1 + 1.0L) / gm1 * p / r, h = hp + ke;
  LD i2chp = 1.0L / (2.0L * cs * hp), ihp = 1.0L / hp, i2hp = 0.5L * ihp;
  LD R[5][5] = {{1, 1, 1, 0, 0},
                {u - cs, u, u + cs, 0, 0},
                {v, v, v, 1, 0},
                {w, w, w, 0, 1},
                {h - u * cs, ke, h + u * cs, v, w}};
  LD Ri[5][5] = {{(cs * ke + u * hp) * i2chp, (-hp - cs * u) * i2chp, -v * i2hp, -w * i2hp, i2hp},
                 {(hp - ke) * ihp, u * ihp, v * ihp, w * ihp, -ihp},
                 {(cs * ke - u * hp) * i2chp, (hp - cs * u) * i2chp, -v * i2hp, -w * i2hp, i2hp},
                 {-v, 0, 1, 0, 0},
                 {-w, 0, 0, 1, 0}};
  LD F = 0;
  for (int a = 0; a < N; ++a)
    for (int b = 0; b < N; ++b) {
      LD s = 0;
      for (int k = 0; k < 5; ++k) s += R[sel<N>(a)][k] * lam[k] * Ri[k][sel<N>(b)];
      F += y[a] * s * x[b];
    }
  return F;
}

// y^T J(w) x in long double
template <int N>
static LD jac_form(LD gm1, const LD* q, const double* y, const double* x) {
  LD rho = q[0], v1 = q[1], v2 = q[2], v3 = q[3], pres = q[4];
  LD s2 = v1 * v1 + v2 * v2 + v3 * v3, hp = (gm1 + 1) / gm1 * pres / rho;
  LD c1 = ((gm1 - 1) * s2 / 2 - hp) * v1, c2 = hp + s2 / 2 - gm1 * v1 * v1;
  LD J[5][5] = {{0, 1, 0, 0, 0},
                {gm1 * s2 / 2 - v1 * v1, (2 - gm1) * v1, -gm1 * v2, -gm1 * v3, gm1},
                {-v1 * v2, v2, v1, 0, 0},
                {-v1 * v3, v3, 0, v1, 0},
                {c1, c2, -gm1 * v2 * v1, -gm1 * v3 * v1, (gm1 + 1) * v1}};
  LD F = 0;
  for (int a = 0; a < N; ++a)
    for (int b = 0; b < N; ++b) F += y[a] * J[sel<N>(a)][sel<N>(b)] * x[b];
  return F;
}

template <int N>
static double worst_of(std::mt19937_64& g, int samples) {
  std::uniform_real_distribution<double> U(-1, 1);
  const double gm1 = 0.4;
  double worst = 0;
  for (int t = 0; t < samples; ++t) {
    double wl[5] = {1 + 0.3 * U(g), 30 * U(g), 20 * U(g), 20 * U(g), 1e5 * (1 + 0.2 * U(g))};
    double wr[5] = {1 + 0.3 * U(g), 30 * U(g), 20 * U(g), 20 * U(g), 1e5 * (1 + 0.2 * U(g))};
    double y[5], x[5];
    for (int k = 0; k < 5; ++k) {
      y[k] = U(g);
      x[k] = U(g);
    }
    double gl[5] = {}, gr[5] = {}, gj[5] = {};
    absA_bilinear_vjp<N>(gm1, wl, wr, y, x, gl, gr);
    jac_bilinear_vjp<N>(gm1, wl, y, x, gj);
    for (int side = 0; side < 3; ++side)
      for (int c = 0; c < 5; ++c) {
        LD L[5], R[5];
        for (int q = 0; q < 5; ++q) {
          L[q] = wl[q];
          R[q] = wr[q];
        }
        LD* W = side == 1 ? R : L;
        const LD h = (c >= 1 && c <= 3) ? 1e-4L : 1e-6L * fabsl(W[c]);
        const LD w0 = W[c];
        LD kink = 1e30L, kp = 1e30L, km = 1e30L;
        if (side < 2) absA_form<N>(gm1, L, R, y, x, &kink);
        W[c] = w0 + h;
        LD fp = side < 2 ? absA_form<N>(gm1, L, R, y, x, &kp) : jac_form<N>(gm1, L, y, x);
        W[c] = w0 - h;
        LD fm = side < 2 ? absA_form<N>(gm1, L, R, y, x, &km) : jac_form<N>(gm1, L, y, x);
        if (side < 2 && fminl(kink, fminl(kp, km)) < 1e-3L) continue;  // stencil on a kink
        const double fd = (double)((fp - fm) / (2 * h));
        const double an = side == 0 ? gl[c] : (side == 1 ? gr[c] : gj[c]);
        const double scale = fabs(fd) + fabs(an);
        if (scale == 0.) continue;
        const double e = fabs(fd - an) / scale;
        if (e > worst) worst = e;
      }
  }
  return worst;
}

int main() {
  std::mt19937_64 g(2027);
  const double w3 = worst_of<3>(g, 2000), w5 = worst_of<5>(g, 2000);
  std::printf("worst %.3e %.3e\n", w3, w5);
  return 0;
}
