// oracle_diffusion.hpp — isotropic viscosity + heat conduction forcing of the
// oracle (TEST INFRASTRUCTURE ONLY), restating DiffusionImpl::forward
// (src/forcing/diffusion.cpp:152-240) on uniform Cartesian grids.
#pragma once

namespace orc {

inline void Block::diffusion(double dt, const double* w, double* du) {
  const auto& c = g.c;
  int64_t sv = g.sv;
  int nv = c.nvar;
  bool act[3] = {g.nc1 > 1, g.nc2 > 1, g.nc3 > 1};
  int64_t st[3] = {g.s1, g.s2, g.s3};
  double dx[3] = {g.dx1, g.dx2, g.dx3};
  // interior cell box (lo inclusive, hi exclusive) per axis (x1, x2, x3)
  int lo[3] = {g.il, g.jl, g.kl}, hi[3] = {g.iu + 1, g.ju + 1, g.ku + 1};
  int64_t n = g.cells();

  auto at = [&](int i, int j, int k) { return g.idx(k, j, i); };

  // divergence of velocity on the interior extended by one cell along every
  // active axis: ((0 + d1) + d2) + d3 with centred differences
  std::vector<double> div_vel;
  if (c.nu_iso > 0.) {
    div_vel.assign(n, 0.);
    int elo[3], ehi[3];
    for (int a = 0; a < 3; ++a) {
      elo[a] = lo[a] - (act[a] ? 1 : 0);
      ehi[a] = hi[a] + (act[a] ? 1 : 0);
    }
    for (int a = 0; a < 3; ++a) {
      if (!act[a]) continue;
      const double* v = w + (IVX + a) * sv;
      for (int k = elo[2]; k < ehi[2]; ++k)
        for (int j = elo[1]; j < ehi[1]; ++j)
          for (int i = elo[0]; i < ehi[0]; ++i) {
            int64_t t = at(i, j, k);
            div_vel[t] += (v[t + st[a]] - v[t - st[a]]) / (2. * dx[a]);
          }
    }
  }
  std::vector<double> rho_cv, temp(n);
  double cv = c.rgas / (c.gammad - 1.);
  for (int64_t t = 0; t < n; ++t) temp[t] = w[IPR * sv + t] / (w[IDN * sv + t] * c.rgas);
  if (c.kappa_iso > 0.) {
    rho_cv.assign(n, 0.);
    for (int64_t t = 0; t < n; ++t) rho_cv[t] = w[IDN * sv + t] * cv;
  }

  std::vector<double> flux[3];
  for (int a = 0; a < 3; ++a) {
    if (!act[a]) continue;
    flux[a].assign((int64_t)nv * sv, 0.);
    double* F = flux[a].data();
    int fhi[3] = {hi[0], hi[1], hi[2]};
    fhi[a] += 1;  // faces lo..hi (inclusive) along the flux axis
    int64_t s = st[a];
    for (int k = lo[2]; k < fhi[2]; ++k)
      for (int j = lo[1]; j < fhi[1]; ++j)
        for (int i = lo[0]; i < fhi[0]; ++i) {
          int64_t t = at(i, j, k);
          double rho_face = 0.5 * (w[IDN * sv + t] + w[IDN * sv + t - s]);
          if (c.nu_iso > 0.) {
            double div_face = 0.5 * (div_vel[t] + div_vel[t - s]);
            for (int b = 0; b < 3; ++b) {
              const double* vb = w + (IVX + b) * sv;
              double stress = (vb[t] - vb[t - s]) / dx[a];
              if (b == a) {
                stress = 2. * stress - (2. / 3.) * div_face;
              } else if (act[b]) {
                const double* va = w + (IVX + a) * sv;
                double d0 = (va[t + st[b]] - va[t - st[b]]) / (2. * dx[b]);
                double d1 = (va[t - s + st[b]] - va[t - s - st[b]]) / (2. * dx[b]);
                stress += 0.5 * (d0 + d1);
              }
              double mflux = -c.nu_iso * rho_face * stress;
              F[(IVX + b) * sv + t] = mflux;
              F[IPR * sv + t] += 0.5 * (vb[t] + vb[t - s]) * mflux;
            }
          }
          if (c.kappa_iso > 0.) {
            F[IPR * sv + t] -= c.kappa_iso * (0.5 * (rho_cv[t] + rho_cv[t - s])) *
                               ((temp[t] - temp[t - s]) / dx[a]);
          }
        }
  }
  // du -= dt * div(F) on the interior
  double A[3] = {g.area1(), g.area2(), g.area3()};
  double V = g.vol();
  for (int k = g.kl; k <= g.ku; ++k)
    for (int j = g.jl; j <= g.ju; ++j)
      for (int i = g.il; i <= g.iu; ++i) {
        int64_t t = at(i, j, k);
        for (int v = 0; v < nv; ++v) {
          int64_t q = v * sv + t;
          double d = 0.;
          for (int a = 0; a < 3; ++a)
            if (act[a]) d += A[a] * flux[a][q + st[a]] - A[a] * flux[a][q];
          du[q] -= dt * (d / V);
        }
      }
}

}  // namespace orc
