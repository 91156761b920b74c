// riemann_adj.cuh — hand-written reverse (vector-Jacobian products) of the
// Riemann fluxes of common.cuh: given the cotangent gF of the five fluxes at a
// face, accumulate gL += (dF/dL)^T gF and gR += (dF/dR)^T gF.
//
// Each function replays its forward (hllc_flux / lmars_flux / roe_flux, same
// operation order and the same branch choices) and then walks the statements
// backwards; every switch is differentiated on the branch the forward takes.
// They cost a few forward evaluations, against ten dual-number passes for the
// generic forward-mode product.  Forward formulas: src/riemann/hllc_impl.h:16-130,
// src/riemann/lmars_impl.h:16-78, src/riemann/roe_impl.h:23-211.
#pragma once

#include "common.cuh"

namespace snapb {

// ---------------------------------------------------------------------------
// LMARS
// ---------------------------------------------------------------------------
__device__ __forceinline__ void lmars_vjp(const double* L, const double* R, int ivx,
                                          double gamma, const double* gF, double* gL,
                                          double* gR) {
  const int ivy = IVX + (ivx - IVX + 1) % 3;
  const int ivz = IVX + (ivx - IVX + 2) % 3;
  const double igm1 = 1. / (gamma - 1.);
  const double irl = 1. / L[IDN], irr = 1. / R[IDN];
  const double ke_l = 0.5 * (sqr(L[ivx]) + sqr(L[ivy]) + sqr(L[ivz]));
  const double ke_r = 0.5 * (sqr(R[ivx]) + sqr(R[ivy]) + sqr(R[ivz]));
  const double hl = L[IPR] * igm1 * irl + ke_l + L[IPR] * irl;
  const double hr = R[IPR] * igm1 * irr + ke_r + R[IPR] * irr;
  const double rhobar = 0.5 * (L[IDN] + R[IDN]);
  const double cbar = sqrt(0.5 * gamma * (L[IPR] + R[IPR]) / rhobar);
  const double Q = rhobar * cbar;
  const double ubar = 0.5 * (L[ivx] + R[ivx]) + 0.5 / Q * (L[IPR] - R[IPR]);
  const bool left = ubar > 0.;
  const double* S = left ? L : R;
  double* gS = left ? gL : gR;
  const double h = left ? hl : hr;
  const double m = ubar * S[IDN];
  // F = (m, m uS + pbar, m vS, m wS, m h)
  const double gm = gF[IDN] + gF[ivx] * S[ivx] + gF[ivy] * S[ivy] + gF[ivz] * S[ivz] +
                    gF[IPR] * h;
  const double gpbar = gF[ivx];
  gS[ivx] += gF[ivx] * m;
  gS[ivy] += gF[ivy] * m;
  gS[ivz] += gF[ivz] * m;
  const double gh = gF[IPR] * m;
  // h of the upwind side: p/rho (igm1 + 1) + ke
  {
    const double ir = 1. / S[IDN];
    gS[IPR] += gh * (igm1 + 1.) * ir;
    gS[IDN] -= gh * S[IPR] * (igm1 + 1.) * ir * ir;
    gS[ivx] += gh * S[ivx];
    gS[ivy] += gh * S[ivy];
    gS[ivz] += gh * S[ivz];
  }
  // m = ubar rho_S
  const double gubar = gm * S[IDN];
  gS[IDN] += gm * ubar;
  // pbar = (pL + pR)/2 + Q (uL - uR)/2,  ubar = (uL + uR)/2 + (pL - pR)/(2Q)
  gL[ivx] += 0.5 * gubar + 0.5 * Q * gpbar;
  gR[ivx] += 0.5 * gubar - 0.5 * Q * gpbar;
  gL[IPR] += 0.5 * gpbar + 0.5 * gubar / Q;
  gR[IPR] += 0.5 * gpbar - 0.5 * gubar / Q;
  const double gQ = gpbar * 0.5 * (L[ivx] - R[ivx]) - gubar * 0.5 * (L[IPR] - R[IPR]) / (Q * Q);
  // Q = sqrt(gamma (pL + pR) rhobar / 2)
  const double dQdp = 0.25 * gamma * rhobar / Q;
  const double dQdr = 0.25 * gamma * (L[IPR] + R[IPR]) / Q;
  gL[IPR] += gQ * dQdp;
  gR[IPR] += gQ * dQdp;
  gL[IDN] += 0.5 * gQ * dQdr;
  gR[IDN] += 0.5 * gQ * dQdr;
}

// ---------------------------------------------------------------------------
// HLLC
// ---------------------------------------------------------------------------
__device__ __forceinline__ void hllc_vjp(const double* L, const double* R, int ivx, double gamma,
                                         const double* gF, double* gL, double* gR) {
  const double TINY = 1.0e-10;
  const int ivy = IVX + (ivx - IVX + 1) % 3;
  const int ivz = IVX + (ivx - IVX + 2) % 3;
  const double igm1 = 1. / (gamma - 1.);
  const double cl = sqrt(gamma * L[IPR] / L[IDN]);
  const double cr = sqrt(gamma * R[IPR] / R[IDN]);
  const double el = L[IPR] * igm1 + 0.5 * L[IDN] * (sqr(L[IVX]) + sqr(L[IVY]) + sqr(L[IVZ]));
  const double er = R[IPR] * igm1 + 0.5 * R[IDN] * (sqr(R[IVX]) + sqr(R[IVY]) + sqr(R[IVZ]));
  const double rhoa = 0.5 * (L[IDN] + R[IDN]);
  const double ca = 0.5 * (cl + cr);
  const double pmid = 0.5 * (L[IPR] + R[IPR] + (L[ivx] - R[ivx]) * rhoa * ca);
  const double gf = (gamma + 1.) / (2. * gamma);
  const bool shl = !(pmid <= L[IPR]), shr = !(pmid <= R[IPR]);
  const double ql = shl ? sqrt(1. + gf * (pmid / L[IPR] - 1.)) : 1.;
  const double qr = shr ? sqrt(1. + gf * (pmid / R[IPR] - 1.)) : 1.;
  const double al = L[ivx] - cl * ql;
  const double ar = R[ivx] + cr * qr;
  const double bp = ar > 0. ? ar : TINY;
  const double bm = al < 0. ? al : -TINY;
  const double vxl1 = L[ivx] - al, vxr1 = R[ivx] - ar;
  const double tl = L[IPR] + vxl1 * L[IDN] * L[ivx];
  const double tr = R[IPR] + vxr1 * R[IDN] * R[ivx];
  const double ml = L[IDN] * vxl1;
  const double mr = -(R[IDN] * vxr1);
  const double ims = 1. / (ml + mr);
  const double am = (tl - tr) * ims;
  const double cpr = (ml * tr + mr * tl) * ims;
  const double cp = cpr > 0. ? cpr : 0.;
  const double vxl = L[ivx] - bm, vxr = R[ivx] - bp;
  double sl, sr, sm, id;
  const bool pos = am >= 0.;
  if (pos) {
    id = 1. / (am - bm);
    sl = am * id;
    sr = 0.;
    sm = -bm * id;
  } else {
    id = 1. / (bp - am);
    sl = 0.;
    sr = -am * id;
    sm = bp * id;
  }
  // F_k = sl fl_k + sr fr_k (+ sm cp in ivx, + sm cp am in IPR)
  const double fl[5] = {L[IDN] * vxl, L[IDN] * L[ivx] * vxl + L[IPR], L[IDN] * L[ivy] * vxl,
                        L[IDN] * L[ivz] * vxl, el * vxl + L[IPR] * L[ivx]};
  const double fr[5] = {R[IDN] * vxr, R[IDN] * R[ivx] * vxr + R[IPR], R[IDN] * R[ivy] * vxr,
                        R[IDN] * R[ivz] * vxr, er * vxr + R[IPR] * R[ivx]};
  const double g[5] = {gF[IDN], gF[ivx], gF[ivy], gF[ivz], gF[IPR]};
  double gsl = 0., gsr = 0.;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    gsl += g[k] * fl[k];
    gsr += g[k] * fr[k];
  }
  const double gsm = g[1] * cp + g[4] * cp * am;
  double gcp = g[1] * sm + g[4] * sm * am;
  double gam = g[4] * sm * cp;
  double gbm = 0., gbp = 0.;
  // fl, fr with vxl = uL - bm, vxr = uR - bp
  double gel = 0., ger = 0.;
  {
    const double gvxl = sl * (g[0] * L[IDN] + g[1] * L[IDN] * L[ivx] + g[2] * L[IDN] * L[ivy] +
                              g[3] * L[IDN] * L[ivz] + g[4] * el);
    gL[IDN] += sl * (g[0] * vxl + g[1] * L[ivx] * vxl + g[2] * L[ivy] * vxl + g[3] * L[ivz] * vxl);
    gL[ivx] += sl * (g[1] * L[IDN] * vxl + g[4] * L[IPR]) + gvxl;
    gL[ivy] += sl * g[2] * L[IDN] * vxl;
    gL[ivz] += sl * g[3] * L[IDN] * vxl;
    gL[IPR] += sl * (g[1] + g[4] * L[ivx]);
    gel = sl * g[4] * vxl;
    gbm -= gvxl;
    const double gvxr = sr * (g[0] * R[IDN] + g[1] * R[IDN] * R[ivx] + g[2] * R[IDN] * R[ivy] +
                              g[3] * R[IDN] * R[ivz] + g[4] * er);
    gR[IDN] += sr * (g[0] * vxr + g[1] * R[ivx] * vxr + g[2] * R[ivy] * vxr + g[3] * R[ivz] * vxr);
    gR[ivx] += sr * (g[1] * R[IDN] * vxr + g[4] * R[IPR]) + gvxr;
    gR[ivy] += sr * g[2] * R[IDN] * vxr;
    gR[ivz] += sr * g[3] * R[IDN] * vxr;
    gR[IPR] += sr * (g[1] + g[4] * R[ivx]);
    ger = sr * g[4] * vxr;
    gbp -= gvxr;
  }
  // wave-speed weights
  if (pos) {
    const double id2 = id * id;
    gam += gsl * (-bm * id2) + gsm * (bm * id2);
    gbm += gsl * (am * id2) + gsm * (-am * id2);
  } else {
    const double id2 = id * id;
    gam += gsr * (-bp * id2) + gsm * (bp * id2);
    gbp += gsr * (am * id2) + gsm * (-am * id2);
  }
  // contact speed and pressure
  const double gcpr = cpr > 0. ? gcp : 0.;
  double gtl = gam * ims + gcpr * mr * ims;
  double gtr = -gam * ims + gcpr * ml * ims;
  double gml = gcpr * tr * ims, gmr = gcpr * tl * ims;
  const double gims = gam * (tl - tr) + gcpr * (ml * tr + mr * tl);
  const double gD = -gims * ims * ims;
  gml += gD;
  gmr += gD;
  double gvxl1 = gml * L[IDN], gvxr1 = -gmr * R[IDN];
  gL[IDN] += gml * vxl1;
  gR[IDN] += -gmr * vxr1;
  gL[IPR] += gtl;
  gvxl1 += gtl * L[IDN] * L[ivx];
  gL[IDN] += gtl * vxl1 * L[ivx];
  gL[ivx] += gtl * vxl1 * L[IDN];
  gR[IPR] += gtr;
  gvxr1 += gtr * R[IDN] * R[ivx];
  gR[IDN] += gtr * vxr1 * R[ivx];
  gR[ivx] += gtr * vxr1 * R[IDN];
  // vxl1 = uL - al, vxr1 = uR - ar
  gL[ivx] += gvxl1;
  double gal = -gvxl1;
  gR[ivx] += gvxr1;
  double gar = -gvxr1;
  if (ar > 0.) gar += gbp;
  if (al < 0.) gal += gbm;
  // al = uL - cl ql, ar = uR + cr qr
  gL[ivx] += gal;
  double gcl = -gal * ql, gql = -gal * cl;
  gR[ivx] += gar;
  double gcr = gar * qr, gqr = gar * cr;
  double gpmid = 0.;
  if (shl) {
    gpmid += gql * gf / (2. * ql * L[IPR]);
    gL[IPR] -= gql * gf * pmid / (2. * ql * L[IPR] * L[IPR]);
  }
  if (shr) {
    gpmid += gqr * gf / (2. * qr * R[IPR]);
    gR[IPR] -= gqr * gf * pmid / (2. * qr * R[IPR] * R[IPR]);
  }
  // pmid = (pL + pR + (uL - uR) rhoa ca)/2
  gL[IPR] += 0.5 * gpmid;
  gR[IPR] += 0.5 * gpmid;
  gL[ivx] += 0.5 * gpmid * rhoa * ca;
  gR[ivx] -= 0.5 * gpmid * rhoa * ca;
  const double grhoa = 0.5 * gpmid * (L[ivx] - R[ivx]) * ca;
  const double gca = 0.5 * gpmid * (L[ivx] - R[ivx]) * rhoa;
  gL[IDN] += 0.5 * grhoa;
  gR[IDN] += 0.5 * grhoa;
  gcl += 0.5 * gca;
  gcr += 0.5 * gca;
  // el, er: p/(gamma-1) + rho |v|^2 / 2
  gL[IPR] += gel * igm1;
  gL[IDN] += gel * 0.5 * (sqr(L[IVX]) + sqr(L[IVY]) + sqr(L[IVZ]));
  gR[IPR] += ger * igm1;
  gR[IDN] += ger * 0.5 * (sqr(R[IVX]) + sqr(R[IVY]) + sqr(R[IVZ]));
#pragma unroll
  for (int v = IVX; v <= IVZ; ++v) {
    gL[v] += gel * L[IDN] * L[v];
    gR[v] += ger * R[IDN] * R[v];
  }
  // c = sqrt(gamma p / rho)
  gL[IPR] += gcl * cl / (2. * L[IPR]);
  gL[IDN] -= gcl * cl / (2. * L[IDN]);
  gR[IPR] += gcr * cr / (2. * R[IPR]);
  gR[IDN] -= gcr * cr / (2. * R[IDN]);
}

// ---------------------------------------------------------------------------
// Roe (with the LLF fallback on negative intermediate densities)
// ---------------------------------------------------------------------------
// reverse of the physical flux f(S) = (rho u, rho u^2 + p, rho u v, rho u w,
// (E + p) u) with coefficients c[k] on f_k; E's cotangent is returned in *gE
__device__ __forceinline__ void euler_flux_vjp(const double* S, double E, int ivx, int ivy,
                                               int ivz, const double* c, double* gS,
                                               double* gE) {
  const double r = S[IDN], u = S[ivx], vy = S[ivy], vz = S[ivz], p = S[IPR];
  gS[IDN] += c[0] * u + c[1] * u * u + c[2] * u * vy + c[3] * u * vz;
  gS[ivx] += c[0] * r + c[1] * 2. * r * u + c[2] * r * vy + c[3] * r * vz + c[4] * (E + p);
  gS[ivy] += c[2] * r * u;
  gS[ivz] += c[3] * r * u;
  gS[IPR] += c[1] + c[4] * u;
  *gE += c[4] * u;
}

// reverse of E = p/(gamma-1) + rho |v|^2 / 2
__device__ __forceinline__ void energy_vjp(const double* S, double igm1, double gE, double* gS) {
  gS[IPR] += gE * igm1;
  gS[IDN] += gE * 0.5 * (sqr(S[IVX]) + sqr(S[IVY]) + sqr(S[IVZ]));
#pragma unroll
  for (int v = IVX; v <= IVZ; ++v) gS[v] += gE * S[IDN] * S[v];
}

__device__ __forceinline__ double sgn_of(double x) { return x < 0. ? -1. : 1.; }

__device__ __forceinline__ void roe_vjp(const double* L, const double* R, int ivx, double gamma,
                                        const double* gF, double* gL, double* gR) {
  const double TINY = 1.0e-10;
  const int ivy = IVX + (ivx - IVX + 1) % 3;
  const int ivz = IVX + (ivx - IVX + 2) % 3;
  const double igm1 = 1. / (gamma - 1.);
  const double etl = L[IPR] * igm1 + 0.5 * L[IDN] * (sqr(L[IVX]) + sqr(L[IVY]) + sqr(L[IVZ]));
  const double etr = R[IPR] * igm1 + 0.5 * R[IDN] * (sqr(R[IVX]) + sqr(R[IVY]) + sqr(R[IVZ]));
  const double sdl = sqrt(L[IDN]), sdr = sqrt(R[IDN]);
  const double isd = 1. / (sdl + sdr);
  const double rhobar = sdl * sdr;
  const double v1 = (sdl * L[ivx] + sdr * R[ivx]) * isd;
  const double v2 = (sdl * L[ivy] + sdr * R[ivy]) * isd;
  const double v3 = (sdl * L[ivz] + sdr * R[ivz]) * isd;
  const double hl = (etl + L[IPR]) / L[IDN];
  const double hr = (etr + R[IPR]) / R[IDN];
  const double h = (hl * sdl + hr * sdr) * isd;
  const double A = L[IDN] / sdl + R[IDN] / sdr;
  const double qbar = A * isd;
  const double vsq = v1 * v1 + v2 * v2 + v3 * v3;
  const double gm1 = gamma - 1.;
  const double q = h - 0.5 * vsq;
  const double qq = q > TINY ? q : TINY;
  const double csr = gm1 * qq;
  const double cs_sq = csr > TINY ? csr : TINY;
  const double cs = sqrt(cs_sq);
  const double lam_m = v1 - cs, lam_p = v1 + cs;
  const double spd_m = fabs(lam_m), spd_0 = fabs(v1), spd_p = fabs(lam_p);
  const double du = R[ivx] - L[ivx], dv = R[ivy] - L[ivy], dw = R[ivz] - L[ivz];
  const double dp = R[IPR] - L[IPR];
  const double ics = 1. / cs, ics2 = 1. / cs_sq;
  const double alpha_m = -0.5 * rhobar * ics * du + 0.5 * dp * ics2;
  const double alpha_p = 0.5 * rhobar * ics * du + 0.5 * dp * ics2;
  const double alpha_v = rhobar * dv, alpha_w = rhobar * dw;
  const double ac0 = R[IDN] - L[IDN] - dp * ics2 * qbar;
  const double rho1 = L[IDN] + alpha_m * qbar;
  const double rho2 = rho1 + ac0;
  const double g[5] = {gF[IDN], gF[ivx], gF[ivy], gF[ivz], gF[IPR]};
  double getl = 0., getr = 0.;
  if ((rho1 < 0.) || (rho2 < 0.)) {
    // local Lax-Friedrichs
    const double cl = sqrt(gamma * L[IPR] / L[IDN]);
    const double cr = sqrt(gamma * R[IPR] / R[IDN]);
    const double al = fabs(L[ivx]) + cl, ar = fabs(R[ivx]) + cr;
    const bool lmax = al > ar;
    const double a = 0.5 * (lmax ? al : ar);
    const double half[5] = {0.5 * g[0], 0.5 * g[1], 0.5 * g[2], 0.5 * g[3], 0.5 * g[4]};
    euler_flux_vjp(L, etl, ivx, ivy, ivz, half, gL, &getl);
    euler_flux_vjp(R, etr, ivx, ivy, ivz, half, gR, &getr);
    const double ga = -(g[0] * (R[IDN] - L[IDN]) + g[1] * (R[IDN] * R[ivx] - L[IDN] * L[ivx]) +
                        g[2] * (R[IDN] * R[ivy] - L[IDN] * L[ivy]) +
                        g[3] * (R[IDN] * R[ivz] - L[IDN] * L[ivz]) + g[4] * (etr - etl));
    // - a (conserved jump)
    gR[IDN] -= a * (g[0] + g[1] * R[ivx] + g[2] * R[ivy] + g[3] * R[ivz]);
    gL[IDN] += a * (g[0] + g[1] * L[ivx] + g[2] * L[ivy] + g[3] * L[ivz]);
    gR[ivx] -= a * g[1] * R[IDN];
    gL[ivx] += a * g[1] * L[IDN];
    gR[ivy] -= a * g[2] * R[IDN];
    gL[ivy] += a * g[2] * L[IDN];
    gR[ivz] -= a * g[3] * R[IDN];
    gL[ivz] += a * g[3] * L[IDN];
    getr -= a * g[4];
    getl += a * g[4];
    const double gsel = 0.5 * ga;
    if (lmax) {
      gL[ivx] += gsel * sgn_of(L[ivx]);
      gL[IPR] += gsel * cl / (2. * L[IPR]);
      gL[IDN] -= gsel * cl / (2. * L[IDN]);
    } else {
      gR[ivx] += gsel * sgn_of(R[ivx]);
      gR[IPR] += gsel * cr / (2. * R[IPR]);
      gR[IDN] -= gsel * cr / (2. * R[IDN]);
    }
    energy_vjp(L, igm1, getl, gL);
    energy_vjp(R, igm1, getr, gR);
    return;
  }
  if (lam_m > 0.) {
    euler_flux_vjp(L, etl, ivx, ivy, ivz, g, gL, &getl);
    energy_vjp(L, igm1, getl, gL);
    return;
  }
  if (lam_p < 0.) {
    euler_flux_vjp(R, etr, ivx, ivy, ivz, g, gR, &getr);
    energy_vjp(R, igm1, getr, gR);
    return;
  }
  // central average minus the wave dissipation
  const double half[5] = {0.5 * g[0], 0.5 * g[1], 0.5 * g[2], 0.5 * g[3], 0.5 * g[4]};
  euler_flux_vjp(L, etl, ivx, ivy, ivz, half, gL, &getl);
  euler_flux_vjp(R, etr, ivx, ivy, ivz, half, gR, &getr);
  const double G0 = -0.5 * g[0], G1 = -0.5 * g[1], G2 = -0.5 * g[2], G3 = -0.5 * g[3],
               G4 = -0.5 * g[4];
  const double X = rhobar * (hr - hl - v1 * du) + ac0 * h - dp;
  const double Pm = G0 * qbar + G1 * (v1 - cs) + G2 * v2 + G3 * v3 + G4 * (h - v1 * cs);
  const double Pp = G0 * qbar + G1 * (v1 + cs) + G2 * v2 + G3 * v3 + G4 * (h + v1 * cs);
  const double g_sm = alpha_m * Pm, g_am = spd_m * Pm;
  const double g_sp = alpha_p * Pp, g_ap = spd_p * Pp;
  const double g_s0 = G0 * ac0 + G1 * v1 * ac0 + G2 * (v2 * ac0 + alpha_v) +
                      G3 * (v3 * ac0 + alpha_w) + G4 * X;
  double g_ac0 = spd_0 * (G0 + G1 * v1 + G2 * v2 + G3 * v3 + G4 * h);
  const double g_av = spd_0 * G2, g_aw = spd_0 * G3;
  const double wsum = spd_m * alpha_m + spd_0 * ac0 + spd_p * alpha_p;
  double g_qbar = G0 * (spd_m * alpha_m + spd_p * alpha_p);
  double g_v1 = G1 * wsum + G4 * (-spd_m * alpha_m * cs + spd_p * alpha_p * cs) -
                spd_0 * G4 * rhobar * du;
  double g_cs = G1 * (-spd_m * alpha_m + spd_p * alpha_p) +
                G4 * (-spd_m * alpha_m * v1 + spd_p * alpha_p * v1);
  double g_v2 = G2 * wsum, g_v3 = G3 * wsum;
  double g_h = G4 * wsum;
  double g_rhobar = spd_0 * G4 * (hr - hl - v1 * du);
  double g_hr = spd_0 * G4 * rhobar, g_hl = -spd_0 * G4 * rhobar;
  double g_du = -spd_0 * G4 * rhobar * v1;
  double g_dp = -spd_0 * G4;
  double g_dv = 0., g_dw = 0.;
  // wave speeds
  g_v1 += g_sm * sgn_of(lam_m) + g_s0 * sgn_of(v1) + g_sp * sgn_of(lam_p);
  g_cs += -g_sm * sgn_of(lam_m) + g_sp * sgn_of(lam_p);
  // ac0 = rhoR - rhoL - dp ics2 qbar
  gR[IDN] += g_ac0;
  gL[IDN] -= g_ac0;
  g_dp -= g_ac0 * ics2 * qbar;
  double g_ics2 = -g_ac0 * dp * qbar;
  g_qbar -= g_ac0 * dp * ics2;
  // alpha_v, alpha_w
  g_rhobar += g_av * dv + g_aw * dw;
  g_dv += g_av * rhobar;
  g_dw += g_aw * rhobar;
  // alpha_m, alpha_p
  double g_ics = (g_ap - g_am) * 0.5 * rhobar * du;
  g_rhobar += (g_ap - g_am) * 0.5 * ics * du;
  g_du += (g_ap - g_am) * 0.5 * rhobar * ics;
  g_dp += (g_am + g_ap) * 0.5 * ics2;
  g_ics2 += (g_am + g_ap) * 0.5 * dp;
  // ics = 1/cs, ics2 = 1/cs_sq, cs = sqrt(cs_sq), clamps
  g_cs -= g_ics * ics * ics;
  double g_cssq = -g_ics2 * ics2 * ics2 + g_cs / (2. * cs);
  const double g_qq = csr > TINY ? g_cssq * gm1 : 0.;
  const double g_q = q > TINY ? g_qq : 0.;
  g_h += g_q;
  g_v1 -= g_q * v1;
  g_v2 -= g_q * v2;
  g_v3 -= g_q * v3;
  // jumps
  gR[ivx] += g_du;
  gL[ivx] -= g_du;
  gR[ivy] += g_dv;
  gL[ivy] -= g_dv;
  gR[ivz] += g_dw;
  gL[ivz] -= g_dw;
  gR[IPR] += g_dp;
  gL[IPR] -= g_dp;
  // Roe averages
  double g_sdl = 0., g_sdr = 0., g_isd = 0.;
  g_isd += g_qbar * A;
  {
    const double gA = g_qbar * isd;
    gL[IDN] += gA / sdl;
    gR[IDN] += gA / sdr;
    g_sdl -= gA * L[IDN] / (sdl * sdl);
    g_sdr -= gA * R[IDN] / (sdr * sdr);
  }
  g_hl += g_h * sdl * isd;
  g_hr += g_h * sdr * isd;
  g_sdl += g_h * hl * isd;
  g_sdr += g_h * hr * isd;
  g_isd += g_h * (hl * sdl + hr * sdr);
  getl += g_hl / L[IDN];
  gL[IPR] += g_hl / L[IDN];
  gL[IDN] -= g_hl * (etl + L[IPR]) / (L[IDN] * L[IDN]);
  getr += g_hr / R[IDN];
  gR[IPR] += g_hr / R[IDN];
  gR[IDN] -= g_hr * (etr + R[IPR]) / (R[IDN] * R[IDN]);
  const int sl3[3] = {ivx, ivy, ivz};
  const double gv[3] = {g_v1, g_v2, g_v3};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int c = sl3[k];
    g_sdl += gv[k] * L[c] * isd;
    g_sdr += gv[k] * R[c] * isd;
    gL[c] += gv[k] * sdl * isd;
    gR[c] += gv[k] * sdr * isd;
    g_isd += gv[k] * (sdl * L[c] + sdr * R[c]);
  }
  g_sdl += g_rhobar * sdr;
  g_sdr += g_rhobar * sdl;
  g_sdl -= g_isd * isd * isd;
  g_sdr -= g_isd * isd * isd;
  gL[IDN] += g_sdl / (2. * sdl);
  gR[IDN] += g_sdr / (2. * sdr);
  energy_vjp(L, igm1, getl, gL);
  energy_vjp(R, igm1, getr, gR);
}

// gL += (dF/dL)^T gF, gR += (dF/dR)^T gF for the hydro solvers
__device__ __forceinline__ void riemann_vjp_rev(int solver, const double* L, const double* R,
                                                int ivx, double gamma, const double* gF,
                                                double* gL, double* gR) {
  if (solver == SNAPB_RIEMANN_HLLC)
    hllc_vjp(L, R, ivx, gamma, gF, gL, gR);
  else if (solver == SNAPB_RIEMANN_LMARS)
    lmars_vjp(L, R, ivx, gamma, gF, gL, gR);
  else
    roe_vjp(L, R, ivx, gamma, gF, gL, gR);
}

}  // namespace snapb
