// pert.cuh — FP32 perturbation form: Riemann fluxes with the pressure split.
//
// The state is stored as FP32 perturbations about an FP64 reference profile
// rho_bar(x1), p_bar(x1).  At a face the pressure is p = pf + p', with pf an
// FP64 face reference value common to both sides.  These solvers take the full
// FP32 states (for wave speeds, enthalpies, upwinding) and the perturbation
// pressures p'L, p'R, and return the flux WITHOUT the pf term in the normal
// momentum component: F_mom = F_mom(full) - pf.  Every solver's normal momentum
// flux is pf times a weight sum of exactly one plus terms in p', so the split
// is exact algebra; it removes the catastrophic cancellation of the large
// hydrostatic pressure in FP32.  Energy fluxes keep the full pressure.
// Formulas as in common.cuh (src/riemann/{hllc,lmars,roe}_impl.h).
#pragma once

#include "common.cuh"

namespace snapb {

__device__ __forceinline__ void hllc_flux_split(const float* L, const float* R, float pl,
                                                float pr, float pf, int ivx, float gamma,
                                                float* F) {
  const float TINY = 1.0e-10f;
  int ivy = IVX + (ivx - IVX + 1) % 3;
  int ivz = IVX + (ivx - IVX + 2) % 3;
  float igm1 = fdiv(1.f, gamma - 1.f);
  float cl = sqrtf(fdiv(gamma * L[IPR], L[IDN]));
  float cr = sqrtf(fdiv(gamma * R[IPR], R[IDN]));
  float el = L[IPR] * igm1 + 0.5f * L[IDN] * (sqr(L[IVX]) + sqr(L[IVY]) + sqr(L[IVZ]));
  float er = R[IPR] * igm1 + 0.5f * R[IDN] * (sqr(R[IVX]) + sqr(R[IVY]) + sqr(R[IVZ]));
  float rhoa = 0.5f * (L[IDN] + R[IDN]);
  float ca = 0.5f * (cl + cr);
  float pmid = 0.5f * (L[IPR] + R[IPR] + (L[ivx] - R[ivx]) * rhoa * ca);
  float gf = fdiv(gamma + 1.f, 2.f * gamma);
  float ql = pmid <= L[IPR] ? 1.f : sqrtf(1.f + gf * (fdiv(pmid, L[IPR]) - 1.f));
  float qr = pmid <= R[IPR] ? 1.f : sqrtf(1.f + gf * (fdiv(pmid, R[IPR]) - 1.f));
  float al = L[ivx] - cl * ql;
  float ar = R[ivx] + cr * qr;
  float bp = ar > 0.f ? ar : TINY;
  float bm = al < 0.f ? al : -TINY;
  float vxl = L[ivx] - al;
  float vxr = R[ivx] - ar;
  float tl = pl + vxl * L[IDN] * L[ivx];  // perturbation parts of tl, tr
  float tr = pr + vxr * R[IDN] * R[ivx];
  float ml = L[IDN] * vxl;
  float mr = -(R[IDN] * vxr);
  float ims = fdiv(1.f, ml + mr);
  float am = (tl - tr) * ims;
  float cpp = (ml * tr + mr * tl) * ims;  // contact pressure minus pf
  if (pf + cpp <= 0.f) cpp = -pf;         // clamp of the full contact pressure at 0
  float cp = pf + cpp;
  vxl = L[ivx] - bm;
  vxr = R[ivx] - bp;
  float sl, sr, sm;
  if (am >= 0.f) {
    float id = fdiv(1.f, am - bm);
    sl = am * id;
    sr = 0.f;
    sm = -bm * id;
  } else {
    float id = fdiv(1.f, bp - am);
    sl = 0.f;
    sr = -am * id;
    sm = bp * id;
  }
  float fl, fr;
  F[IDN] = sl * (L[IDN] * vxl) + sr * (R[IDN] * vxr);
  fl = L[IDN] * L[ivx] * vxl + pl;
  fr = R[IDN] * R[ivx] * vxr + pr;
  F[ivx] = sl * fl + sr * fr + sm * cpp;
  F[ivy] = sl * (L[IDN] * L[ivy] * vxl) + sr * (R[IDN] * R[ivy] * vxr);
  F[ivz] = sl * (L[IDN] * L[ivz] * vxl) + sr * (R[IDN] * R[ivz] * vxr);
  fl = el * vxl + L[IPR] * L[ivx];
  fr = er * vxr + R[IPR] * R[ivx];
  F[IPR] = sl * fl + sr * fr + sm * cp * am;
}

__device__ __forceinline__ void lmars_flux_split(const float* L, const float* R, float pl,
                                                 float pr, int ivx, float gamma, float* F) {
  int ivy = IVX + (ivx - IVX + 1) % 3;
  int ivz = IVX + (ivx - IVX + 2) % 3;
  float igm1 = fdiv(1.f, gamma - 1.f);
  float irl = fdiv(1.f, L[IDN]), irr = fdiv(1.f, R[IDN]);
  float hl = L[IPR] * igm1 * irl + 0.5f * (sqr(L[ivx]) + sqr(L[ivy]) + sqr(L[ivz])) + L[IPR] * irl;
  float hr = R[IPR] * igm1 * irr + 0.5f * (sqr(R[ivx]) + sqr(R[ivy]) + sqr(R[ivz])) + R[IPR] * irr;
  float rhobar = 0.5f * (L[IDN] + R[IDN]);
  float cbar = sqrtf(fdiv(0.5f * gamma * (L[IPR] + R[IPR]), rhobar));
  float pbarp = 0.5f * (pl + pr) + 0.5f * (rhobar * cbar) * (L[ivx] - R[ivx]);
  float ubar = 0.5f * (L[ivx] + R[ivx]) + fdiv(0.5f, rhobar * cbar) * (pl - pr);
  const float* S = ubar > 0.f ? L : R;
  float h = ubar > 0.f ? hl : hr;
  float m = ubar * S[IDN];
  F[IDN] = m;
  F[ivx] = m * S[ivx] + pbarp;
  F[ivy] = m * S[ivy];
  F[ivz] = m * S[ivz];
  F[IPR] = m * h;
}

__device__ __forceinline__ void roe_flux_split(const float* L, const float* R, float pl,
                                               float pr, int ivx, float gamma, float* F) {
  const float TINY = 1.0e-10f;
  int ivy = IVX + (ivx - IVX + 1) % 3;
  int ivz = IVX + (ivx - IVX + 2) % 3;
  float igm1 = fdiv(1.f, gamma - 1.f);
  float etl = L[IPR] * igm1 + 0.5f * L[IDN] * (sqr(L[IVX]) + sqr(L[IVY]) + sqr(L[IVZ]));
  float etr = R[IPR] * igm1 + 0.5f * R[IDN] * (sqr(R[IVX]) + sqr(R[IVY]) + sqr(R[IVZ]));
  float sdl = sqrtf(L[IDN]), sdr = sqrtf(R[IDN]);
  float isd = fdiv(1.f, sdl + sdr);
  float rhobar = sdl * sdr;
  float v1 = (sdl * L[ivx] + sdr * R[ivx]) * isd;
  float v2 = (sdl * L[ivy] + sdr * R[ivy]) * isd;
  float v3 = (sdl * L[ivz] + sdr * R[ivz]) * isd;
  float hl = fdiv(etl + L[IPR], L[IDN]);
  float hr = fdiv(etr + R[IPR], R[IDN]);
  float h = (hl * sdl + hr * sdr) * isd;
  float rl0 = L[IDN], rr0 = R[IDN];
  float fl0 = rl0 * L[ivx], fr0 = rr0 * R[ivx];
  float fl1 = L[IDN] * L[ivx] * L[ivx] + pl, fr1 = R[IDN] * R[ivx] * R[ivx] + pr;
  float fl2 = L[IDN] * L[ivx] * L[ivy], fr2 = R[IDN] * R[ivx] * R[ivy];
  float fl3 = L[IDN] * L[ivx] * L[ivz], fr3 = R[IDN] * R[ivx] * R[ivz];
  float fl4 = (etl + L[IPR]) * L[ivx], fr4 = (etr + R[IPR]) * R[ivx];
  float qbar = (fdiv(rl0, sdl) + fdiv(rr0, sdr)) * isd;
  float vsq = v1 * v1 + v2 * v2 + v3 * v3;
  float q = h - 0.5f * vsq;
  float qq = q > TINY ? q : TINY;
  float cs_sq = (gamma - 1.f) * qq;
  cs_sq = cs_sq > TINY ? cs_sq : TINY;
  float cs = sqrtf(cs_sq);
  float lam_m = v1 - cs, lam_p = v1 + cs;
  float spd_m = fabsf(lam_m), spd_0 = fabsf(v1), spd_p = fabsf(lam_p);
  float du = R[ivx] - L[ivx], dv = R[ivy] - L[ivy], dw = R[ivz] - L[ivz];
  float dp = pr - pl;
  float ics = fdiv(1.f, cs), ics2 = fdiv(1.f, cs_sq);
  float alpha_m = -0.5f * rhobar * ics * du + 0.5f * dp * ics2;
  float alpha_p = 0.5f * rhobar * ics * du + 0.5f * dp * ics2;
  float ac0 = rr0 - rl0 - dp * ics2 * qbar;
  float rho1 = rl0 + alpha_m * qbar;
  bool llf = (rho1 < 0.f) || (rho1 + ac0 < 0.f);
  if (llf) {
    float cl = sqrtf(fdiv(gamma * L[IPR], L[IDN]));
    float cr = sqrtf(fdiv(gamma * R[IPR], R[IDN]));
    float a = 0.5f * fmaxf(fabsf(L[ivx]) + cl, fabsf(R[ivx]) + cr);
    F[IDN] = 0.5f * (fl0 + fr0) - a * (rr0 - rl0);
    F[ivx] = 0.5f * (fl1 + fr1) - a * (R[IDN] * R[ivx] - L[IDN] * L[ivx]);
    F[ivy] = 0.5f * (fl2 + fr2) - a * (R[IDN] * R[ivy] - L[IDN] * L[ivy]);
    F[ivz] = 0.5f * (fl3 + fr3) - a * (R[IDN] * R[ivz] - L[IDN] * L[ivz]);
    F[IPR] = 0.5f * (fl4 + fr4) - a * (etr - etl);
    return;
  }
  if (lam_m > 0.f) {
    F[IDN] = fl0, F[ivx] = fl1, F[ivy] = fl2, F[ivz] = fl3, F[IPR] = fl4;
    return;
  }
  if (lam_p < 0.f) {
    F[IDN] = fr0, F[ivx] = fr1, F[ivy] = fr2, F[ivz] = fr3, F[IPR] = fr4;
    return;
  }
  float a0 = ac0;
  F[IDN] = 0.5f * (fl0 + fr0) - 0.5f * (spd_m * alpha_m * qbar + spd_0 * ac0 + spd_p * alpha_p * qbar);
  F[ivx] = 0.5f * (fl1 + fr1) - 0.5f * (spd_m * alpha_m * (v1 - cs) + spd_0 * (v1 * a0) +
                                        spd_p * alpha_p * (v1 + cs));
  F[ivy] = 0.5f * (fl2 + fr2) - 0.5f * (spd_m * alpha_m * v2 + spd_0 * (v2 * a0 + rhobar * dv) +
                                        spd_p * alpha_p * v2);
  F[ivz] = 0.5f * (fl3 + fr3) - 0.5f * (spd_m * alpha_m * v3 + spd_0 * (v3 * a0 + rhobar * dw) +
                                        spd_p * alpha_p * v3);
  F[IPR] = 0.5f * (fl4 + fr4) - 0.5f * (spd_m * alpha_m * (h - v1 * cs) +
                                        spd_0 * (rhobar * (hr - hl - v1 * du) + a0 * h - dp) +
                                        spd_p * alpha_p * (h + v1 * cs));
}

__device__ __forceinline__ void riemann_flux_split(int solver, const float* L, const float* R,
                                                   float pl, float pr, float pf, int ivx,
                                                   float gamma, float* F) {
  if (solver == SNAPB_RIEMANN_HLLC)
    hllc_flux_split(L, R, pl, pr, pf, ivx, gamma, F);
  else if (solver == SNAPB_RIEMANN_LMARS)
    lmars_flux_split(L, R, pl, pr, ivx, gamma, F);
  else
    roe_flux_split(L, R, pl, pr, ivx, gamma, F);
}

// Face profiles: compile-time specializations of the FP32 sweeps.  Profile 0
// reads every reconstruction and solver choice at run time; profiles 1, 2 and
// 3 are the default reconstruction (WENO5 for density and scalars, the linear
// 5-point interpolation for velocities and pressure, no scaling) with the
// LMARS, HLLC and Roe solvers.  The host picks the profile (face_profile32).
template <int FP>
__device__ __forceinline__ void sweep_face_states(int typ, bool scale, int v, const float* q,
                                                  float& wl, float& wr) {
  if constexpr (FP == 0)
    face_states<float>(typ, scale, q, wl, wr);
  else
    face_states<float>(v == IDN || v >= 5 ? SNAPB_RECON_WENO5 : SNAPB_RECON_CP5, false, q, wl, wr);
}
template <int FP>
__device__ __forceinline__ void sweep_riemann(int solver, const float* L, const float* R, float pl,
                                              float pr, float pf, int ivx, float gamma, float* F) {
  if constexpr (FP == 1)
    lmars_flux_split(L, R, pl, pr, ivx, gamma, F);
  else if constexpr (FP == 2)
    hllc_flux_split(L, R, pl, pr, pf, ivx, gamma, F);
  else if constexpr (FP == 3)
    roe_flux_split(L, R, pl, pr, ivx, gamma, F);
  else
    riemann_flux_split(solver, L, R, pl, pr, pf, ivx, gamma, F);
}

// linear interpolation weights of the face states (cp5, cp3, dc): the value at
// the right face of q[2] (wl) and the left face of q[3] (wr) from six cells
__device__ __forceinline__ bool linear_face_states(int type, const float* q, float& wl,
                                                   float& wr) {
  if (type == SNAPB_RECON_CP5 || type == SNAPB_RECON_CP3 || type == SNAPB_RECON_DC) {
    face_states<float>(type, false, q, wl, wr);
    return true;
  }
  return false;
}

}  // namespace snapb
