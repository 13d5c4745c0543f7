// kflux.h — face reconstruction (PPM / minmod-theta / donor), the one-sided
// advective flux and the LAXF/HLL combiners. Shared host/device restatement of
// koral/fv/recon.zig, koral/physics/flux.zig and koral/fv/laxf.zig.
#pragma once
#include "kinvert.h"

namespace kp {

struct Faces {
  double left, right;
};

// C finite.c:126 (recon.zig:84), FLUXLIMITER 0
KC_HD Faces recon_linear(const double u[5], double theta) {
  double deltam = u[2] - u[1];
  double deltap = u[3] - u[2];
  double smin = kmath::fmin(kmath::fmin(theta * deltam, 0.5 * (deltam + deltap)), theta * deltap);
  double smax = kmath::fmax(kmath::fmax(theta * deltam, 0.5 * (deltam + deltap)), theta * deltap);
  double slope = (deltam > 0.0) ? smin : smax;
  if (deltam * deltap <= 0.0) slope = 0.0;
  Faces f;
  f.left = u[2] - 0.5 * slope;
  f.right = u[2] + 0.5 * slope;
  return f;
}

KC_HD double my_sign_pm(double x) { return (x >= 0.0) ? 1.0 : -1.0; }

// PPM with non-uniform widths, C finite.c:210 (recon.zig:107). The factors
// that depend only on the five cell widths are formed once per stencil
// position (ppm_coef) and shared by every variable reconstructed there
// (ppm_apply). Each factor is a leading sub-product of the reference's
// left-to-right expressions, so the split gives the one-piece routine's bits.
struct PpmCoef {
  double a, b, c;     // dri   = a * (b * (u3 - u2) + c * (u2 - u1))
  double d, e, f;     // drip1 = d * (e * (u4 - u3) + f * (u3 - u2))
  double g, h, i;     // drim1 = g * (h * (u2 - u1) + i * (u1 - u0))
  double rm, rj, rk, rl, r_inv;  // right face
  double lm, lj, lk, ll, l_inv;  // left face
};
KC_HD PpmCoef ppm_coef(const double dx[5]) {
  double dxm2 = dx[0], dxm1 = dx[1], dx0 = dx[2], dxp1 = dx[3], dxp2 = dx[4];
  double dxp2_plus_dxp1 = dxp2 + dxp1;
  double dxp2_plus_dxp1_inv = 1.0 / dxp2_plus_dxp1;
  double dxp1_plus_dx0 = dxp1 + dx0;
  double dxp1_plus_dx0_inv = 1.0 / dxp1_plus_dx0;
  double dx0_plus_dxm1 = dx0 + dxm1;
  double dx0_plus_dxm1_inv = 1.0 / dx0_plus_dxm1;
  double dxm1_plus_dxm2 = dxm1 + dxm2;
  double dxm1_plus_dxm2_inv = 1.0 / dxm1_plus_dxm2;
  double dxm1_plus_dx0_plus_dxp1_inv = 1.0 / (dxm1 + dx0 + dxp1);
  double dx0_plus_dxp1_plus_dxp2_inv = 1.0 / (dx0 + dxp1 + dxp2);
  double dxm2_plus_dxm1_plus_dx0_inv = 1.0 / (dxm2 + dxm1 + dx0);
  double dx0_plus_twodxm1 = dx0 + 2.0 * dxm1;
  double dxp1_plus_twodx0 = dxp1 + 2.0 * dx0;
  double dxm1_plus_twodxm2 = dxm1 + 2.0 * dxm2;
  double twodxp1_plus_dx0 = 2.0 * dxp1 + dx0;
  double twodxp2_plus_dxp1 = 2.0 * dxp2 + dxp1;
  double twodx0_plus_dxm1 = 2.0 * dx0 + dxm1;
  PpmCoef k;
  k.a = dx0 * dxm1_plus_dx0_plus_dxp1_inv;
  k.b = dx0_plus_twodxm1 * dxp1_plus_dx0_inv;
  k.c = twodxp1_plus_dx0 * dx0_plus_dxm1_inv;
  k.d = dxp1 * dx0_plus_dxp1_plus_dxp2_inv;
  k.e = dxp1_plus_twodx0 * dxp2_plus_dxp1_inv;
  k.f = twodxp2_plus_dxp1 * dxp1_plus_dx0_inv;
  k.g = dxm1 * dxm2_plus_dxm1_plus_dx0_inv;
  k.h = dxm1_plus_twodxm2 * dx0_plus_dxm1_inv;
  k.i = twodx0_plus_dxm1 * dxm1_plus_dxm2_inv;
  double z1 = dx0_plus_dxm1 / dxp1_plus_twodx0;
  double z2 = dxp2_plus_dxp1 / twodxp1_plus_dx0;
  k.r_inv = 1.0 / (dxm1 + dx0 + dxp1 + dxp2);
  k.rm = dx0 * dxp1_plus_dx0_inv;
  k.rj = (2.0 * dxp1 * dx0) * dxp1_plus_dx0_inv * (z1 - z2);
  k.rk = dx0 * z1;
  k.rl = dxp1 * z2;
  z1 = dxm1_plus_dxm2 / dx0_plus_twodxm1;
  z2 = dxp1_plus_dx0 / twodx0_plus_dxm1;
  k.l_inv = 1.0 / (dxm2 + dxm1 + dx0 + dxp1);
  k.lm = dxm1 * dx0_plus_dxm1_inv;
  k.lj = (2.0 * dx0 * dxm1) * dx0_plus_dxm1_inv * (z1 - z2);
  k.lk = dxm1 * z1;
  k.ll = dx0 * z2;
  return k;
}
KC_HD Faces ppm_apply(const double u[5], const PpmCoef& k) {
  double dri = k.a * (k.b * (u[3] - u[2]) + k.c * (u[2] - u[1]));
  double drip1 = k.d * (k.e * (u[4] - u[3]) + k.f * (u[3] - u[2]));
  double drim1 = k.g * (k.h * (u[2] - u[1]) + k.i * (u[1] - u[0]));

  dri = ((u[3] - u[2]) * (u[2] - u[1]) > 0.0)
            ? kmath::fmin(kmath::fabs(dri),
                          kmath::fmin(2.0 * kmath::fabs(u[2] - u[1]), 2.0 * kmath::fabs(u[2] - u[3]))) * my_sign_pm(dri)
            : 0.0;
  drip1 = ((u[4] - u[3]) * (u[3] - u[2]) > 0.0)
              ? kmath::fmin(kmath::fabs(drip1),
                            kmath::fmin(2.0 * kmath::fabs(u[3] - u[2]), 2.0 * kmath::fabs(u[3] - u[4]))) * my_sign_pm(drip1)
              : 0.0;
  drim1 = ((u[2] - u[1]) * (u[1] - u[0]) > 0.0)
              ? kmath::fmin(kmath::fabs(drim1),
                            kmath::fmin(2.0 * kmath::fabs(u[1] - u[0]), 2.0 * kmath::fabs(u[1] - u[2]))) * my_sign_pm(drim1)
              : 0.0;

  double right = u[2] + k.rm * (u[3] - u[2]) + k.r_inv * (k.rj * (u[3] - u[2]) - k.rk * drip1 + k.rl * dri);
  double left = u[1] + k.lm * (u[2] - u[1]) + k.l_inv * (k.lj * (u[2] - u[1]) - k.lk * dri + k.ll * drim1);

  bool flat = (right - u[2]) * (u[2] - left) <= 0.0;
  if (flat) {
    left = u[2];
    right = u[2];
  }
  if ((right - left) * (left - (3.0 * u[2] - 2.0 * right)) < 0.0) left = 3.0 * u[2] - 2.0 * right;
  if ((right - left) * ((3.0 * u[2] - 2.0 * left) - right) < 0.0) right = 3.0 * u[2] - 2.0 * left;
  Faces f;
  f.left = left;
  f.right = right;
  return f;
}
KC_HD Faces recon_ppm(const double u[5], const double dx[5]) { return ppm_apply(u, ppm_coef(dx)); }

enum : int { RECON_DONOR = 0, RECON_LINEAR = 1, RECON_PPM = 2 };
KC_HD Faces reconstruct(int scheme, const double u[5], const double dx[5], double theta) {
  if (scheme == RECON_PPM) return recon_ppm(u, dx);
  if (scheme == RECON_LINEAR) return recon_linear(u, theta);
  Faces f;
  f.left = u[2];
  f.right = u[2];
  return f;
}

// C f_flux_prime (koral/physics/flux.zig:40). Returns E_NANFLUX on a
// non-finite flux.
// (the body, inlined by kernels that keep its arrays in registers)
KC_HD int f_flux_prime_inl(const double pp[NV], int idim, const Geom& g, double gam, double ff[NV]) {
  double gdetu = g.gdet;
  double rho = pp[RHO], ugas = pp[UU], s = pp[ENTR];
  double vcon[4] = {0.0, pp[VX], pp[VY], pp[VZ]};
  double ucon[4], ucov[4];
  velr_to_vel4(vcon, g, ucon);
  lower_vec(ucon, g, ucov);
  double B[3] = {pp[B1], pp[B2], pp[B3]};
  double bcon[4], bcov[4], bsq;
  bcon_bcov_bsq(B, ucon, ucov, g, bcon, bcov, bsq);
  double tij_uu[4][4];
  tij_from_state(pp, g, gam, ucon, bcon, bsq, tij_uu);
  double trow[4];
  lower_second_row(tij_uu, g, idim + 1, trow);
  double pre = (gam - 1.0) * ugas;
  double etap = ugas + pre + bsq;
  double utp1 = calc_utp1(vcon, g);
  int d = idim + 1;
  ff[RHO] = gdetu * rho * ucon[d];
  ff[ENTR] = gdetu * s * ucon[d];
  ff[UU] = gdetu * (etap * ucon[d] * ucov[0] + rho * ucon[d] * utp1);
  ff[UU] += -gdetu * bcon[d] * bcov[0];
  ff[VX] = gdetu * trow[1];
  ff[VY] = gdetu * trow[2];
  ff[VZ] = gdetu * trow[3];
  ff[B1] = gdetu * (bcon[1] * ucon[d] - bcon[d] * ucon[1]);
  ff[B2] = gdetu * (bcon[2] * ucon[d] - bcon[d] * ucon[2]);
  ff[B3] = gdetu * (bcon[3] * ucon[d] - bcon[d] * ucon[3]);
  double rij_uu[4][4], rrow[4];
  calc_rij(pp, g, rij_uu);
  lower_second_row(rij_uu, g, d, rrow);
  for (int nu = 0; nu < 4; ++nu) ff[EE + nu] = gdetu * rrow[nu];
  for (int i = 0; i < NV; ++i)
    if (!kmath::isfinite(ff[i])) return E_NANFLUX;
  return E_OK;
}
KC_HDN int f_flux_prime(const double pp[NV], int idim, const Geom& g, double gam, double ff[NV]) { return f_flux_prime_inl(pp, idim, g, gam, ff); }

// Lax-Friedrichs, koral/fv/laxf.zig:13
KC_HD double laxf(double fl, double fr, double ul, double ur, double ag) { return 0.5 * (fr + fl - ag * (ur - ul)); }
// HLL, koral/fv/laxf.zig:19
KC_HD double hll(double fl, double fr, double ul, double ur, double al, double ar) {
  if (al > 0.0) return fl;
  if (ar < 0.0) return fr;
  return (-al * fr + ar * fl + al * ar * (ur - ul)) / (ar - al);
}

}  // namespace kp
