// kcore.h — per-point geometry, velocity conversions, p2u and the MHD stress
// tensor, shared by the CPU oracle and the sm_100a kernels.
//
// Every function restates one reference function with the reference's
// operation order (no FMA contraction on either side), so the host and device
// builds produce identical bits. Reference paths are relative to the
// koral-zig project root.
#pragma once
#include "kmath.h"

namespace kp {

// ---- state-vector layout (koral/layout.zig:52, PUFFY: NV = 13) -------------
enum : int {
  RHO = 0, UU = 1, VX = 2, VY = 3, VZ = 4, ENTR = 5,
  B1 = 6, B2 = 7, B3 = 8, EE = 9, FX = 10, FY = 11, FZ = 12,
  NV = 13
};

// Internal error codes (the reference's relele.Error set, koral/relele.zig:51).
enum : int { E_OK = 0, E_VELCONV = 3, E_SPACELIKE = 4, E_NANFLUX = 5 };

enum VelType : int { VEL4 = 1, VEL3 = 2, VELR = 3 };  // koral/relele.zig:40
enum UtMode : int { RECOMPUTE_UT = 0, TRUST_UT = 1 };
enum Coords : int { MINK = 0, BL = 1, KS = 2, MKS2 = 3 };

// Per-point geometry (koral/geometry.zig:29): the 4x5 blocks keep C's layout,
// gg[i][4] = dln(sqrt -g)/dx^i for i<3, gg[3][4] = sqrt(-g), GG[3][4] = gttpert.
struct Geom {
  double gg[4][5];
  double GG[4][5];
  double gdet, alpha, gttpert;
  double xx[4];
};

// alpha exactly as MetricCache.geometryFromBlocks computes it
// (koral/metric/precompute.zig:467): sqrt(-1/g^tt).
KC_HD void geom_finish(Geom& g) {
  g.gdet = g.gg[3][4];
  g.gttpert = g.GG[3][4];
  g.alpha = kmath::sqrt(-1.0 / g.GG[0][0]);
}

KC_HD double kron(int i, int j) { return i == j ? 1.0 : 0.0; }

// koral/relele.zig:84
KC_HD double dot(const double a[4], const double b[4]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3];
}
// A_mu -> A^mu (koral/relele.zig:97, C indices_12)
KC_HD void raise_vec(const double a1[4], const Geom& g, double a2[4]) {
  double t[4];
  for (int i = 0; i < 4; ++i) {
    t[i] = 0.0;
    for (int k = 0; k < 4; ++k) t[i] += a1[k] * g.GG[i][k];
  }
  for (int i = 0; i < 4; ++i) a2[i] = t[i];
}
// A^mu -> A_mu (koral/relele.zig:112, C indices_21)
KC_HD void lower_vec(const double a1[4], const Geom& g, double a2[4]) {
  double t[4];
  for (int i = 0; i < 4; ++i) {
    t[i] = 0.0;
    for (int j = 0; j < 4; ++j) t[i] += a1[j] * g.gg[i][j];
  }
  for (int i = 0; i < 4; ++i) a2[i] = t[i];
}
// T^mu nu -> T^mu_nu (koral/relele.zig:160, C indices_2221)
KC_HDM void lower_second(const double t1[4][4], const Geom& g, double t2[4][4]) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double s = 0.0;
      for (int k = 0; k < 4; ++k) s += t1[i][k] * g.gg[k][j];
      t2[i][j] = s;
    }
}
// one row of lower_second (koral/relele.zig:179)
KC_HD void lower_second_row(const double t1[4][4], const Geom& g, int row, double out[4]) {
  for (int j = 0; j < 4; ++j) {
    double s = 0.0;
    for (int k = 0; k < 4; ++k) s += t1[row][k] * g.gg[k][j];
    out[j] = s;
  }
}
// T_mu nu -> T^mu nu (koral/relele.zig:127, C indices_1122)
KC_HDM void raise_both(const double t1[4][4], const Geom& g, double t2[4][4]) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double s = 0.0;
      for (int k = 0; k < 4; ++k)
        for (int l = 0; l < 4; ++l) s += t1[k][l] * g.GG[i][k] * g.GG[j][l];
      t2[i][j] = s;
    }
}
// uout^mu = A^mu_nu uin^nu (koral/relele.zig:191, C multiply2)
KC_HD void transform_vec(const double uin[4], const double a[4][4], double uout[4]) {
  double t[4];
  for (int i = 0; i < 4; ++i) {
    t[i] = 0.0;
    for (int j = 0; j < 4; ++j) t[i] += a[i][j] * uin[j];
  }
  for (int i = 0; i < 4; ++i) uout[i] = t[i];
}
// T2 = A A T1 (koral/relele.zig:205, C multiply22)
KC_HDM void transform_tensor(const double t1[4][4], const double a[4][4], double t2[4][4]) {
  double t[4][4];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double s = 0.0;
      for (int k = 0; k < 4; ++k)
        for (int l = 0; l < 4; ++l) s += a[i][k] * a[j][l] * t1[k][l];
      t[i][j] = s;
    }
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) t2[i][j] = t[i][j];
}

// u^t from VEL3 (koral/relele.zig:226, C fill_utinvel3)
KC_HD double ut_from_vel3(const double v[4], const Geom& g) {
  double b = 0.0, c = 0.0;
  for (int i = 1; i < 4; ++i) {
    b += v[i] * g.gg[0][i];
    for (int j = 1; j < 4; ++j) c += v[i] * v[j] * g.gg[i][j];
  }
  return kmath::sqrt(-1.0 / (g.gg[0][0] + 2.0 * b + c));
}
// u^t from spatial u^i (koral/relele.zig:243, C fill_utinucon)
KC_HD int ut_from_spatial_ucon(const double u[4], const Geom& g, double& ut) {
  double a = g.gg[0][0], b = 0.0, c = 1.0;
  for (int i = 1; i < 4; ++i) {
    b += u[i] * g.gg[0][i];
    for (int j = 1; j < 4; ++j) c += u[i] * u[j] * g.gg[i][j];
  }
  double delta = b * b - a * c;
  if (delta < 0.0) return E_SPACELIKE;
  ut = (-b - kmath::sqrt(delta)) / a;
  return E_OK;
}
// alpha*gamma of a VELR vector (koral/relele.zig:260, C calc_alpgam)
KC_HD double alpha_gamma(const double u[4], const Geom& g) {
  double qsq = 0.0;
  for (int i = 1; i < 4; ++i)
    for (int j = 1; j < 4; ++j) qsq += u[i] * u[j] * g.gg[i][j];
  double alpgam2 = (-1.0 / g.GG[0][0]) * (1.0 + qsq);
  return (alpgam2 < 0.0) ? 1.0 : kmath::sqrt(alpgam2);
}
// VELR -> VEL4, infallible (koral/relele.zig:276)
KC_HD void velr_to_vel4(const double uin[4], const Geom& g, double out[4]) {
  double alpgam = alpha_gamma(uin, g);
  double o0 = -alpgam * g.GG[0][0];
  double o1 = uin[1] - alpgam * g.GG[0][1];
  double o2 = uin[2] - alpgam * g.GG[0][2];
  double o3 = uin[3] - alpgam * g.GG[0][3];
  out[0] = o0;
  out[1] = o1;
  out[2] = o2;
  out[3] = o3;
}
// general contravariant conversion (koral/relele.zig:292, C conv_vels_core)
KC_HDM int convert(const double uin[4], int from, int to, const Geom& g, int utmode, double uout[4]) {
  bool ut_known = utmode == TRUST_UT;
  if (from == to) {
    double t[4] = {uin[0], uin[1], uin[2], uin[3]};
    if (from == VEL4 && !ut_known) {
      int e = ut_from_spatial_ucon(uin, g, t[0]);
      if (e) return e;
    }
    for (int i = 0; i < 4; ++i) uout[i] = t[i];
    return E_OK;
  }
  double o[4];
  if (from == VEL4) {
    double ut = uin[0];
    if (!ut_known) {
      int e = ut_from_spatial_ucon(uin, g, ut);
      if (e) return e;
    }
    if (to == VEL3) {
      o[0] = 1.0;
      o[1] = uin[1] / ut;
      o[2] = uin[2] / ut;
      o[3] = uin[3] / ut;
    } else {  // VELR
      o[0] = ut;
      for (int i = 1; i < 4; ++i) o[i] = uin[i] - ut * g.GG[0][i] / g.GG[0][0];
    }
  } else if (from == VEL3) {
    double ut = ut_from_vel3(uin, g);
    if (ut < 1.0 || kmath::isnan(ut)) return E_VELCONV;
    o[0] = ut;
    o[1] = uin[1] * ut;
    o[2] = uin[2] * ut;
    o[3] = uin[3] * ut;
    if (to == VELR) {
      for (int i = 1; i < 4; ++i) o[i] = o[i] - o[0] * g.GG[0][i] / g.GG[0][0];
    }
  } else {  // VELR
    if (to == VEL4) {
      velr_to_vel4(uin, g, o);
    } else {  // VEL3
      double alpgam = alpha_gamma(uin, g);
      o[0] = -alpgam * g.GG[0][0];
      o[1] = uin[1] / o[0] + g.GG[0][1] / g.GG[0][0];
      o[2] = uin[2] / o[0] + g.GG[0][2] / g.GG[0][0];
      o[3] = uin[3] / o[0] + g.GG[0][3] / g.GG[0][0];
    }
  }
  for (int i = 0; i < 4; ++i) uout[i] = o[i];
  return E_OK;
}

// Gas u^mu, u_mu from the VELR primitives (koral/relele.zig:356, infallible)
KC_HDM void ucon_ucov_from_prims(double v1, double v2, double v3, const Geom& g, double ucon[4], double ucov[4]) {
  double uin[4] = {0.0, v1, v2, v3};
  velr_to_vel4(uin, g, ucon);
  lower_vec(ucon, g, ucov);
}

// n^mu = -alpha g^{mu 0} (koral/relele.zig:376, C calc_normalobs_ncon)
KC_HD void normal_obs_con(const Geom& g, double ncon[4]) {
  for (int i = 0; i < 4; ++i) ncon[i] = -g.alpha * g.GG[i][0];
}
// koral/relele.zig:383 (C calc_normalobs_4vel)
KC_HD void normal_obs_4vel(const Geom& g, double out[4]) {
  double alp = 1.0 / kmath::sqrt(-g.GG[0][0]);
  double a[4] = {-alp, 0.0, 0.0, 0.0};
  raise_vec(a, g, out);
}
// koral/relele.zig:390 (C calc_normalobs_relvel)
KC_HD void normal_obs_velr(const Geom& g, double out[4]) {
  double ucon[4];
  normal_obs_4vel(g, ucon);
  out[0] = ucon[0];
  for (int i = 1; i < 4; ++i) out[i] = ucon[i] - ucon[0] * g.GG[0][i] / g.GG[0][0];
}

// ---- magnetic four-vector (koral/physics/bfield.zig) ------------------------
// b^mu from B^i and the gas four-velocity (bfield.zig:27, C calc_bcon_4vel)
KC_HD void bcon_from_4vel(const double B[3], const double ucon[4], const double ucov[4], double bcon[4]) {
  double b0 = B[0] * ucov[1] + B[1] * ucov[2] + B[2] * ucov[3];
  double inv_ut = 1.0 / ucon[0];
  bcon[0] = b0;
  for (int j = 1; j < 4; ++j) bcon[j] = (B[j - 1] + b0 * ucon[j]) * inv_ut;
}
// b^mu, b_mu, b^2 (bfield.zig:47, C calc_bcon_bcov_bsq_from_4vel)
KC_HDM void bcon_bcov_bsq(const double B[3], const double ucon[4], const double ucov[4], const Geom& g,
                         double bcon[4], double bcov[4], double& bsq) {
  bcon_from_4vel(B, ucon, ucov, bcon);
  lower_vec(bcon, g, bcov);
  bsq = dot(bcon, bcov);
}
// primitive B^i from b^mu (bfield.zig:60)
KC_HD void big_bcon_from_4vel(const double bcon[4], const double ucon[4], double Bcon[4]) {
  Bcon[0] = 0.0;
  for (int j = 1; j < 4; ++j) Bcon[j] = bcon[j] * ucon[0] - bcon[0] * ucon[j];
}

// ---- gas thermodynamics (koral/physics/hydro.zig) ---------------------------
// S(rho, u) (hydro.zig:31, C calc_Sfromu, log form)
KC_HDM double s_from_u(double rho, double u, double gam) {
  double gammam1 = gam - 1.0;
  double indexn = 1.0 / gammam1;
  double pre = gammam1 * u;
  return rho * kmath::log(kmath::pow(pre, indexn) / kmath::pow(rho, indexn + 1.0));
}
// inverse of s_from_u (hydro.zig:43, C calc_ufromS)
KC_HDM double u_from_s(double s, double rho, double gam) {
  double gammam1 = gam - 1.0;
  double indexn = 1.0 / gammam1;
  return kmath::pow(kmath::pow(rho, indexn + 1.0) * kmath::exp(s / rho), gammam1) / gammam1;
}

// T^mu nu with u and b already in hand (hydro.zig:87, C calc_Tij)
KC_HD void tij_from_state(const double pp[NV], const Geom& g, double gam, const double ucon[4], const double bcon[4],
                          double bsq, double t[4][4]) {
  double rho = pp[RHO], uu = pp[UU];
  double p = (gam - 1.0) * uu;
  double w = rho + uu + p;
  double eta = w + bsq;
  double ptot = p + 0.5 * bsq;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) t[i][j] = eta * ucon[i] * ucon[j] + ptot * g.GG[i][j] - bcon[i] * bcon[j];
}
// hydro.zig:53
KC_HDM void calc_tij(const double pp[NV], const Geom& g, double gam, double t[4][4]) {
  double ucon[4], ucov[4], bcon[4], bcov[4], bsq;
  ucon_ucov_from_prims(pp[VX], pp[VY], pp[VZ], g, ucon, ucov);
  double B[3] = {pp[B1], pp[B2], pp[B3]};
  bcon_bcov_bsq(B, ucon, ucov, g, bcon, bcov, bsq);
  tij_from_state(pp, g, gam, ucon, bcon, bsq, t);
}

// ---- p2u (koral/p2u.zig) ----------------------------------------------------
// 1 + u_t without cancellation (p2u.zig:17, C calc_utp1, VELR branch)
KC_HD double calc_utp1(const double vcon[4], const Geom& g) {
  double qsq = 0.0;
  for (int i = 1; i < 4; ++i)
    for (int j = 1; j < 4; ++j) qsq += vcon[i] * vcon[j] * g.gg[i][j];
  double alpha = g.alpha;
  double alphasq = alpha * alpha;
  double alpgam = kmath::sqrt(alphasq * (1.0 + qsq));
  double betasqoalphasq = g.gg[0][1] * g.GG[0][1] + g.gg[0][2] * g.GG[0][2] + g.gg[0][3] * g.GG[0][3];
  double ud0tilde = 0.0;
  for (int j = 1; j < 4; ++j) ud0tilde += vcon[j] * g.gg[0][j];
  return ud0tilde + (g.gttpert - alphasq * (betasqoalphasq + qsq)) / (1.0 + alpgam);
}

// hydro + magnetic conserveds (p2u.zig:39, C p2u_mhd)
KC_HDM void p2u_mhd(const double pp[NV], double uu[NV], const Geom& g, double gam) {
  double gdetu = g.gdet;
  double rho = pp[RHO], ugas = pp[UU], s = pp[ENTR];
  double vcon[4] = {0.0, pp[VX], pp[VY], pp[VZ]};
  double ucon[4], ucov[4];
  velr_to_vel4(vcon, g, ucon);
  lower_vec(ucon, g, ucov);
  double B[3] = {pp[B1], pp[B2], pp[B3]};
  double bcon[4], bcov[4], bsq;
  bcon_bcov_bsq(B, ucon, ucov, g, bcon, bcov, bsq);
  double ut = ucon[0];
  double rhout = rho * ut;
  double sut = s * ut;
  double pre = (gam - 1.0) * ugas;
  double w = rho + ugas + pre;
  double eta = w + bsq;
  double etap = ugas + pre + bsq;
  double ptot = pre + 0.5 * bsq;
  double utp1 = calc_utp1(vcon, g);
  double tttt = etap * ucon[0] * ucov[0] + rho * ucon[0] * utp1 + ptot - bcon[0] * bcov[0];
  double ttr = eta * ucon[0] * ucov[1] - bcon[0] * bcov[1];
  double ttth = eta * ucon[0] * ucov[2] - bcon[0] * bcov[2];
  double ttph = eta * ucon[0] * ucov[3] - bcon[0] * bcov[3];
  uu[RHO] = gdetu * rhout;
  uu[UU] = gdetu * tttt;
  uu[VX] = gdetu * ttr;
  uu[VY] = gdetu * ttth;
  uu[VZ] = gdetu * ttph;
  uu[ENTR] = gdetu * sut;
  uu[B1] = gdetu * pp[B1];
  uu[B2] = gdetu * pp[B2];
  uu[B3] = gdetu * pp[B3];
}

// M1 radiative conserveds R^t_mu (p2u.zig:103, C p2u_rad)
KC_HDM void p2u_rad(const double pp[NV], double uu[NV], const Geom& g) {
  double gdetu = g.gdet;
  const double four_third = 4.0 / 3.0, one_third = 1.0 / 3.0;
  double erf = pp[EE];
  double vin[4] = {0.0, pp[FX], pp[FY], pp[FZ]};
  double urf[4];
  velr_to_vel4(vin, g, urf);
  double rtopp[4];
  for (int i = 0; i < 4; ++i) rtopp[i] = four_third * erf * urf[0] * urf[i] + one_third * erf * g.GG[0][i];
  lower_vec(rtopp, g, rtopp);
  for (int i = 0; i < 4; ++i) uu[EE + i] = gdetu * rtopp[i];
}

// full conserved vector (p2u.zig:135, C p2u)
KC_HDM void p2u(const double pp[NV], double uu[NV], const Geom& g, double gam) {
  p2u_mhd(pp, uu, g, gam);
  p2u_rad(pp, uu, g);
}

}  // namespace kp
