// kinvert.h — conserved -> primitive inversion (MHD Noble W-Newton and the
// closed-form M1 inversion), the MHD and radiation floors, the M1 tensor and
// the characteristic speeds. Shared host/device restatement of
// koral/solve/invert.zig, koral/solve/invert_rad.zig,
// koral/physics/radiation.zig and koral/physics/wavespeeds.zig.
#pragma once
#include "kcore.h"

namespace kp {

// Floor thresholds (koral/solve/invert.zig:60, FloorParams.puffy at :81).
struct FloorParams {
  double rhofloor, uurhoratiomin, uurhoratiomax, b2rhoratiomax, b2uuratiomax, gammamaxhd;
  int isentropic_b2rhofloors;
  int b2uufloor;
  double horizon_x1;
};
// Radiation caps (koral/solve/invert_rad.zig:36, RadParams.puffy at :47).
struct RadParams {
  double gammamaxrad, eradfloor, eerhoratiomin, eerhoratiomax, eeuuratiomin, eeuuratiomax;
};

// ---- MHD u2p (koral/solve/invert.zig) --------------------------------------
struct U2pRes {
  double f, df, err;
};
KC_HD void w_kinematics(double W, double Wp, double D, double Qtsq, double QdotBsq, double Bsq, double& v2,
                        double& gamma, double& gamma2, double& rho0, double& wmrho0) {
  double x = Bsq + W;
  double wsq = W * W;
  v2 = (wsq * Qtsq + QdotBsq * (Bsq + 2.0 * W)) / (wsq * (x * x));
  gamma2 = 1.0 / (1.0 - v2);
  gamma = kmath::sqrt(gamma2);
  rho0 = D / gamma;
  wmrho0 = Wp / gamma2 - D * v2 / (1.0 + gamma);
}
// invert.zig:121 (C f_u2p_hot, Noble)
KC_HD U2pRes f_u2p_hot(double Wp, const double cons[7], double pgamma) {
  double Qn = cons[0], Qtsq = cons[1], D = cons[2], QdotBsq = cons[3], Bsq = cons[4];
  double W = Wp + D;
  double x = Bsq + W;
  double wsq = W * W;
  double w3 = wsq * W;
  double x3 = x * x * x;
  double v2, gamma, gamma2, rho0, wmrho0;
  w_kinematics(W, Wp, D, Qtsq, QdotBsq, Bsq, v2, gamma, gamma2, rho0, wmrho0);
  double u = wmrho0 / pgamma;
  double p = (pgamma - 1.0) * u;
  U2pRes r;
  r.f = Qn + W - p + 0.5 * Bsq * (1.0 + v2) - QdotBsq / 2.0 / wsq;
  r.err = kmath::fabs(r.f) / (kmath::fabs(Qn) + kmath::fabs(W) + kmath::fabs(p) + kmath::fabs(0.5 * Bsq * (1.0 + v2)) +
                              kmath::fabs(QdotBsq / 2.0 / wsq));
  double dvsq = -2.0 / x3 * (Qtsq + QdotBsq * (3.0 * W * x + Bsq * Bsq) / w3);
  double dp1 = (pgamma - 1.0) * (1.0 - v2) / pgamma;
  double idwmrho0dp = (pgamma - 1.0) / pgamma;
  double dwmrho0dvsq = D * (gamma * 0.5 - 1.0) - Wp;
  double dp2 = dwmrho0dvsq * idwmrho0dp;
  double dpdW = dp1 + dp2 * dvsq;
  r.df = 1.0 - dpdW + QdotBsq / (wsq * W) + 0.5 * Bsq * dvsq;
  return r;
}
// invert.zig:170 (C f_u2p_entropy)
KC_HD U2pRes f_u2p_entropy(double Wp, const double cons[7], double pgamma) {
  double Qtsq = cons[1], D = cons[2], QdotBsq = cons[3], Bsq = cons[4], Sc = cons[5];
  double W = Wp + D;
  double x = Bsq + W;
  double wsq = W * W;
  double w3 = wsq * W;
  double x3 = x * x * x;
  double v2, gamma, gamma2, rho0, wmrho0;
  w_kinematics(W, Wp, D, Qtsq, QdotBsq, Bsq, v2, gamma, gamma2, rho0, wmrho0);
  double pressure = (pgamma - 1.0) / pgamma * wmrho0;
  double indexn = 1.0 / (pgamma - 1.0);
  double ssofchi = kmath::log(kmath::pow(pressure, indexn) / kmath::pow(rho0, indexn + 1.0));
  U2pRes r;
  r.f = -Sc + D * ssofchi;
  r.err = kmath::fabs(r.f) / (kmath::fabs(Sc) + kmath::fabs(D * ssofchi));
  double dssdrho = pgamma / ((1.0 - pgamma) * rho0);
  double dssdchi = 1.0 / ((pgamma - 1.0) * wmrho0);
  double dwmrho0dw = 1.0 / (gamma * gamma);
  double dwmrho0dvsq = D * (gamma * 0.5 - 1.0) - Wp;
  double drho0dvsq = -D * gamma * 0.5;
  double dvsq = -2.0 / x3 * (Qtsq + QdotBsq * (3.0 * W * x + Bsq * Bsq) / w3);
  double dssdw = dwmrho0dw * dssdchi;
  double dssdvsq = drho0dvsq * dssdrho + dwmrho0dvsq * dssdchi;
  double dssdwp = dssdw + dssdvsq * dvsq;
  r.df = D * dssdwp;
  return r;
}
enum : int { ETYPE_HOT = 0, ETYPE_ENTROPY = 1 };
KC_HD U2pRes u2p_residual(int etype, double Wp, const double cons[7], double pgamma) {
  return etype == ETYPE_HOT ? f_u2p_hot(Wp, cons, pgamma) : f_u2p_entropy(Wp, cons, pgamma);
}
// invert.zig:224
KC_HD bool w_out_of_bounds(double W, double Qtsq, double QdotBsq, double Bsq, const U2pRes& res) {
  return (W * W * W * (W + 2.0 * Bsq) - QdotBsq * (2.0 * W + Bsq)) <= W * W * (Qtsq - Bsq * Bsq) ||
         !kmath::isfinite(res.f) || !kmath::isfinite(res.df);
}

// C u2p_solver_W (invert.zig:240). pp is in/out (the Newton seed).
// (the body, inlined by kernels that keep its arrays in registers)
KC_HD int u2p_solver_w_inl(const double uu[NV], double pp[NV], const Geom& g, int etype, double pgamma) {
  const double conv = 1.0e-10;
  const double big = 1.0 / 1.0e-80;
  double gdetu_inv = 1.0 / g.gdet;
  double alpha = g.alpha;
  double D = uu[RHO] * gdetu_inv * alpha;
  double Sc = uu[ENTR] * gdetu_inv * alpha;
  double Qcov[4] = {(uu[UU] * gdetu_inv - uu[RHO] * gdetu_inv) * alpha, uu[VX] * gdetu_inv * alpha,
                    uu[VY] * gdetu_inv * alpha, uu[VZ] * gdetu_inv * alpha};
  double Qcon[4];
  raise_vec(Qcov, g, Qcon);
  double Bcon[4] = {0.0, uu[B1] * gdetu_inv * alpha, uu[B2] * gdetu_inv * alpha, uu[B3] * gdetu_inv * alpha};
  double Bcov[4];
  lower_vec(Bcon, g, Bcov);
  double Bsq = dot(Bcon, Bcov);
  double QdotB = dot(Qcov, Bcon);
  double QdotBsq = QdotB * QdotB;
  double ncov[4] = {-alpha, 0.0, 0.0, 0.0};
  double ncon[4];
  raise_vec(ncov, g, ncon);
  double Qn = Qcon[0] * ncov[0];
  double Qtcon[4];
  for (int i = 0; i < 4; ++i) {
    Qtcon[i] = 0.0;
    for (int j = 0; j < 4; ++j) Qtcon[i] += (kron(i, j) + ncon[i] * ncov[j]) * Qcon[j];
  }
  double Qtcov[4];
  lower_vec(Qtcon, g, Qtcov);
  double Qt2 = dot(Qtcon, Qtcov);
  double Qtsq = Qt2;

  double rho = pp[RHO];
  double uint_ = pp[UU];
  double utcon0[4] = {0.0, pp[VX], pp[VY], pp[VZ]};
  double qsq = 0.0;
  for (int i = 1; i < 4; ++i)
    for (int j = 1; j < 4; ++j) qsq += utcon0[i] * utcon0[j] * g.gg[i][j];
  double gamma2 = 1.0 + qsq;
  double W = (rho + pgamma * uint_) * gamma2;
  double cons[7] = {Qn, Qt2, D, QdotBsq, Bsq, Sc, 0.0};

  int i_increase = 0;
  while (true) {
    U2pRes res = u2p_residual(etype, W - D, cons, pgamma);
    if (w_out_of_bounds(W, Qtsq, QdotBsq, Bsq, res) && i_increase < 50) {
      W *= 10.0;
      i_increase += 1;
      continue;
    }
    break;
  }
  if (i_increase >= 50) return -150;

  int iter = 0;
  while (iter < 50) {
    double Wprev = W;
    iter += 1;
    U2pRes res = u2p_residual(etype, W - D, cons, pgamma);
    double f0 = res.f, dfdW = res.df, errr = res.err;
    if (errr < conv) break;
    if (dfdW == 0.0) {
      W *= 1.1;
      continue;
    }
    double Wnew = W - f0 / dfdW;
    int idump = 0;
    double dumpfac = 1.0;
    while (true) {
      U2pRes rtmp = u2p_residual(etype, Wnew - D, cons, pgamma);
      if (w_out_of_bounds(Wnew, Qtsq, QdotBsq, Bsq, rtmp) && idump < 100) {
        idump += 1;
        dumpfac /= 2.0;
        Wnew = W - dumpfac * f0 / dfdW;
        continue;
      }
      break;
    }
    if (idump >= 100) return -101;
    W = Wnew;
    if (kmath::fabs(W) > big) return -103;
    if (kmath::fabs((W - Wprev) / Wprev) < conv && errr < 1.0e-1) break;
  }
  if (iter >= 50) return -102;
  if (!kmath::isfinite(W)) return -103;

  double wsq = W * W;
  double xsq = (Bsq + W) * (Bsq + W);
  double v2 = (wsq * Qtsq + QdotBsq * (Bsq + 2.0 * W)) / (wsq * xsq);
  gamma2 = 1.0 / (1.0 - v2);
  double gamma = kmath::sqrt(gamma2);
  rho = D / gamma;
  double entr = Sc / gamma;
  uint_ = 1.0 / pgamma * (W / gamma2 - rho);
  double utcon[4];
  utcon[0] = 0.0;
  for (int i = 1; i < 4; ++i) utcon[i] = gamma / (W + Bsq) * (Qtcon[i] + QdotB * Bcon[i] / W);
  if (!kmath::isfinite(utcon[1])) return -120;
  if (uint_ < 0.0 || gamma2 < 0.0 || kmath::isnan(W) || !kmath::isfinite(W)) return -104;
  pp[RHO] = rho;
  pp[UU] = uint_;
  pp[VX] = utcon[1];
  pp[VY] = utcon[2];
  pp[VZ] = utcon[3];
  if (rho < 0.0) return -105;
  pp[ENTR] = entr;
  pp[B1] = uu[B1] * gdetu_inv;
  pp[B2] = uu[B2] * gdetu_inv;
  pp[B3] = uu[B3] * gdetu_inv;
  return 0;
}
KC_HDN int u2p_solver_w(const double uu[NV], double pp[NV], const Geom& g, int etype, double pgamma) {
  return u2p_solver_w_inl(uu, pp, g, etype, pgamma);
}

struct U2pMhdRes {
  int ret;
  bool entropy_used;
  bool fixup;
};
// MHD part of C's u2p cascade (invert.zig:422)
// INL: both W solves (hot energy, entropy fallback) inlined, so the kernel keeps
// the conserved and primitive arrays in registers instead of a call frame
template <bool INL>
KC_HDM U2pMhdRes u2p_mhd_t(const double uu_in[NV], double pp[NV], const Geom& g, double pgamma, const FloorParams& fl) {
  double uu[NV], ppbak[NV], ppmhd[NV];
  for (int i = 0; i < NV; ++i) {
    uu[i] = uu_in[i];
    ppbak[i] = pp[i];
    ppmhd[i] = pp[i];
  }
  double gdetu = g.gdet;
  int ret = 0;
  bool entropy_used = false;
  if (uu[RHO] * g.alpha / gdetu < 0.0) {
    ppmhd[RHO] = fl.rhofloor;
    uu[RHO] = fl.rhofloor * gdetu / g.alpha;
    ret = -2;
  }
  int u2pret = INL ? u2p_solver_w_inl(uu, ppmhd, g, ETYPE_HOT, pgamma) : u2p_solver_w(uu, ppmhd, g, ETYPE_HOT, pgamma);
  if (u2pret < 0) {
    ret = -1;
    entropy_used = true;
    u2pret = INL ? u2p_solver_w_inl(uu, ppmhd, g, ETYPE_ENTROPY, pgamma) : u2p_solver_w(uu, ppmhd, g, ETYPE_ENTROPY, pgamma);
    if (u2pret < 0) ret = -2;
  }
  if (u2pret >= 0) {
    for (int i = 0; i < NV; ++i) pp[i] = ppmhd[i];
  } else {
    for (int i = 0; i < NV; ++i) pp[i] = ppbak[i];
    ret = -3;
  }
  U2pMhdRes r;
  r.ret = ret;
  r.entropy_used = entropy_used;
  r.fixup = ret < -1;
  return r;
}
KC_HDM U2pMhdRes u2p_mhd(const double uu_in[NV], double pp[NV], const Geom& g, double pgamma, const FloorParams& fl) {
  return u2p_mhd_t<false>(uu_in, pp, g, pgamma, fl);
}

// C check_floors_mhd, DRIFTFRAME (invert.zig:474). Returns -1 if floored.
// guard_count is incremented when a drift-frame guard diverted the algebra
// (the reference's n_guard_recoveries, invert.zig:44).
// (the body, inlined by kernels that keep its arrays in registers)
KC_HD int check_floors_mhd_inl(double pp[NV], const Geom& g, double pgamma, const FloorParams& fl, int& guard_count) {
  int ret = 0;
  if (pp[RHO] < fl.rhofloor) {
    pp[RHO] = fl.rhofloor;
    ret = -1;
  }
  if (pp[UU] < fl.uurhoratiomin * pp[RHO]) {
    pp[UU] = fl.uurhoratiomin * pp[RHO];
    ret = -1;
  }
  if (pp[UU] > fl.uurhoratiomax * pp[RHO]) {
    pp[UU] = fl.uurhoratiomax * pp[RHO];
    ret = -1;
  }
  {
    double ucon[4], ucov[4];
    ucon_ucov_from_prims(pp[VX], pp[VY], pp[VZ], g, ucon, ucov);
    double B[3] = {pp[B1], pp[B2], pp[B3]};
    double bcon[4], bcov[4], bsq;
    bcon_bcov_bsq(B, ucon, ucov, g, bcon, bcov, bsq);
    double f = 1.0, fuu = 1.0;
    bool floored = false;
    if (bsq > fl.b2rhoratiomax * pp[RHO]) {
      f = bsq / (fl.b2rhoratiomax * pp[RHO]);
      floored = true;
    }
    if (fl.b2uufloor && bsq > fl.b2uuratiomax * pp[UU]) {
      fuu = bsq / (fl.b2uuratiomax * pp[UU]);
      floored = true;
    }
    if (floored) {
      double wold = pp[RHO] + pp[UU] * pgamma;
      pp[RHO] *= f;
      pp[UU] *= fl.isentropic_b2rhofloors ? f : fuu;
      double wnew = pp[RHO] + pp[UU] * pgamma;
      bool guarded = false;
      if (g.xx[1] >= fl.horizon_x1) {
        do {
          double Bcon[4] = {0.0, pp[B1], pp[B2], pp[B3]};
          double Bcov[4];
          lower_vec(Bcon, g, Bcov);
          double Bsq = dot(Bcon, Bcov);
          double Bmag = kmath::sqrt(Bsq);
          if (!(bsq > 1.0e-10 * wnew && Bsq > 1.0e-10 * wnew)) {
            guarded = true;
            break;
          }
          double betapar = -bcon[0] / (bsq * ucon[0]);
          double betasq = betapar * betapar * bsq;
          double betasqmax = 1.0 - 1.0 / (fl.gammamaxhd * fl.gammamaxhd);
          if (betasq > betasqmax) betasq = betasqmax;
          double gammapar = 1.0 / kmath::sqrt(1.0 - betasq);
          double ucondr[4];
          for (int iv = 0; iv < 4; ++iv) ucondr[iv] = gammapar * (ucon[iv] + betapar * bcon[iv]);
          if (!kmath::isfinite(ucondr[0]) || kmath::fabs(ucondr[0]) < 1.0e-10) {
            guarded = true;
            break;
          }
          double udotB = dot(ucon, Bcov);
          double QdotB = udotB * wold * ucon[0];
          double xx = 2.0 * QdotB / (Bmag * wnew * ucondr[0]);
          if (!(xx <= 1.0e10)) {
            xx = 1.0e10;
            guarded = true;
          }
          if (!(xx >= -1.0e10)) {
            xx = -1.0e10;
            guarded = true;
          }
          double vpar = xx / (ucondr[0] * (1.0 + kmath::sqrt(1.0 + xx * xx)));
          double vcon[4];
          vcon[0] = 1.0;
          for (int iv = 1; iv < 4; ++iv) vcon[iv] = vpar * Bcon[iv] / Bmag + ucondr[iv] / ucondr[0];
          for (int idamp = 0; idamp < 50; ++idamp) {
            double bv = 0.0, cv = 0.0;
            for (int iv = 1; iv < 4; ++iv) {
              bv += vcon[iv] * g.gg[0][iv];
              for (int jv = 1; jv < 4; ++jv) cv += vcon[iv] * vcon[jv] * g.gg[iv][jv];
            }
            if (g.gg[0][0] + 2.0 * bv + cv < -1.0 / (fl.gammamaxhd * fl.gammamaxhd)) break;
            guarded = true;
            vpar *= 0.5;
            for (int iv = 1; iv < 4; ++iv) vcon[iv] = vpar * Bcon[iv] / Bmag + ucondr[iv] / ucondr[0];
          }
          double ucont[4];
          if (convert(vcon, VEL3, VELR, g, RECOMPUTE_UT, ucont) != E_OK) {
            guarded = true;
            break;
          }
          pp[VX] = ucont[1];
          pp[VY] = ucont[2];
          pp[VZ] = ucont[3];
        } while (false);
      }
      if (guarded) guard_count += 1;
      ret = -1;
    }
  }
  {
    double qsq = 0.0;
    for (int i = 1; i < 4; ++i)
      for (int j = 1; j < 4; ++j) qsq += pp[VX - 1 + i] * pp[VX - 1 + j] * g.gg[i][j];
    double gamma2 = 1.0 + qsq;
    if (gamma2 > fl.gammamaxhd * fl.gammamaxhd) {
      double qsqmax = fl.gammamaxhd * fl.gammamaxhd - 1.0;
      double a = kmath::sqrt(qsqmax / qsq);
      for (int j = 1; j < 4; ++j) pp[VX - 1 + j] *= a;
      ret = -1;
    }
  }
  if (ret < 0) pp[ENTR] = s_from_u(pp[RHO], pp[UU], pgamma);
  return ret;
}
KC_HDN int check_floors_mhd(double pp[NV], const Geom& g, double pgamma, const FloorParams& fl, int& guard_count) { return check_floors_mhd_inl(pp, g, pgamma, fl, guard_count); }

// ---- M1 radiation (koral/physics/radiation.zig) ----------------------------
// R^mu nu of the M1 closure (radiation.zig:79, C calc_Rij_M1)
KC_HDM void calc_rij(const double pp[NV], const Geom& g, double rij[4][4]) {
  const double four_third = 4.0 / 3.0, one_third = 1.0 / 3.0;
  double erf = pp[EE];
  double vin[4] = {0.0, pp[FX], pp[FY], pp[FZ]};
  double urf[4];
  velr_to_vel4(vin, g, urf);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) rij[i][j] = four_third * erf * urf[i] * urf[j] + one_third * erf * g.GG[i][j];
}
// C calc_ff_Rtt (radiation.zig:104): rtt = -R^mu_nu u^nu u_mu; also gas ucon
KC_HDM double calc_ff_rtt(const double pp[NV], const Geom& g, double ucon_out[4]) {
  double ucon[4], ucov[4];
  ucon_ucov_from_prims(pp[VX], pp[VY], pp[VZ], g, ucon, ucov);
  double rij_uu[4][4], rij_ud[4][4];
  calc_rij(pp, g, rij_uu);
  lower_second(rij_uu, g, rij_ud);
  double rtt = 0.0;
  for (int ia = 0; ia < 4; ++ia)
    for (int ib = 0; ib < 4; ++ib) rtt += -rij_ud[ia][ib] * ucon[ib] * ucov[ia];
  if (ucon_out)
    for (int i = 0; i < 4; ++i) ucon_out[i] = ucon[i];
  return rtt;
}

// ---- M1 inversion (koral/solve/invert_rad.zig) -----------------------------
// C get_m1closure_gammarel2 (invert_rad.zig:66)
KC_HDM double m1_gammarel2(const Geom& g, const double av[4]) {
  const double gsl = 1.0 - 1e-10;
  double gn11 = g.GG[0][0], gn12 = g.GG[0][1], gn13 = g.GG[0][2], gn14 = g.GG[0][3];
  double gn22 = g.GG[1][1], gn23 = g.GG[1][2], gn24 = g.GG[1][3];
  double gn33 = g.GG[2][2], gn34 = g.GG[2][3], gn44 = g.GG[3][3];
  double rdtt = av[0], rdtx = av[1], rdty = av[2], rdtz = av[3];
  double mix = gn12 * rdtx + gn13 * rdty + gn14 * rdtz;
  double sq = kmath::sqrt(4.0 * (gn11 * gn11) * (rdtt * rdtt) + mix * mix +
                          gn11 * (8.0 * gn12 * rdtt * rdtx + 3.0 * gn22 * (rdtx * rdtx) + 8.0 * gn13 * rdtt * rdty +
                                  6.0 * gn23 * rdtx * rdty + 3.0 * gn33 * (rdty * rdty) + 8.0 * gn14 * rdtt * rdtz +
                                  6.0 * gn24 * rdtx * rdtz + 6.0 * gn34 * rdty * rdtz + 3.0 * gn44 * (rdtz * rdtz)));
  double den = gn11 * (rdtt * rdtt) + 2.0 * gn12 * rdtt * rdtx + gn22 * (rdtx * rdtx) + 2.0 * gn13 * rdtt * rdty +
               2.0 * gn23 * rdtx * rdty + gn33 * (rdty * rdty) + 2.0 * (gn14 * rdtt + gn24 * rdtx + gn34 * rdty) * rdtz +
               gn44 * (rdtz * rdtz);
  double gamma2a = kmath::div((-0.25 * (2.0 * (gn11 * gn11) * (rdtt * rdtt) + mix * (mix + sq) +
                             gn11 * (4.0 * gn12 * rdtt * rdtx + gn22 * (rdtx * rdtx) + 2.0 * gn23 * rdtx * rdty +
                                     gn33 * (rdty * rdty) + 2.0 * gn24 * rdtx * rdtz + 2.0 * gn34 * rdty * rdtz +
                                     gn44 * (rdtz * rdtz) + rdtt * (4.0 * gn13 * rdty + 4.0 * gn14 * rdtz + sq)))), den);
  double gamma2;
  if (gamma2a < gsl || !kmath::isfinite(gamma2a)) {
    double gamma2b = kmath::div((0.25 * (-2.0 * (gn11 * gn11) * (rdtt * rdtt) -
                              1.0 * gn11 *
                                  (4.0 * gn12 * rdtt * rdtx + gn22 * (rdtx * rdtx) +
                                   rdty * (4.0 * gn13 * rdtt + 2.0 * gn23 * rdtx + gn33 * rdty) +
                                   2.0 * (2.0 * gn14 * rdtt + gn24 * rdtx + gn34 * rdty) * rdtz + gn44 * (rdtz * rdtz)) +
                              gn11 * rdtt * sq + mix * (-1.0 * gn12 * rdtx - 1.0 * gn13 * rdty - 1.0 * gn14 * rdtz + sq))), den);
    gamma2 = gamma2b;
  } else {
    gamma2 = gamma2a;
  }
  double alpha = g.alpha;
  double gammarel2 = gamma2 * alpha * alpha;
  if (gammarel2 > gsl && gammarel2 < 1.0) gammarel2 = 1.0;
  return gammarel2;
}
// C get_m1closure_gammarel2_cold (invert_rad.zig:136)
KC_HDM void m1_cold(const Geom& g, const double av_in[4], double gammarel2, double av[4], double& erf, double urfconrel[4]) {
  double gn11 = g.GG[0][0], gn12 = g.GG[0][1], gn13 = g.GG[0][2], gn14 = g.GG[0][3];
  double gn22 = g.GG[1][1], gn23 = g.GG[1][2], gn24 = g.GG[1][3];
  double gn33 = g.GG[2][2], gn34 = g.GG[2][3], gn44 = g.GG[3][3];
  double alpha = g.alpha;
  double rdtx = av_in[1], rdty = av_in[2], rdtz = av_in[3];
  double utsq = kmath::div(gammarel2, (alpha * alpha));
  for (int i = 0; i < 4; ++i) av[i] = av_in[i];
  double mix = gn13 * rdty + gn14 * rdtz;
  double disc = kmath::sqrt(((gn12 * gn12) * (rdtx * rdtx) + 2.0 * gn12 * rdtx * mix + mix * mix -
                             1.0 * gn11 *
                                 (gn22 * (rdtx * rdtx) + 2.0 * gn23 * rdtx * rdty + gn33 * (rdty * rdty) +
                                  2.0 * gn24 * rdtx * rdtz + 2.0 * gn34 * rdty * rdtz + gn44 * (rdtz * rdtz))) *
                            utsq * (gn11 + utsq) * ((gn11 + 4.0 * utsq) * (gn11 + 4.0 * utsq)));
  av[0] = kmath::div((0.25 * (-4.0 * (gn12 * rdtx + gn13 * rdty + gn14 * rdtz) * utsq * (gn11 + utsq) + disc)), (gn11 * utsq * (gn11 + utsq)));
  erf = kmath::div((0.75 * disc), (utsq * (gn11 + utsq) * (gn11 + 4.0 * utsq)));
  double avcon[4];
  raise_vec(av, g, avcon);
  double gammarel = kmath::sqrt(gammarel2);
  for (int i = 0; i < 4; ++i) urfconrel[i] = 0.0;
  if (erf > 0.0) {
    for (int jj = 1; jj < 4; ++jj)
      urfconrel[jj] = kmath::div(alpha * (avcon[jj] + 1.0 / 3.0 * erf * g.GG[0][jj] * (4.0 * gammarel2 - 1.0)), (4.0 / 3.0 * erf * gammarel));
  }
}

struct U2pRadRes {
  int ret;
  bool corrected;
};
// C u2p_rad (invert_rad.zig:189). Writes pp[EE..FZ] on success.
// (the body, inlined by kernels that keep its arrays in registers)
KC_HD U2pRadRes u2p_rad_inl(const double uu[NV], double pp[NV], const Geom& g, const RadParams& rp) {
  const double gsl = 1.0 - 1e-10;
  const double numepsilon = 2.220446049250313e-16;
  double gdetu = g.gdet;
  double alpha = g.alpha;
  double avcov[4] = {kmath::div(uu[EE], gdetu), kmath::div(uu[FX], gdetu), kmath::div(uu[FY], gdetu), kmath::div(uu[FZ], gdetu)};
  double avcon[4];
  raise_vec(avcov, g, avcon);
  double gammarel2 = m1_gammarel2(g, avcov);
  double erf = kmath::div(3.0 * avcon[0] * alpha * alpha, (4.0 * gammarel2 - 1.0));
  double gammamax = rp.gammamaxrad;
  bool nonfailure = gammarel2 >= 1.0 && erf > rp.eradfloor && gammarel2 <= kmath::div(kmath::div(gammamax * gammamax, gsl), gsl);
  double urfcon[4];
  bool corrected = false;
  U2pRadRes res;
  if (nonfailure) {
    double gammarel = kmath::sqrt(gammarel2);
    for (int ii = 0; ii < 4; ++ii)
      urfcon[ii] = kmath::div(alpha * (avcon[ii] + 1.0 / 3.0 * erf * g.GG[0][ii] * (4.0 * gammarel2 - 1.0)), (4.0 / 3.0 * erf * gammarel));
  } else {
    double one_eps = 1.0 + 10.0 * numepsilon;
    double s_av[4], s_erf, s_urf[4], f_av[4], f_erf, f_urf[4];
    m1_cold(g, avcov, one_eps * one_eps, s_av, s_erf, s_urf);
    m1_cold(g, avcov, gammamax * gammamax, f_av, f_erf, f_urf);
    if (kmath::fabs(s_av[0] - avcov[0]) > kmath::fabs(f_av[0] - avcov[0])) {
      raise_vec(f_av, g, avcon);
      for (int i = 0; i < 4; ++i) urfcon[i] = f_urf[i];
      gammarel2 = gammamax * gammamax;
      erf = f_erf;
    } else {
      raise_vec(s_av, g, avcon);
      for (int i = 0; i < 4; ++i) urfcon[i] = s_urf[i];
      gammarel2 = one_eps * one_eps;
      erf = s_erf;
    }
    corrected = true;
    if (!kmath::isfinite(erf) || !kmath::isfinite(gammarel2) || !kmath::isfinite(urfcon[1]) ||
        !kmath::isfinite(urfcon[2]) || !kmath::isfinite(urfcon[3])) {
      res.ret = -1;
      res.corrected = corrected;
      return res;
    }
  }
  pp[EE] = erf;
  pp[FX] = urfcon[1];
  pp[FY] = urfcon[2];
  pp[FZ] = urfcon[3];
  res.ret = 0;
  res.corrected = corrected;
  return res;
}
KC_HDN U2pRadRes u2p_rad(const double uu[NV], double pp[NV], const Geom& g, const RadParams& rp) { return u2p_rad_inl(uu, pp, g, rp); }

// C check_floors_rad (invert_rad.zig:266)
KC_HDM int check_floors_rad(double pp[NV], const Geom& g, const RadParams& rp) {
  int ret = 0;
  double ehat = -calc_ff_rtt(pp, g, nullptr);
  double eratio = kmath::div(pp[EE], ehat);
  if (pp[EE] < rp.eradfloor) {
    pp[EE] = rp.eradfloor;
    ret = -1;
  }
  if (ehat < rp.eerhoratiomin * pp[RHO]) {
    pp[EE] = eratio * rp.eerhoratiomin * pp[RHO];
    ret = -1;
  }
  if (ehat > rp.eerhoratiomax * pp[RHO]) {
    pp[RHO] = kmath::div(1.0, rp.eerhoratiomax) * ehat;
    ret = -1;
  }
  if (ehat < rp.eeuuratiomin * pp[UU]) {
    pp[EE] = eratio * rp.eeuuratiomin * pp[UU];
    ret = -1;
  }
  if (ehat > rp.eeuuratiomax * pp[UU]) {
    pp[UU] = kmath::div(1.0, rp.eeuuratiomax) * ehat;
    ret = -1;
  }
  return ret;
}

// ---- characteristic speeds (koral/physics/wavespeeds.zig) ------------------
// C calc_wavespeeds_lr_core (wavespeeds.zig:32)
KC_HD void lr_core(const double ucon[4], const Geom& g, const double ws2[3], const bool active[3], double aret[6]) {
  for (int i = 0; i < 6; ++i) aret[i] = 0.0;
  double Bcov[4] = {1.0, 0.0, 0.0, 0.0};
  double Bcon[4];
  raise_vec(Bcov, g, Bcon);
  double Bsq = dot(Bcon, Bcov);
  double Bu = dot(Bcov, ucon);
  double Bu2 = Bu * Bu;
  for (int dim = 0; dim < 3; ++dim) {
    if (!active[dim]) continue;
    double wspeed2 = ws2[dim];
    double Acov[4] = {0.0, 0.0, 0.0, 0.0};
    Acov[dim + 1] = 1.0;
    double Acon[4];
    raise_vec(Acov, g, Acon);
    double Asq = dot(Acon, Acov);
    double Au = dot(Acov, ucon);
    double AB = dot(Acon, Bcov);
    double Au2 = Au * Au;
    double AuBu = Au * Bu;
    double b = -2.0 * (AuBu * (1.0 - wspeed2) - AB * wspeed2);
    double a = Bu2 * (1.0 - wspeed2) - Bsq * wspeed2;
    double discr = 4.0 * wspeed2 *
                   ((AB * AB - Asq * Bsq) * wspeed2 + (2.0 * AB * Au * Bu - Asq * Bu2 - Bsq * Au2) * (wspeed2 - 1.0));
    discr = kmath::sqrt(discr);
    double cst1 = (-b + discr) / (2.0 * a);
    double cst2 = (-b - discr) / (2.0 * a);
    if (cst2 > cst1) {
      aret[2 * dim] = cst1;
      aret[2 * dim + 1] = cst2;
    } else {
      aret[2 * dim] = cst2;
      aret[2 * dim + 1] = cst1;
    }
  }
}
// wavespeeds.zig:86
KC_HD double gas_wspeed2(double rho, double uu, double bsq, double gam) {
  double pre = (gam - 1.0) * uu;
  double cs2 = gam * pre / (rho + uu + pre);
  if (cs2 > 0.95) cs2 = 0.95;
  double va2 = bsq / (bsq + (rho + uu + pre));
  if (va2 < 0.0) va2 = 0.0;
  return cs2 + va2 - cs2 * va2;
}
// C calc_wavespeeds_lr_pure gas part with co-going clamps (wavespeeds.zig:100)
KC_HD void gas_wavespeeds_lr(const double pp[NV], const Geom& g, double gam, const bool active[3], double a[6]) {
  double ucon[4], ucov[4], bcon[4], bcov[4], bsq;
  ucon_ucov_from_prims(pp[VX], pp[VY], pp[VZ], g, ucon, ucov);
  double B[3] = {pp[B1], pp[B2], pp[B3]};
  bcon_bcov_bsq(B, ucon, ucov, g, bcon, bcov, bsq);
  double vtot2 = gas_wspeed2(pp[RHO], pp[UU], bsq, gam);
  double ws[3] = {vtot2, vtot2, vtot2};
  lr_core(ucon, g, ws, active, a);
  for (int dim = 0; dim < 3; ++dim) {
    if (a[2 * dim] > 0.0) a[2 * dim] = 0.0;
    if (a[2 * dim + 1] < 0.0) a[2 * dim + 1] = 0.0;
  }
}
// C calc_rad_wavespeeds (radiation.zig:177): aval[0..6] unlimited, [6..12] tau-damped
KC_HD void rad_wavespeeds(const double pp[NV], const Geom& g, const double tautot[3], const bool active[3], double aval[12]) {
  const double four_third = 4.0 / 3.0, one_third = 1.0 / 3.0;
  double vin[4] = {0.0, pp[FX], pp[FY], pp[FZ]};
  double urf[4];
  velr_to_vel4(vin, g, urf);
  double rv2rad = one_third;
  double ws0[3] = {rv2rad, rv2rad, rv2rad};
  lr_core(urf, g, ws0, active, aval);
  double rv2dim[3];
  for (int dim = 0; dim < 3; ++dim) {
    if (tautot[dim] <= 0.0) {
      rv2dim[dim] = rv2rad;
    } else {
      double rv2tau = (four_third * four_third) / (tautot[dim] * tautot[dim]);
      rv2dim[dim] = kmath::fmin(rv2rad, rv2tau);
    }
  }
  double ws1[3] = {rv2dim[0], rv2dim[1], rv2dim[1]};  // z uses the y depth (rad.c:3702)
  lr_core(urf, g, ws1, active, aval + 6);
}

}  // namespace kp
