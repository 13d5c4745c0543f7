// kvisc.h — the pure per-cell kernels of the radiative shear viscosity and of
// the mimic dynamo. Shared host/device restatement of
// koral/physics/radvisc.zig, koral/sim/dynamo.zig (dampBphi, dynamoDeltaA,
// fieldAngle) and koral/math/misc.zig.
#pragma once
#include "kmetric.h"
#include "kopts.h"

namespace kp {

// C step_function (koral/math/misc.zig:7)
KC_HD double step_function(double x, double x9) {
  double k = 1.47222 / x9;
  return 1.0 / (1.0 + kmath::exp(-2.0 * k * x));
}

// Lab-frame shear sigma_ij from assembled velocity gradients
// (radvisc.zig:67, C rad.c:4090). kr[k*16 + i*4 + j] = Gamma^k_ij.
KC_HD void shear_from_gradients(const double du[4][4], const double du2[4][4], const double ucon[4], const double ucov[4],
                                const Geom& g, const double* kr, double s[4][4]) {
  double dcu[4][4], dcudiag[4];
  for (int i = 0; i < 4; ++i) {
    for (int j = 0; j < 4; ++j) {
      double krsum = 0.0;
      for (int k = 0; k < 4; ++k) krsum += kr[k * 16 + i * 4 + j] * ucov[k];
      dcu[i][j] = du[i][j] - krsum;
    }
    double krsum = 0.0;
    for (int k = 0; k < 4; ++k) krsum += kr[i * 16 + i * 4 + k] * ucon[k];
    dcudiag[i] = du2[i][i] + krsum;
  }
  double theta = 0.0;
  for (int i = 0; i < 4; ++i) theta += dcudiag[i];
  double p11[4][4], p21[4][4];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      p11[i][j] = g.gg[i][j] + ucov[i] * ucov[j];
      p21[i][j] = kron(i, j) + ucon[i] * ucov[j];
    }
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) s[i][j] = 0.0;
  for (int i = 1; i < 4; ++i)
    for (int j = 1; j < 4; ++j) {
      double sum1 = 0.0, sum2 = 0.0;
      for (int k = 0; k < 4; ++k) {
        sum1 += dcu[i][k] * p21[k][j];
        sum2 += dcu[j][k] * p21[k][i];
      }
      s[i][j] = 0.5 * (sum1 + sum2) - 1.0 / 3.0 * theta * p11[i][j];
    }
  for (int i = 1; i < 4; ++i) {
    double v = -1.0 / ucon[0] * (ucon[1] * s[1][i] + ucon[2] * s[2][i] + ucon[3] * s[3][i]);
    s[i][0] = v;
    s[0][i] = v;
  }
  s[0][0] = -1.0 / ucon[0] * (ucon[1] * s[1][0] + ucon[2] * s[2][0] + ucon[3] * s[3][0]);
}

// C calc_rad_visccoeff limiter chain (radvisc.zig:145)
KC_HD double visc_coeff(double chi, double mindx, double r_bl, double rhor, double alpha, double global_dt) {
  const double small = 1.0e-80;
  double mfp = 1.0 / chi;
  double rmin = 1.2 * rhor;
  double mfplim = r_bl;
  if (mfp > mfplim || chi < small) mfp = mfplim;
  if (mfp < 0.0 || !kmath::isfinite(mfp)) mfp = 0.0;
  mfp *= step_function(r_bl - rmin, 0.2 * rmin);
  if (r_bl <= 1.0 * rhor) mfp = 0.0;
  double nu = alpha * mfp;
  double nulimit = mindx * mindx / 2.0 / global_dt / 2.0;
  if (nu > nulimit) nu = nulimit;
  return nu;
}

// R^i_j = lower_second(-2 nu E sigma^ij) (radvisc.zig:170)
KC_HD void rij_visc(double nu, double erad, const double shear[4][4], const Geom& g, double out[4][4]) {
  double rv[4][4];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) rv[i][j] = -2.0 * nu * erad * shear[i][j];
  lower_second(rv, g, out);
}

// RADVISCMAXVELDAMP face addition (radvisc.zig:186)
KC_HD void add_visc_flux(double ff[NV], const double uu[NV], const double rv[4][4], const Geom& g, int dim, bool y_active,
                         bool z_active, double maxvel) {
  double gdetu = g.gdet;
  double vel[3] = {0.0, 0.0, 0.0};
  for (int id = 0; id < 3; ++id) {
    for (int ii = 1; ii < 4; ++ii) {
      if (ii == 2 && !y_active) continue;
      if (ii == 3 && !z_active) continue;
      if (kmath::fabs(uu[EE + ii]) < 1.0e-10 * kmath::fabs(uu[EE])) continue;
      vel[id] = rv[id + 1][ii] / (uu[EE + ii] / gdetu) * kmath::sqrt(g.gg[id + 1][id + 1]);
    }
  }
  double maxv = kmath::fabs(vel[dim]);
  double dampfac = 1.0;
  if (maxv > maxvel) dampfac = maxvel / maxv;
  for (int nu = 0; nu < 4; ++nu) ff[EE + nu] += gdetu * dampfac * rv[dim + 1][nu];
}

// ---- mimic dynamo law (koral/sim/dynamo.zig:65-160) -------------------------
KC_HD double damp_bphi(double alphabeta, double facradius, double faczh, double dt_over_pk, double beta, double betasat,
                       double bphi) {
  double dbphi = -alphabeta * facradius * faczh * dt_over_pk * kmath::fmax(0.0, beta - betasat) / betasat * bphi;
  if ((dbphi + bphi) * bphi < 0.0) dbphi = -bphi;
  return dbphi;
}
struct DynamoOut {
  double aphi, bphi;
  bool skip;
};
// dynamo.zig:103 (C magn.c:1042-1151)
KC_HD DynamoOut dynamo_delta_a(const DynamoParams& dp, double a, double dt, double rhor, double risco, double r, double th,
                               double bphi, double bsq, double angle_in, double prermhd, double gg33, double scaleth) {
  DynamoOut o;
  if (r < 1.0001 * rhor) {
    o.aphi = 0.0;
    o.bphi = bphi;
    o.skip = true;
    return o;
  }
  double omk = 1.0 / (a + kmath::sqrt(r * r * r));
  double pk = 2.0 * KP_PI / omk;
  double angle = angle_in;
  double facangle = 0.0;
  if (kmath::isfinite(angle)) {
    if (angle < -1.0) angle = -1.0;
    facangle = kmath::fmax(0.0, (dp.thetaangle - angle) / dp.thetaangle);
  }
  double facradius = step_function(r - 1.0 * risco, 0.1 * risco);
  double beta = 0.5 * bsq / prermhd;
  double hrdtheta;
  if (dp.calchronthego) {
    hrdtheta = scaleth;
    if (hrdtheta > 0.9 * KP_PI / 2.0) hrdtheta = 0.9 * KP_PI / 2.0;
  } else {
    hrdtheta = dp.expectedhr * KP_PI / 2.0;
  }
  double zh = (KP_PI / 2.0 - th) / hrdtheta;
  double faczh = kmath::fmax(0.0, 1.0 - zh * zh);
  double facmagnetization = faczh;
  double effalpha = dp.alphadynamo;
  if (dp.alphaflipssign) effalpha = -(KP_PI / 2.0 - th) / (hrdtheta / 2.0) * dp.alphadynamo;
  o.aphi = effalpha * (hrdtheta / (KP_PI / 2.0)) / 0.4 * dt / pk * r * gg33 * bphi * facradius * facmagnetization * facangle;
  o.bphi = bphi;
  if (dp.dampbeta) {
    double dbphi = damp_bphi(dp.alphabeta, facradius, faczh, dt / pk, beta, dp.betasaturated, bphi);
    o.bphi = bphi + dbphi;
  }
  o.skip = false;
  return o;
}
// field pitch in BL (dynamo.zig:291 fieldAngle, C calc_angle_brbphibsq)
KC_HD int field_angle(const Geom& gm, const Geom& gbl, const double jac[4][4], const double pp[NV], double& angle,
                      double& bsq) {
  double ppbl[NV];
  int e = trans_pmhd_coco_j(pp, gm, gbl, jac, ppbl);
  if (e) return e;
  double ucon[4], ucov[4], bcon[4], bcov[4];
  ucon_ucov_from_prims(ppbl[VX], ppbl[VY], ppbl[VZ], gbl, ucon, ucov);
  double B[3] = {ppbl[B1], ppbl[B2], ppbl[B3]};
  bcon_bcov_bsq(B, ucon, ucov, gbl, bcon, bcov, bsq);
  double brbphi = kmath::sqrt(gbl.gg[1][1] * gbl.gg[3][3]) * bcon[1] * bcon[3];
  angle = -brbphi / bsq;
  return E_OK;
}

}  // namespace kp
