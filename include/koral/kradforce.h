// kradforce.h — thermodynamic constants, opacities, the radiation state fill,
// the thermal four-force G^mu with Comptonization, and the chi used by the
// wavespeed limiter. Shared host/device restatement of
// koral/physics/thermo.zig, koral/physics/opacities.zig,
// koral/physics/radforce.zig and koral/frames.zig (the boosts).
#pragma once
#include "kinvert.h"

namespace kp {

// koral/units.zig:13-32 (CGS constants, exact ko.h values)
#define KP_GGG 6.674e-8
#define KP_CCC 2.9979246e10
#define KP_MSUNCM 147700.0
#define KP_K_BOLTZ_CGS 1.3806488e-16
#define KP_M_ELECTR_CGS 9.1094e-28
#define KP_M_PROTON_CGS 1.67262158e-24
#define KP_SIGMA_RAD_CGS 5.670367e-5
#define KP_H_CGS 6.6260755e-27
#define KP_BIG 1.0e80

// koral/physics/thermo.zig:77 — the precomputed C globals. Built once on the
// host (consts_init) and copied verbatim to the device.
struct Consts {
  double masscm;
  double hfrac, hefrac, a_inv_mean, z2diva_mean;
  double lengu2cgs, numdensgu2cgs, rhogu2cgs, kappacgs2gu;
  double k_boltz_cgs, h_cgs, sigma_rad_cgs, m_proton_cgs, m_electr_cgs;
  double fourpi, sigma_rad_over_pi, four_sigmarad, one_over_four_sigmarad;
  double k_over_mecsq, kb_over_me, kb_over_mugas_mp, mugas_mp_over_kb, one_over_mue_mp, one_over_mui_mp;
  double one_over_log_2p6;
  // units helpers with the ko.h macro shapes (koral/units.zig:97,110)
  double kappa_cgs2gu_fac;  // (CCC*CCC)/(GGG*masscm)
  double enden_gu2cgs_fac;  // (CCC^4)/(GGG*masscm^2)
};

// Opacity channel switches (koral/physics/opacities.zig:61, Channels.puffy)
struct Channels {
  int bremsstrahlung, synchrotron, kleinnishina, comptonization, synchrotron_bridge;
};
enum : int { KAPPAES_NONE = 0, KAPPAES_PUFFY = 1, KAPPAES_GREY = 2 };
enum : int { KAPPA_DEFAULT = 0, KAPPA_GREY = 1 };

// koral/physics/radforce.zig:86 (radforce.Params)
struct OpacParams {
  Consts c;
  Channels ch;
  int kappa_mode;
  double kappa_grey;
  int kappaes_mode;
  double kappaes_grey;
  double opdamp;
};

// ---- thermo (koral/physics/thermo.zig) --------------------------------------
enum : int { TEMP_MIN_DUMMY = 0 };
#define KP_TEMPEMINIMAL 1.0e2
#define KP_TEMPIMINIMAL 1.0e2

// C calc_LTE_TfromE (thermo.zig:153)
KC_HD double lte_T_from_E(const Consts& c, double e) { return kmath::sqrt(kmath::sqrt(c.one_over_four_sigmarad * e)); }
// C calc_LTE_EfromT (thermo.zig:148)
KC_HD double lte_E_from_T(const Consts& c, double t) { return c.four_sigmarad * t * t * t * t; }
// C calc_PEQ_Tfromurho (thermo.zig:165)
KC_HD double t_from_urho(const Consts& c, double uint_, double rho, double gam) {
  double p = uint_ * (gam - 1.0);
  return kmath::div(c.mugas_mp_over_kb * p, rho);
}
// C calc_PEQ_ufromTrho (thermo.zig:176)
KC_HD double u_from_trho(const Consts& c, double t, double rho, double gam) {
  double p = c.kb_over_mugas_mp * rho * t;
  return kmath::div(p, (gam - 1.0));
}
struct Temps {
  double tgas, te, ti;
};
// C calc_PEQ_Teifrompp single-temperature branch (thermo.zig:188)
KC_HDM Temps temps_from_urho(const Consts& c, double uint_, double rho, double gam) {
  Temps t;
  t.tgas = t_from_urho(c, uint_, rho, gam);
  double te = t.tgas, ti = t.tgas;
  te = kmath::isfinite(te) ? te : KP_BIG;
  ti = kmath::isfinite(ti) ? ti : KP_BIG;
  te = (te < KP_TEMPEMINIMAL) ? KP_TEMPEMINIMAL : te;
  ti = (ti < KP_TEMPIMINIMAL) ? KP_TEMPIMINIMAL : ti;
  t.te = te;
  t.ti = ti;
  return t;
}
KC_HD double thermal_ne(const Consts& c, double rho) { return c.one_over_mue_mp * rho; }

// ---- opacities (koral/physics/opacities.zig) -------------------------------
struct Opac {
  double gas_abs, rad_abs, gas_num, rad_num, gas_ross, rad_ross, tot_emissivity;
};
enum : int { OPAC_FULL = 0, OPAC_RESIDUAL = 1, OPAC_CHI = 2 };

// C calc_opacities_from_state (opacities.zig:131), MESA channel absent
KC_HDN Opac calc_opacities(const Consts& c, const Channels& ch, double rho, double te, double trad, double tradbb,
                           double ne, double bsq, int level) {
  bool want_rad = level != OPAC_CHI;
  bool want_full = level == OPAC_FULL;
  double rt_te = kmath::sqrt(te);
  double rhocgs = c.rhogu2cgs * rho;
  double nethcgs = ne * c.numdensgu2cgs;
  double bsqcgs = c.fourpi * (bsq * c.enden_gu2cgs_fac);
  double bmagcgs = kmath::sqrt(bsqcgs);
  double bbenergy = (4.0 * c.sigma_rad_cgs) * te * te * te * te;
  double kappagasff = 0, kapparadff = 0, kappagasffross = 0, kapparadffross = 0;
  double kappagassyn = 0, kapparadsyn = 0, kapparadnumsyn = 0, kapparadsynross = 0, kappagassynross = 0;
  if (ch.bremsstrahlung) {
    double mfrac = 1.0 - c.hfrac - c.hefrac;
    double emis_ff = 1.4e-27 * nethcgs * (kmath::div((c.hfrac + c.hefrac + c.z2diva_mean * mfrac), c.m_proton_cgs)) * rt_te * 1.2 *
                     (1.0 + 4.4e-10 * te);
    kappagasff = c.kappacgs2gu * (kmath::div(emis_ff, bbenergy)) * rho;
    if (want_rad) {
      double zeta = kmath::div(trad, te);
      double zeta_inv = kmath::div(1.0, zeta);
      double zeta_inv_3 = zeta_inv * zeta_inv * zeta_inv;
      kapparadff = kappagasff * kmath::log1p(1.6 * zeta) * c.one_over_log_2p6 * zeta_inv_3;
      double zeta_root5 = kmath::pow(zeta, 0.2);
      double zeta_root5_inv_4 = kmath::div(1.0, (zeta_root5 * zeta_root5 * zeta_root5 * zeta_root5));
      double zeta_root5_inv_3 = zeta_root5 * zeta_root5_inv_4;
      double scale_pla_ros_ff =
          kmath::div(14.12, (432.7 - 106.8 * zeta_root5_inv_3 + 43.17 * zeta_root5_inv_4 + 57.88 * zeta_inv));
      kapparadffross = kappagasff * scale_pla_ros_ff * zeta_inv_3;
    }
    if (want_full) kappagasffross = kappagasff * 0.0330;
  }
  if (ch.synchrotron) {
    bool bridge = ch.synchrotron_bridge != 0;
    double tc_n = 5.07783e9;
    double trad_syn = trad;
    if (bridge) {
      double trad_lim = kmath::div(kmath::pow(tradbb, 4.0 / 3.0), kmath::pow(te, 1.0 / 3.0));
      trad_syn = (trad < trad_lim) ? trad_lim : trad;
    }
    double emis_synchro = 3.61e-34 * (kmath::div(nethcgs, rhocgs)) * te * te * bmagcgs * bmagcgs;
    kappagassyn = c.kappacgs2gu * (kmath::div(emis_synchro, bbenergy)) * rho;
    if (want_rad) {
      double nu_mbsyn = 1.19e-13 * te * te;
      double zbr = kmath::div(kmath::div(c.k_boltz_cgs * trad_syn, c.h_cgs), nu_mbsyn);
      double zeta_a_denom_rad =
          1.79 * kmath::cbrt(zbr * zbr * zbr * zbr * zbr * bmagcgs * bmagcgs * bmagcgs * bmagcgs) +
          1.35 * kmath::cbrt(zbr * zbr * zbr * zbr * zbr * zbr * zbr * bmagcgs * bmagcgs) + 0.248 * zbr * zbr * zbr;
      double ia_by_b_rad = kmath::div(bmagcgs * bmagcgs, zeta_a_denom_rad);
      double te5 = te * te * te * te * te;
      kapparadsyn = c.kappacgs2gu * (kmath::div(2.13e39 * (kmath::div(nethcgs, rhocgs)), te5) * ia_by_b_rad) * rho;
      if (bridge)
        kapparadsyn += c.kappacgs2gu *
                       (kmath::div(2.35869e-21 * (kmath::div(nethcgs, rhocgs)) * (bmagcgs * bmagcgs), (trad_syn * trad_syn * trad_syn))) * rho;
      if (want_full) {
        double zeta_a_denom_num = (0.025 * kmath::cbrt(zbr * zbr * zbr * zbr * bmagcgs * bmagcgs) +
                                   0.169 * kmath::cbrt(zbr * zbr * zbr * zbr * zbr * bmagcgs) + 0.287 * zbr * zbr);
        double ia_by_b_num = kmath::div(bmagcgs, zeta_a_denom_num);
        kapparadnumsyn = c.kappacgs2gu * (kmath::div(2.13e39 * (kmath::div(nethcgs, rhocgs)), te5) * ia_by_b_num) * rho;
        if (bridge) kapparadnumsyn *= kmath::div((kmath::div(te, tc_n)), (1.0 + kmath::div(te, tc_n)));
      }
      double bmb = (bmagcgs > 0.0) ? kmath::pow(bmagcgs, -0.463) : 0.0;
      double ia_by_b_ross_rad =
          kmath::div(0.13 * kmath::pow(bmagcgs, 0.69), (kmath::pow(zbr, 1.69) * kmath::exp(1.6 * kmath::pow(zbr, 0.463) * bmb)));
      kapparadsynross = c.kappacgs2gu * (kmath::div(2.13e39 * (kmath::div(nethcgs, rhocgs)), te5) * ia_by_b_ross_rad) * rho;
      if (want_full) {
        double zbg = kmath::div(kmath::div(c.k_boltz_cgs * te, c.h_cgs), nu_mbsyn);
        double ia_by_b_ross_gas =
            kmath::div(0.13 * kmath::pow(bmagcgs, 0.69), (kmath::pow(zbg, 1.69) * kmath::exp(1.6 * kmath::pow(zbg, 0.463) * bmb)));
        kappagassynross = c.kappacgs2gu * (kmath::div(2.13e39 * (kmath::div(nethcgs, rhocgs)), te5) * ia_by_b_ross_gas) * rho;
      }
    }
    if (bridge)
      kappagassyn += c.kappacgs2gu * (kmath::div(2.35869e-21 * (kmath::div(nethcgs, rhocgs)) * (bmagcgs * bmagcgs), (te * te * te))) * rho;
    if (!bridge) {
      double terel = te * c.k_over_mecsq;
      double terelfactor = kmath::div((terel * terel), (1.0 + terel * terel));
      kappagassyn *= terelfactor;
      if (want_rad) {
        kapparadsyn *= terelfactor;
        kapparadsynross *= terelfactor;
        if (want_full) {
          kapparadnumsyn *= terelfactor;
          kappagassynross *= terelfactor;
        }
      }
    }
  }
  Opac o;
  o.gas_abs = kappagasff + kappagassyn;
  o.rad_abs = kapparadff + kapparadsyn;
  o.gas_num = kappagasff;
  o.rad_num = kapparadff + kapparadnumsyn;
  o.gas_ross = kappagasffross + kappagassynross;
  o.rad_ross = kapparadffross + kapparadsynross;
  o.tot_emissivity = 0.0;
  return o;
}

// PUFFY Klein-Nishina scattering opacity (opacities.zig:352, C kappaes.c)
KC_HD double kappaes_puffy(const Consts& c, const Channels& ch, double rho, double trad) {
  double opac_correction = 1.0;
  if (ch.kleinnishina) {
    double tkn = trad;
    opac_correction = kmath::div(1.0, (1.0 + kmath::pow(kmath::div(tkn, 4.5e8), 0.86)));
  }
  return ((0.2 * (1.0 + c.hfrac)) * opac_correction) * c.kappa_cgs2gu_fac * rho;
}
KC_HD double kappaes_at(const OpacParams& op, double rho, double trad) {
  if (op.kappaes_mode == KAPPAES_PUFFY) return kappaes_puffy(op.c, op.ch, rho, trad);
  if (op.kappaes_mode == KAPPAES_GREY) return op.kappaes_grey * rho;
  return 0.0;
}

// ---- radiation state (koral/physics/radforce.zig:174) ----------------------
struct RadState {
  double rho, uint_, tgas, te, ti, sgas, ne;
  double ucon[4], ucov[4];
  double bsq;
  double rij[4][4];
  double ehat, tradbb, trad, kappaes, kappa;
  Opac opac;
};

// C fill_struct_of_state radiation branch (radforce.zig:241). full=true fills
// every field; full=false is the solver's slim fill (sgas and the
// number/gas-Rosseland channels left zero, exactly as the reference).
KC_HDN void fill_rad_state(const double pp[NV], const Geom& g, double gam, const OpacParams& op, bool full, RadState& st) {
  const Consts& c = op.c;
  double rho = pp[RHO], uint_ = pp[UU];
  Temps t = temps_from_urho(c, uint_, rho, gam);
  st.sgas = full ? c.kb_over_mugas_mp * s_from_u(rho, uint_, gam) : 0.0;
  st.ne = thermal_ne(c, rho);
  ucon_ucov_from_prims(pp[VX], pp[VY], pp[VZ], g, st.ucon, st.ucov);
  double B[3] = {pp[B1], pp[B2], pp[B3]};
  double bcon[4], bcov[4];
  bcon_bcov_bsq(B, st.ucon, st.ucov, g, bcon, bcov, st.bsq);
  calc_rij(pp, g, st.rij);
  double ehat = 0.0;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) ehat += st.rij[i][j] * st.ucov[i] * st.ucov[j];
  st.ehat = ehat;
  st.tradbb = lte_T_from_E(c, ehat);
  st.trad = st.tradbb;
  st.kappaes = kappaes_at(op, rho, st.trad);
  if (op.kappa_mode == KAPPA_DEFAULT) {
    st.opac = calc_opacities(c, op.ch, rho, t.te, st.trad, st.tradbb, st.ne, st.bsq, full ? OPAC_FULL : OPAC_RESIDUAL);
    if (full) {
      double b = c.sigma_rad_over_pi * t.te * t.te * t.te * t.te;
      st.opac.tot_emissivity = st.opac.gas_abs * c.fourpi * b;
    }
    st.kappa = st.opac.gas_abs;
  } else {
    double kap = op.kappa_grey * rho;
    double b = c.sigma_rad_over_pi * t.te * t.te * t.te * t.te;
    st.opac.gas_abs = kap;
    st.opac.rad_abs = kap;
    st.opac.gas_num = kap;
    st.opac.rad_num = kap;
    st.opac.gas_ross = kap;
    st.opac.rad_ross = kap;
    st.opac.tot_emissivity = kap * c.fourpi * b;
    st.kappa = kap;
  }
  st.rho = rho;
  st.uint_ = uint_;
  st.tgas = t.tgas;
  st.te = t.te;
  st.ti = t.ti;
}

// ---- Lorentz boosts (koral/frames.zig:38-96) --------------------------------
KC_HD void lorentz_from_pair(const double ucon[4], const double ucov[4], const double wcon[4], const double wcov[4],
                             double l[4][4]) {
  double om[4][4];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) om[i][j] = ucon[i] * wcov[j] - wcon[i] * ucov[j];
  double gam = -dot(wcon, ucov);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double omsum = 0.0;
      for (int k = 0; k < 4; ++k) omsum += om[i][k] * om[k][j];
      l[i][j] = kron(i, j) + kmath::div(1.0, (1.0 + gam)) * omsum + om[i][j];
    }
}
KC_HD void normal_obs_concov(const Geom& g, double con[4], double cov[4]) {
  double alpha = kmath::sqrt(kmath::div(-1.0, g.GG[0][0]));
  cov[0] = -alpha;
  cov[1] = 0.0;
  cov[2] = 0.0;
  cov[3] = 0.0;
  raise_vec(cov, g, con);
}
// C calc_Lorentz_lab2ff (frames.zig:77)
KC_HDM void lorentz_lab2ff(double v1, double v2, double v3, const Geom& g, double l[4][4]) {
  double ucon[4], ucov[4], wcon[4], wcov[4];
  ucon_ucov_from_prims(v1, v2, v3, g, ucon, ucov);
  normal_obs_concov(g, wcon, wcov);
  lorentz_from_pair(ucon, ucov, wcon, wcov, l);
}
// C calc_Lorentz_ff2lab (frames.zig:84)
KC_HDM void lorentz_ff2lab(double v1, double v2, double v3, const Geom& g, double l[4][4]) {
  double wcon[4], wcov[4], ucon[4], ucov[4];
  ucon_ucov_from_prims(v1, v2, v3, g, wcon, wcov);
  normal_obs_concov(g, ucon, ucov);
  lorentz_from_pair(ucon, ucov, wcon, wcov, l);
}
// A2 = alpha (L_lab2ff A1) (frames.zig:101, C boost2_lab2ff)
KC_HDM void boost2_lab2ff(const double a1[4], double v1, double v2, double v3, const Geom& g, double a2[4]) {
  double l[4][4];
  lorentz_lab2ff(v1, v2, v3, g, l);
  transform_vec(a1, l, a2);
  double alpha = kmath::sqrt(kmath::div(-1.0, g.GG[0][0]));
  for (int i = 0; i < 4; ++i) a2[i] *= alpha;
}
// A2 = L_ff2lab (A1 / alpha) (frames.zig:108, C boost2_ff2lab)
KC_HDM void boost2_ff2lab(const double a1[4], double v1, double v2, double v3, const Geom& g, double a2[4]) {
  double l[4][4];
  lorentz_ff2lab(v1, v2, v3, g, l);
  double alpha = kmath::sqrt(kmath::div(-1.0, g.GG[0][0]));
  double at[4];
  for (int i = 0; i < 4; ++i) at[i] = kmath::div(a1[i], alpha);
  transform_vec(at, l, a2);
}
// T2 = L L T1, no alpha (frames.zig:147, C boost22_ff2lab)
KC_HDM void boost22_ff2lab(const double t1[4][4], double v1, double v2, double v3, const Geom& g, double t2[4][4]) {
  double l[4][4];
  lorentz_ff2lab(v1, v2, v3, g, l);
  transform_tensor(t1, l, t2);
}

// ---- four-force (koral/physics/radforce.zig:370-494) ------------------------
KC_HD double compton_gi_coeff(const Consts& c, const RadState& st) {
  double thetae = c.kb_over_me * st.te;
  return kmath::div(st.kappaes * st.ehat * ((4.0 * c.kb_over_me) * (st.trad - st.te)) *
         (1.0 + 3.683 * thetae + 4.0 * thetae * thetae), (1.0 + 4.0 * thetae));
}
// C calc_all_Gi_with_state thermal part (radforce.zig:432) before the
// opacity-damping factor. full=false leaves ff[1..3] zero and skips the boost
// (the solver path).
KC_HDM void calc_gi_undamped(const RadState& st, double v1, double v2, double v3, const Geom& g, const OpacParams& op,
                             bool full, double gi_ff[4], double gi_lab[4]) {
  const Consts& c = op.c;
  double b = c.sigma_rad_over_pi * st.te * st.te * st.te * st.te;
  double k_rad_abs = st.opac.rad_abs, k_gas_abs = st.opac.gas_abs, k_rad_ross = st.opac.rad_ross;
  double kappaes = st.kappaes;
  double ruu = st.ehat;
  for (int i = 0; i < 4; ++i) {
    double ru = 0.0;
    for (int j = 0; j < 4; ++j) ru += st.rij[i][j] * st.ucov[j];
    gi_lab[i] = -(k_rad_ross + kappaes) * ru - ((k_rad_ross + kappaes - k_rad_abs) * ruu + k_gas_abs * c.fourpi * b) * st.ucon[i];
  }
  if (full) {
    boost2_lab2ff(gi_lab, v1, v2, v3, g, gi_ff);
  } else {
    for (int i = 0; i < 4; ++i) gi_ff[i] = 0.0;
  }
  gi_ff[0] = -k_gas_abs * c.fourpi * b + k_rad_abs * st.ehat;
  if (op.ch.comptonization) {
    double coeff = compton_gi_coeff(c, st);
    for (int i = 0; i < 4; ++i) gi_lab[i] += coeff * st.ucon[i];
    gi_ff[0] += coeff;
  }
}
// the opacity-damping factor of the implicit ladder's damped levels
KC_HD void damp_gi(double od, double gi_ff[4], double gi_lab[4]) {
  if (od != 1.0) {
    for (int i = 0; i < 4; ++i) {
      gi_ff[i] *= od;
      gi_lab[i] *= od;
    }
  }
}
// C calc_all_Gi_with_state thermal part (radforce.zig:432), damped by op.opdamp
KC_HDM void calc_gi_from_state(const RadState& st, double v1, double v2, double v3, const Geom& g, const OpacParams& op,
                              bool full, double gi_ff[4], double gi_lab[4]) {
  calc_gi_undamped(st, v1, v2, v3, g, op, full, gi_ff, gi_lab);
  damp_gi(op.opdamp, gi_ff, gi_lab);
}

// C calc_kappaes standalone flavor, Trad = Te (radforce.zig:522)
KC_HD double calc_kappaes_standalone(const double pp[NV], double gam, const OpacParams& op) {
  Temps t = temps_from_urho(op.c, pp[UU], pp[RHO], gam);
  return kappaes_at(op, pp[RHO], t.te);
}
// chi = kappa + kappa_es for the tau limiter and the viscous mfp
// (radforce.zig:562, calcChiSlim — bit-identical to calcChi)
KC_HD double calc_chi_slim(const double pp[NV], const Geom& g, double gam, const OpacParams& op) {
  const Consts& c = op.c;
  double rho = pp[RHO], uint_ = pp[UU];
  Temps t = temps_from_urho(c, uint_, rho, gam);
  double ne = thermal_ne(c, rho);
  double ucon[4], ucov[4], bcon[4], bcov[4], bsq;
  ucon_ucov_from_prims(pp[VX], pp[VY], pp[VZ], g, ucon, ucov);
  double B[3] = {pp[B1], pp[B2], pp[B3]};
  bcon_bcov_bsq(B, ucon, ucov, g, bcon, bcov, bsq);
  double kappa;
  if (op.kappa_mode == KAPPA_DEFAULT) {
    Opac o = calc_opacities(c, op.ch, rho, t.te, t.te, t.te, ne, bsq, OPAC_CHI);
    kappa = o.gas_abs;
  } else {
    kappa = op.kappa_grey * rho;
  }
  double kappaes = kappaes_at(op, rho, t.te);
  return kappa + kappaes;
}

}  // namespace kp
