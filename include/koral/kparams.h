// kparams.h — the PUFFY parameter presets and the host-side construction of
// the precomputed physical constants. Host code shared by the engine's
// options builder and the CPU oracle, so both see the same constant bits.
#pragma once
#include "kflux.h"
#include "kimplicit.h"

namespace kp {

// koral/solve/invert.zig:81 (FloorParams.puffy, DRIFTFRAME)
inline FloorParams floor_params_puffy() {
  FloorParams f;
  f.rhofloor = 1.0e-30;
  f.uurhoratiomin = 1.0e-8;
  f.uurhoratiomax = 1.0e0;
  f.b2rhoratiomax = 50.0;
  f.b2uuratiomax = 50.0;
  f.gammamaxhd = 10.0;
  f.isentropic_b2rhofloors = 0;
  f.b2uufloor = 1;
  f.horizon_x1 = -kmath::inf();
  return f;
}

// koral/solve/invert_rad.zig:47 (RadParams.puffy); eradfloor = 10 * SMALL
inline RadParams rad_params_puffy() {
  RadParams r;
  r.gammamaxrad = 10.0;
  r.eradfloor = 1.0e-79;
  r.eerhoratiomin = 1.0e-20;
  r.eerhoratiomax = 1.0e4;
  r.eeuuratiomin = 1.0e-20;
  r.eeuuratiomax = 1.0e20;
  return r;
}

// koral/solve/implicit.zig:138 (ImplicitParams.puffy)
inline ImplicitParams implicit_params_puffy() {
  ImplicitParams p;
  p.conv = 1.0e-10;
  p.entrconv = 1.0e-5;
  p.eps = 1.0e-6;
  p.maxiter = 40;
  p.convrel = 1.0e-8;
  p.convrelerr = 1.0e-4;
  p.convrelentr = 1.0e-4;
  p.convrelentrerr = 1.0e-2;
  p.damping_factor = 3.0;
  p.max_en_change_down = 10.0;
  p.max_en_change_up = 10.0;
  p.max_damping = 1.0e-3;
  p.max_tgas_change = 10.0;
  p.max_trad_change = 10.0;
  p.threshold = 1.0e-2;
  p.start_with_bisect = 1;
  p.scale_jacobian = 1;
  p.allow_rad_ceiling = 1;
  p.allow_entr_in_4dprim = 1;
  p.opdamp_maxlevels = 0;
  p.opdamp_factor = 3.0;
  p.lag_opac = 0;
  return p;
}

// koral/physics/thermo.zig:100 (Consts.init) with the PUFFY composition
// (HFRAC 1, MU_GAS/MU_I/MU_E = 1/2/2 overrides, thermo.zig:46).
inline Consts consts_init(double mass_msun, double hfrac = 1.0, double hefrac = 0.0, double mu_gas = 1.0,
                          double mu_i = 2.0, double mu_e = 2.0) {
  Consts c;
  const double GGG = KP_GGG, CCC = KP_CCC;
  double masscm = mass_msun * KP_MSUNCM;
  c.masscm = masscm;
  c.hfrac = hfrac;
  c.hefrac = hefrac;
  c.a_inv_mean = 0.0570490404519;
  c.z2diva_mean = 5.14445150955;
  double k_boltz = KP_K_BOLTZ_CGS * GGG / CCC / CCC / CCC / CCC / masscm;
  double m_proton = KP_M_PROTON_CGS * (GGG / (masscm * CCC * CCC));
  double m_electr = KP_M_ELECTR_CGS * (GGG / (masscm * CCC * CCC));
  double sigma_rad = KP_SIGMA_RAD_CGS * GGG / CCC / CCC / CCC / CCC / CCC * masscm * masscm;
  double four_sigmarad = 4.0 * sigma_rad;
  const double pi = 3.141592653589793;
  c.lengu2cgs = masscm;
  c.numdensgu2cgs = 1.0 / masscm / masscm / masscm;
  c.rhogu2cgs = 1.0 / GGG * CCC * CCC / masscm / masscm;
  c.kappacgs2gu = 1.0 / GGG * CCC * CCC / masscm;
  c.k_boltz_cgs = KP_K_BOLTZ_CGS;
  c.h_cgs = KP_H_CGS;
  c.sigma_rad_cgs = KP_SIGMA_RAD_CGS;
  c.m_proton_cgs = KP_M_PROTON_CGS;
  c.m_electr_cgs = KP_M_ELECTR_CGS;
  c.fourpi = 4.0 * pi;
  c.sigma_rad_over_pi = sigma_rad / pi;
  c.four_sigmarad = four_sigmarad;
  c.one_over_four_sigmarad = 1.0 / four_sigmarad;
  c.k_over_mecsq = 1.69e-10;
  c.kb_over_me = k_boltz / m_electr;
  c.kb_over_mugas_mp = k_boltz / mu_gas / m_proton;
  c.mugas_mp_over_kb = 1.0 / (k_boltz / mu_gas / m_proton);
  c.one_over_mue_mp = 1.0 / mu_e / m_proton;
  c.one_over_mui_mp = 1.0 / mu_i / m_proton;
  c.one_over_log_2p6 = 0x1.0beb5a290255cp+0;  // 1/ln(2.6), evaluated exactly then rounded
  c.kappa_cgs2gu_fac = (CCC * CCC) / (GGG * masscm);
  c.enden_gu2cgs_fac = (CCC * CCC * CCC * CCC) / (GGG * masscm * masscm);
  return c;
}

// radforce.Params.puffyMass (koral/physics/radforce.zig:128)
inline OpacParams opac_params_puffy(double mass_msun = 10.0) {
  OpacParams o;
  o.c = consts_init(mass_msun);
  o.ch.bremsstrahlung = 1;
  o.ch.synchrotron = 1;
  o.ch.kleinnishina = 1;
  o.ch.comptonization = 1;
  o.ch.synchrotron_bridge = 0;
  o.kappa_mode = KAPPA_DEFAULT;
  o.kappa_grey = 0.0;
  o.kappaes_mode = KAPPAES_PUFFY;
  o.kappaes_grey = 0.0;
  o.opdamp = 1.0;
  return o;
}

// RK2IMEX gamma = 1 - 1/sqrt(2) and 1 - 2 gamma, evaluated exactly and rounded
// once (the reference folds both at compile time, koral/sim.zig:1820,1856).
#define KP_GAM_IMEX 0x1.2bec333018867p-2
#define KP_ONE_M2GAM 0x1.a827999fcef32p-2

}  // namespace kp
