// kopts.h — host-side translation of the C-ABI kc_options into the per-point
// parameter structs, plus the PUFFY presets (koral/problems/puffy/puffy.zig:84
// Physics defaults, :179 makeGridNz, :210 toOptions). Shared by the engine's
// host code and the CPU oracle so both run the same parameter bits.
#pragma once
#include "../koralcuda.h"
#include "kmetric.h"
#include "kparams.h"

namespace kp {

// mimic-dynamo parameters (koral/sim/dynamo.zig:55)
struct DynamoParams {
  double alphadynamo, thetaangle, alphabeta, betasaturated, expectedhr;
  int alphaflipssign, dampbeta, calchronthego;
};

struct SimParams {
  MetricParams mp;
  double gam, tsteplim, minmod_theta;
  FloorParams fl;
  RadParams rp;
  OpacParams op;
  ImplicitParams ip;
  DynamoParams dp;
  int do_fixups, do_u2prad_fixups, do_radimp_fixups;
  int correct_polaraxis, nccorrectpolar;
  int radviscosity;
  double alpharadvisc, maxradviscvel;
  int dynamo;
  int reduceorderatbh, reduceorderafterfixup, dampradwavespeednearaxis;
  int bc[3];
};

inline void options_puffy(kc_options* o) {
  kc_options z = {};
  *o = z;
  o->abi_version = KC_ABI_VERSION;
  o->bhspin = 0.0;
  o->mksr0 = 0.1;
  o->mksh0 = 0.9;
  o->mass = 10.0;
  o->gam = 5.0 / 3.0;
  o->tsteplim = 0.5;
  o->minmod_theta = 1.5;
  FloorParams f = floor_params_puffy();
  o->rhofloor = f.rhofloor;
  o->uurhoratiomin = f.uurhoratiomin;
  o->uurhoratiomax = f.uurhoratiomax;
  o->b2rhoratiomax = f.b2rhoratiomax;
  o->b2uuratiomax = f.b2uuratiomax;
  o->gammamaxhd = f.gammamaxhd;
  o->isentropic_b2rhofloors = f.isentropic_b2rhofloors;
  o->b2uufloor = f.b2uufloor;
  o->horizon_x1 = f.horizon_x1;
  RadParams r = rad_params_puffy();
  o->gammamaxrad = r.gammamaxrad;
  o->eradfloor = r.eradfloor;
  o->eerhoratiomin = r.eerhoratiomin;
  o->eerhoratiomax = r.eerhoratiomax;
  o->eeuuratiomin = r.eeuuratiomin;
  o->eeuuratiomax = r.eeuuratiomax;
  o->bremsstrahlung = 1;
  o->synchrotron = 1;
  o->kleinnishina = 1;
  o->comptonization = 1;
  o->synchrotron_bridge = 0;
  o->scattering = 1;
  o->hfrac = 1.0;
  o->hefrac = 0.0;
  o->mu_gas = 1.0;
  o->mu_i = 2.0;
  o->mu_e = 2.0;
  ImplicitParams p = implicit_params_puffy();
  o->radimp_conv = p.conv;
  o->radimp_entrconv = p.entrconv;
  o->radimp_eps = p.eps;
  o->radimp_maxiter = p.maxiter;
  o->radimp_convrel = p.convrel;
  o->radimp_convrelerr = p.convrelerr;
  o->radimp_convrelentr = p.convrelentr;
  o->radimp_convrelentrerr = p.convrelentrerr;
  o->radimp_damping_factor = p.damping_factor;
  o->radimp_max_en_change_down = p.max_en_change_down;
  o->radimp_max_en_change_up = p.max_en_change_up;
  o->radimp_max_damping = p.max_damping;
  o->radimp_max_tgas_change = p.max_tgas_change;
  o->radimp_max_trad_change = p.max_trad_change;
  o->radimp_threshold = p.threshold;
  o->radimp_start_with_bisect = p.start_with_bisect;
  o->radimp_scale_jacobian = p.scale_jacobian;
  o->radimp_allow_rad_ceiling = p.allow_rad_ceiling;
  o->radimp_allow_entr_in_4dprim = p.allow_entr_in_4dprim;
  o->radimp_opdamp_maxlevels = p.opdamp_maxlevels;
  o->radimp_opdamp_factor = p.opdamp_factor;
  o->radimp_lag_opac = p.lag_opac;
  o->do_fixups = 1;
  o->do_u2prad_fixups = 0;
  o->do_radimp_fixups = 0;
  o->correct_polaraxis = 1;
  o->nccorrectpolar = 2;
  o->radviscosity = 1;
  o->alpharadvisc = 0.1;
  o->maxradviscvel = 0.1;
  o->dynamo = 1;
  o->alphadynamo = 2.0 * 0.314;
  o->thetaangle = 0.25;
  o->alphabeta = 2.0 * 6.28;
  o->betasaturated = 0.1;
  o->expectedhr = 0.3;
  o->alphaflipssign = 1;
  o->dampbeta = 1;
  o->calchronthego = 1;
  o->reduceorderatbh = 0;
  o->reduceorderafterfixup = 0;
  o->dampradwavespeednearaxis = 0;
  o->bc_x = KC_BC_PUFFY;
  o->bc_y = KC_BC_PUFFY;
  o->bc_z = KC_BC_PERIODIC;
  o->precision = KC_PLAIN_FP64;
  o->implicit_mode = KC_IMPLICIT_PER_CELL;
  o->device = 0;
}

// puffy.zig:185 makeGridNz with the default rmin 1.85, rmax 500, mksr0 0.1
inline void grid_puffy(int nx, int ny, int nz, kc_grid* g) {
  g->nx = nx;
  g->ny = ny;
  g->nz = nz;
  g->ng = 3;
  g->minx = kmath::log(1.85 - 0.1);
  g->maxx = kmath::log(500.0 - 0.1);
  g->miny = 0.001;
  g->maxy = 1.0 - 0.001;
  g->minz = -KP_PI / 4.0;
  g->maxz = KP_PI / 4.0;
}

inline void params_from_options(const kc_options& o, SimParams& s) {
  s.mp.a = o.bhspin;
  s.mp.mksr0 = o.mksr0;
  s.mp.mksh0 = o.mksh0;
  s.gam = o.gam;
  s.tsteplim = o.tsteplim;
  s.minmod_theta = o.minmod_theta;
  s.fl.rhofloor = o.rhofloor;
  s.fl.uurhoratiomin = o.uurhoratiomin;
  s.fl.uurhoratiomax = o.uurhoratiomax;
  s.fl.b2rhoratiomax = o.b2rhoratiomax;
  s.fl.b2uuratiomax = o.b2uuratiomax;
  s.fl.gammamaxhd = o.gammamaxhd;
  s.fl.isentropic_b2rhofloors = o.isentropic_b2rhofloors;
  s.fl.b2uufloor = o.b2uufloor;
  s.fl.horizon_x1 = o.horizon_x1;
  s.rp.gammamaxrad = o.gammamaxrad;
  s.rp.eradfloor = o.eradfloor;
  s.rp.eerhoratiomin = o.eerhoratiomin;
  s.rp.eerhoratiomax = o.eerhoratiomax;
  s.rp.eeuuratiomin = o.eeuuratiomin;
  s.rp.eeuuratiomax = o.eeuuratiomax;
  s.op.c = consts_init(o.mass, o.hfrac, o.hefrac, o.mu_gas, o.mu_i, o.mu_e);
  s.op.ch.bremsstrahlung = o.bremsstrahlung;
  s.op.ch.synchrotron = o.synchrotron;
  s.op.ch.kleinnishina = o.kleinnishina;
  s.op.ch.comptonization = o.comptonization;
  s.op.ch.synchrotron_bridge = o.synchrotron_bridge;
  s.op.kappa_mode = KAPPA_DEFAULT;
  s.op.kappa_grey = 0.0;
  s.op.kappaes_mode = o.scattering ? KAPPAES_PUFFY : KAPPAES_NONE;
  s.op.kappaes_grey = 0.0;
  s.op.opdamp = 1.0;
  s.ip.conv = o.radimp_conv;
  s.ip.entrconv = o.radimp_entrconv;
  s.ip.eps = o.radimp_eps;
  s.ip.maxiter = o.radimp_maxiter;
  s.ip.convrel = o.radimp_convrel;
  s.ip.convrelerr = o.radimp_convrelerr;
  s.ip.convrelentr = o.radimp_convrelentr;
  s.ip.convrelentrerr = o.radimp_convrelentrerr;
  s.ip.damping_factor = o.radimp_damping_factor;
  s.ip.max_en_change_down = o.radimp_max_en_change_down;
  s.ip.max_en_change_up = o.radimp_max_en_change_up;
  s.ip.max_damping = o.radimp_max_damping;
  s.ip.max_tgas_change = o.radimp_max_tgas_change;
  s.ip.max_trad_change = o.radimp_max_trad_change;
  s.ip.threshold = o.radimp_threshold;
  s.ip.start_with_bisect = o.radimp_start_with_bisect;
  s.ip.scale_jacobian = o.radimp_scale_jacobian;
  s.ip.allow_rad_ceiling = o.radimp_allow_rad_ceiling;
  s.ip.allow_entr_in_4dprim = o.radimp_allow_entr_in_4dprim;
  s.ip.opdamp_maxlevels = o.radimp_opdamp_maxlevels;
  s.ip.opdamp_factor = o.radimp_opdamp_factor;
  s.ip.lag_opac = o.radimp_lag_opac;
  s.dp.alphadynamo = o.alphadynamo;
  s.dp.thetaangle = o.thetaangle;
  s.dp.alphabeta = o.alphabeta;
  s.dp.betasaturated = o.betasaturated;
  s.dp.expectedhr = o.expectedhr;
  s.dp.alphaflipssign = o.alphaflipssign;
  s.dp.dampbeta = o.dampbeta;
  s.dp.calchronthego = o.calchronthego;
  s.do_fixups = o.do_fixups;
  s.do_u2prad_fixups = o.do_u2prad_fixups;
  s.do_radimp_fixups = o.do_radimp_fixups;
  s.correct_polaraxis = o.correct_polaraxis;
  s.nccorrectpolar = o.nccorrectpolar;
  s.radviscosity = o.radviscosity;
  s.alpharadvisc = o.alpharadvisc;
  s.maxradviscvel = o.maxradviscvel;
  s.dynamo = o.dynamo;
  s.reduceorderatbh = o.reduceorderatbh;
  s.reduceorderafterfixup = o.reduceorderafterfixup;
  s.dampradwavespeednearaxis = o.dampradwavespeednearaxis;
  s.bc[0] = o.bc_x;
  s.bc[1] = o.bc_y;
  s.bc[2] = o.bc_z;
}

// Sim.init preconditions (koral/sim.zig:319-363) that apply to this engine.
inline const char* validate_config(const kc_grid& g, const kc_options& o) {
  if (o.abi_version != KC_ABI_VERSION) return "kc_options.abi_version mismatch";
  if (g.nx < 1 || g.ny < 1 || g.nz < 1) return "grid sizes must be >= 1";
  if (g.ng < 3) return "ghost depth below the PPM stencil (ng < 3)";
  if (o.correct_polaraxis && g.ny <= 2 * o.nccorrectpolar) return "correct_polaraxis needs ny > 2*nccorrectpolar";
  if (o.bc_z == KC_BC_PUFFY) return "the PUFFY boundary callback has no z faces";
  if (g.nz > 1 && g.ny == 1) return "x-z 2D corner filling is not implemented (as in the reference)";
  if (g.ny == 1 && g.nz == 1) return "1-D runs are not supported (calc_BfromA has no 1-D branch)";
  if (o.do_u2prad_fixups || o.do_radimp_fixups || o.reduceorderatbh || o.reduceorderafterfixup)
    return "only the validated PUFFY fixup/order options are supported";
  return nullptr;
}

}  // namespace kp
