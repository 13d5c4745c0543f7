// kimplicit.h — the implicit radiation-gas coupling solve: the 6-rung ladder,
// the 4-primitive Newton with its one-sided finite-difference Jacobian, the
// conservation constraint and the 1-D bisection warm start. Shared host/device
// restatement of koral/solve/implicit.zig (C rad.c:73-2001).
#pragma once
#include "kradforce.h"

namespace kp {

// RADIMP* parameters (koral/solve/implicit.zig:83, ImplicitParams.puffy at :138)
struct ImplicitParams {
  double conv, entrconv, eps;
  int maxiter;
  double convrel, convrelerr, convrelentr, convrelentrerr;
  double damping_factor, max_en_change_down, max_en_change_up, max_damping;
  double max_tgas_change, max_trad_change, threshold;
  int start_with_bisect, scale_jacobian, allow_rad_ceiling, allow_entr_in_4dprim;
  int opdamp_maxlevels;
  double opdamp_factor;
  int lag_opac;
};

enum : int { PRIM_RAD = 1, PRIM_MHD = 2 };
enum : int { EQ_ENERGY = 0, EQ_ENTROPY = 1 };
enum : int { FRAME_LAB = 0, FRAME_FF = 1 };

struct ImplicitResult {
  int ok;
  int rung;
  int iters;
  int whichprim, whicheq, whichframe;
};

// C my_sign (implicit.zig:164): sign(0) = +1
KC_HD double my_sign(double x) {
  if (x > 0.0) return 1.0;
  if (x < 0.0) return -1.0;
  return 1.0;
}

// 4x4 LU inversion with partial pivoting, no error path (implicit.zig:172)
KC_HDN void invert4(const double a_in[4][4], double inv[4][4]) {
  double lu[4][4];
  int perm[4] = {0, 1, 2, 3};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) lu[i][j] = a_in[i][j];
  for (int k = 0; k < 4; ++k) {
    int piv = k;
    double pmax = kmath::fabs(lu[k][k]);
    for (int r = k + 1; r < 4; ++r) {
      if (kmath::fabs(lu[r][k]) > pmax) {
        pmax = kmath::fabs(lu[r][k]);
        piv = r;
      }
    }
    if (piv != k) {
      for (int c = 0; c < 4; ++c) {
        double t = lu[k][c];
        lu[k][c] = lu[piv][c];
        lu[piv][c] = t;
      }
      int tp = perm[k];
      perm[k] = perm[piv];
      perm[piv] = tp;
    }
    for (int r = k + 1; r < 4; ++r) {
      lu[r][k] = kmath::div(lu[r][k], lu[k][k]);
      for (int cc = k + 1; cc < 4; ++cc) lu[r][cc] -= lu[r][k] * lu[k][cc];
    }
  }
  for (int col = 0; col < 4; ++col) {
    double y[4], x[4];
    for (int r = 0; r < 4; ++r) {
      y[r] = (perm[r] == col) ? 1.0 : 0.0;
      for (int cc = 0; cc < r; ++cc) y[r] -= lu[r][cc] * y[cc];
    }
    for (int r = 3; r >= 0; --r) {
      x[r] = y[r];
      for (int cc = r + 1; cc < 4; ++cc) x[r] -= lu[r][cc] * x[cc];
      x[r] = kmath::div(x[r], lu[r][r]);
    }
    for (int rr = 0; rr < 4; ++rr) inv[rr][col] = x[rr];
  }
}

// C implicit_apply_constraints (implicit.zig:240). 0 ok, -1 tolerable, -2 fatal.
KC_HDN int apply_constraints(double pp[NV], double uu[NV], const double uu0[NV], const Geom& g, double gam,
                             const RadParams& rad, const ImplicitParams& ip, int whichprim) {
  double gdetu = g.gdet;
  double gdetu_inv = kmath::div(1.0, gdetu);
  if (whichprim == PRIM_MHD) {
    double ucon[4], ucov[4];
    ucon_ucov_from_prims(pp[VX], pp[VY], pp[VZ], g, ucon, ucov);
    pp[RHO] = kmath::div(uu0[RHO] * gdetu_inv, ucon[0]);
    pp[ENTR] = s_from_u(pp[RHO], pp[UU], gam);
    p2u_mhd(pp, uu, g, gam);
    for (int k = 0; k < 4; ++k) uu[EE + k] = uu0[EE + k] - (uu[UU + k] - uu0[UU + k]);
    U2pRadRes rr = u2p_rad(uu, pp, g, rad);
    int u2pret = rr.ret;
    if (rr.corrected) u2pret = ip.allow_rad_ceiling ? -1 : -2;
    return u2pret;
  } else {
    p2u_rad(pp, uu, g);
    uu[RHO] = uu0[RHO];
    for (int k = 0; k < 4; ++k) uu[UU + k] = uu0[UU + k] - (uu[EE + k] - uu0[EE + k]);
    for (int k = 0; k < 3; ++k) uu[B1 + k] = gdetu * pp[B1 + k];
    int rettemp = u2p_solver_w(uu, pp, g, ETYPE_HOT, gam);
    if (rettemp < 0 && ip.allow_entr_in_4dprim) rettemp = u2p_solver_w(uu, pp, g, ETYPE_ENTROPY, gam);
    int u2pret = (rettemp < 0) ? -2 : 0;
    double ucon[4], ucov[4];
    ucon_ucov_from_prims(pp[VX], pp[VY], pp[VZ], g, ucon, ucov);
    pp[ENTR] = s_from_u(pp[RHO], pp[UU], gam);
    uu[ENTR] = pp[ENTR] * gdetu * ucon[0];
    return u2pret;
  }
}

// C f_implicit_lab_4dprim_with_state (implicit.zig:337); returns the max
// normalized error (NaN entries never win the max, as in the reference).
// `opdamp` is the ladder level's opacity damping (radforce.Params.opdamp,
// carried apart from `op` so the level's parameters are never copied).
KC_HDN double implicit_residual(const double uu[NV], const double pp[NV], const RadState& st, const double uu0[NV],
                                const RadState& st0, double dt, const Geom& g, const OpacParams& op, double opdamp,
                                int whichprim, int whicheq, int whichframe, double f[4]) {
  const double small = 1.0e-80;
  double gdetu = g.gdet;
  double tgas = st.tgas;
  double ehat0 = st0.ehat;
  double ehat = st.ehat;
  double dtau = kmath::div(dt, st.ucon[0]);
  double giff[4], gilab[4], gi[4];
  calc_gi_undamped(st, pp[VX], pp[VY], pp[VZ], g, op, false, giff, gilab);
  damp_gi(opdamp, giff, gilab);
  lower_vec(gilab, g, gi);
  double err[4] = {0.0, 0.0, 0.0, 0.0};
  if (whichprim == PRIM_MHD) {
    for (int k = 1; k < 4; ++k) {
      f[k] = uu[UU + k] - uu0[UU + k] - dt * gdetu * gi[k];
      err[k] = (kmath::fabs(f[k]) > small)
                   ? kmath::div(kmath::fabs(f[k]), (1.0e-20 * uu[UU] + kmath::fabs(uu[UU + k]) + kmath::fabs(uu0[UU + k]) +
                                          kmath::fabs(dt * gdetu * gi[k])))
                   : 0.0;
    }
  } else {
    for (int k = 1; k < 4; ++k) {
      f[k] = uu[EE + k] - uu0[EE + k] + dt * gdetu * gi[k];
      err[k] = (kmath::fabs(f[k]) > small)
                   ? kmath::div(kmath::fabs(f[k]), (1.0e-20 * uu[EE] + kmath::fabs(uu[EE + k]) + kmath::fabs(uu0[EE + k]) +
                                          kmath::fabs(dt * gdetu * gi[k])))
                   : 0.0;
    }
  }
  if (whichframe == FRAME_LAB) {
    if (whichprim == PRIM_RAD) {
      f[0] = uu[EE] - uu0[EE] + dt * gdetu * gi[0];
      err[0] = (kmath::fabs(f[0]) > small)
                   ? kmath::div(kmath::fabs(f[0]), (kmath::fabs(uu[EE]) + kmath::fabs(uu0[EE]) + kmath::fabs(dt * gdetu * gi[0])))
                   : 0.0;
    } else {
      f[0] = uu[UU] - uu0[UU] - dt * gdetu * gi[0];
      err[0] = (kmath::fabs(f[0]) > small)
                   ? kmath::div(kmath::fabs(f[0]), (kmath::fabs(uu[UU]) + kmath::fabs(uu0[UU]) + kmath::fabs(dt * gdetu * gi[0])))
                   : 0.0;
    }
  } else {
    if (whicheq == EQ_ENERGY) {
      if (whichprim == PRIM_RAD) {
        f[0] = ehat - ehat0 + dtau * giff[0];
        err[0] = kmath::div(kmath::fabs(f[0]), (kmath::fabs(ehat) + kmath::fabs(ehat0) + kmath::fabs(dtau * giff[0])));
      } else {
        f[0] = pp[UU] - st0.uint_ - dtau * giff[0];
        err[0] = kmath::div(kmath::fabs(f[0]), (kmath::fabs(pp[UU]) + kmath::fabs(st0.uint_) + kmath::fabs(dtau * giff[0])));
      }
    } else {
      double s0 = st0.sgas;
      double s = st.sgas;
      f[0] = tgas * (s - s0) - dtau * giff[0];
      err[0] = kmath::div(kmath::fabs(f[0]), (kmath::fabs(tgas * s) + kmath::fabs(tgas * s0) + kmath::fabs(dtau * giff[0])));
    }
  }
  double err0 = 0.0;
  for (int k = 0; k < 4; ++k) err0 = (err[k] > err0) ? err[k] : err0;
  return err0;
}

// C f_implicit_1dprim_err (implicit.zig:431)
KC_HDM double f1d_err(double xxx, const double pp0[NV], double dtau, const Geom& g, double gam, const OpacParams& op,
                     int whichprim, double totenergy, double ratio) {
  double ugas, ehat;
  if (whichprim == PRIM_RAD) {
    ehat = xxx * ratio;
    ugas = totenergy - ehat;
  } else {
    ugas = xxx;
    ehat = totenergy - ugas;
  }
  double pp[NV];
  for (int i = 0; i < NV; ++i) pp[i] = pp0[i];
  pp[UU] = ugas;
  pp[EE] = kmath::div(ehat, ratio);
  RadState st;
  fill_rad_state(pp, g, gam, op, false, st);
  double giff[4], gilab[4];
  calc_gi_from_state(st, pp[VX], pp[VY], pp[VZ], g, op, false, giff, gilab);
  if (whichprim == PRIM_RAD) return ehat - kmath::div(pp0[EE], ratio) + dtau * giff[0];
  return ugas - pp0[UU] - dtau * giff[0];
}

// C solve_implicit_lab_1dprim (implicit.zig:473)
KC_HDN int solve_1d_prim(const double pp00[NV], const RadState& st00, const Geom& g, double dt, double gam,
                         const OpacParams& op, double pp0out[NV]) {
  double ehat = st00.ehat;
  double dtau = kmath::div(dt, st00.ucon[0]);
  double totenergy = ehat + pp00[UU];
  int whichprim = (ehat < 1.0e-3 * pp00[UU]) ? PRIM_RAD : PRIM_MHD;
  double tgas = st00.tgas;
  double ratio = kmath::div(ehat, pp00[EE]);
  const double fac = 3.0;
  const double fac1 = fac + 1.0;
  double pp_uu = pp00[UU];
  double pp_ee = pp00[EE];
  if (tgas > 1.0e14) {
    pp_uu = kmath::div(pp00[UU] * 1.0e14, tgas);
    pp_ee = kmath::div((totenergy - pp_uu), ratio);
  }
  double xlo, xhi;
  if (whichprim == PRIM_MHD) {
    xlo = kmath::div(pp_uu, 1.05);
    xhi = kmath::fmin(pp_uu * 1.05, kmath::div((pp_uu + fac * totenergy), fac1));
  } else {
    xlo = kmath::div(pp_ee, 1.05);
    xhi = kmath::fmin(pp_ee * 1.05, kmath::div((pp_ee + kmath::div(fac * totenergy, ratio)), fac1));
  }
  double errlo = f1d_err(xlo, pp00, dtau, g, gam, op, whichprim, totenergy, ratio);
  double errhi = f1d_err(xhi, pp00, dtau, g, gam, op, whichprim, totenergy, ratio);
  const int maxiter = 50;
  const double conv = 1.0e-3;
  int iter = 0;
  while (errlo * errhi > 0.0) {
    iter += 1;
    if (errlo > 0.0) {
      xhi = xlo;
      errhi = errlo;
      xlo /= fac;
      errlo = f1d_err(xlo, pp00, dtau, g, gam, op, whichprim, totenergy, ratio);
    } else {
      xlo = xhi;
      errlo = errhi;
      if (whichprim == PRIM_RAD) xhi = kmath::fmin(xhi * fac, kmath::div((xhi + kmath::div(fac * totenergy, ratio)), fac1));
      else xhi = kmath::fmin(xhi * fac, kmath::div((xhi + fac * totenergy), fac1));
      errhi = f1d_err(xhi, pp00, dtau, g, gam, op, whichprim, totenergy, ratio);
    }
    if (kmath::isnan(errlo) || kmath::isnan(errhi)) iter = maxiter;
    if (iter >= maxiter) break;
  }
  if (iter >= maxiter) {
    for (int i = 0; i < NV; ++i) pp0out[i] = pp00[i];
    return -1;
  }
  double xmid;
  while (true) {
    iter += 1;
    xmid = 0.5 * (xlo + xhi);
    double errmid = f1d_err(xmid, pp00, dtau, g, gam, op, whichprim, totenergy, ratio);
    if (errmid * errlo > 0.0) {
      xlo = xmid;
      errlo = errmid;
    } else {
      xhi = xmid;
      errhi = errmid;
    }
    if (kmath::isnan(xmid) || kmath::isnan(errmid)) {
      for (int i = 0; i < NV; ++i) pp0out[i] = pp00[i];
      return -1;
    }
    if (!(kmath::fabs(kmath::div((xhi - xlo), xmid)) > conv)) break;
  }
  for (int i = 0; i < NV; ++i) pp0out[i] = pp00[i];
  if (whichprim == PRIM_RAD) {
    pp0out[EE] = xmid;
    pp0out[UU] = totenergy - xmid * ratio;
  } else {
    pp0out[UU] = xmid;
    pp0out[EE] = kmath::div((totenergy - xmid), ratio);
  }
  return 0;
}

// one-sided FD step of Jacobian column j (implicit.zig:586)
KC_HD double fd_del(int j, double sign, const double ppp[NV], int sh, double eps, const Geom& g) {
  if (j == 0) return sign * eps * ppp[sh];
  double veleps = eps * my_sign(ppp[j + sh]) * kmath::fmax(kmath::div(1.0e-8, kmath::sqrt(g.gg[j][j])), kmath::fabs(ppp[j + sh]));
  return (ppp[j + sh] >= 0.0) ? sign * veleps : -sign * veleps;
}

KC_HD void lag_opac(RadState& st, const RadState& st00) {
  st.kappaes = st00.kappaes;
  st.opac.gas_abs = st00.opac.gas_abs;
  st.opac.rad_abs = st00.opac.rad_abs;
  st.opac.gas_num = st00.opac.gas_num;
  st.opac.rad_num = st00.opac.rad_num;
  st.opac.gas_ross = st00.opac.gas_ross;
  st.opac.rad_ross = st00.opac.rad_ross;
}

// The loop state of the Newton core at the top of an iteration: what a paused
// solve (RESUME) carries to its next call. iter = iterations done, 0 = not started.
struct CoreCarry {
  double uu[NV], pp[NV];
  RadState state;
  int fret, iter;
};
// C solve_implicit_lab_4dprim Newton core (implicit.zig:642). Returns 1 on
// success (pp_out written, *iters set), 0 on failure.
// RESUME = false is the reference's core as is. RESUME = true starts from
// *carry when carry->iter > 0, runs at most `budget` iterations and then, if the
// solve has not ended, saves its loop state to *carry and returns 2; the
// iterations run are those of the uninterrupted core, so a solve split over
// several calls ends exactly as it would in one.
template <bool RESUME>
KC_HDN int solve_4dprim_core_t(const double uu00[NV], const RadState& state00, const double pp0in[NV], const Geom& g,
                               double dt, double gam, const RadParams& rad, const OpacParams& op, double opdamp,
                               const ImplicitParams& ip, int whichprim, int whicheq, int whichframe, double pp_out[NV],
                               int* iters_out, CoreCarry* carry, int budget) {
  double uu[NV], pp[NV];
  int sh = (whichprim == PRIM_MHD) ? UU : EE;
  double conv = (whicheq == EQ_ENTROPY) ? ip.entrconv : ip.conv;
  bool slim = whicheq != EQ_ENTROPY;
  int fret, iter;
  RadState state;
  if (RESUME && carry->iter > 0) {
    for (int i = 0; i < NV; ++i) {
      uu[i] = carry->uu[i];
      pp[i] = carry->pp[i];
    }
    state = carry->state;
    fret = carry->fret;
    iter = carry->iter;
  } else {
    for (int i = 0; i < NV; ++i) {
      uu[i] = uu00[i];
      pp[i] = pp0in[i];
    }
    fret = apply_constraints(pp, uu, uu00, g, gam, rad, ip, whichprim);
    fill_rad_state(pp, g, gam, op, !slim, state);
    if (ip.lag_opac) lag_opac(state, state00);
    iter = 0;
  }
  const int stop = RESUME ? iter + budget : 0;
  double f1[4], f2[4], jac[4][4];
  bool failed = false;
  bool success = false;
  while (true) {
    if (RESUME && iter >= stop) {
      for (int i = 0; i < NV; ++i) {
        carry->uu[i] = uu[i];
        carry->pp[i] = pp[i];
      }
      carry->state = state;
      carry->fret = fret;
      carry->iter = iter;
      return 2;
    }
    iter += 1;
    double ppp[NV];
    for (int i = 0; i < NV; ++i) ppp[i] = pp[i];
    double xxx[4];
    if (fret < -1) return 0;
    double errbase = implicit_residual(uu, pp, state, uu00, state00, dt, g, op, opdamp, whichprim, whicheq, whichframe, f1);
    if (errbase < conv) {
      success = true;
      break;
    }
    KC_ROLLED
    for (int j = 0; j < 4; ++j) {
      double sign = -1.0;
      while (true) {
        double del = fd_del(j, sign, ppp, sh, ip.eps, g);
        pp[j + sh] = ppp[j + sh] + del;
        fret = apply_constraints(pp, uu, uu00, g, gam, rad, ip, whichprim);
        if (fret < -1) {
          if (sign > 0.0) {
            failed = true;
            break;
          }
          pp[j + sh] = ppp[j + sh];
          sign *= -1.0;
          continue;
        }
        fill_rad_state(pp, g, gam, op, !slim, state);
        if (ip.lag_opac) lag_opac(state, state00);
        implicit_residual(uu, pp, state, uu00, state00, dt, g, op, opdamp, whichprim, whicheq, whichframe, f2);
        for (int i = 0; i < 4; ++i) jac[i][j] = kmath::div((f2[i] - f1[i]), del);
        pp[j + sh] = ppp[j + sh];
        break;
      }
      if (failed) break;
    }
    if (failed) break;
    double scalevec[4] = {pp[sh], 1.0, 1.0, 1.0};
    double invscalevec[4];
    if (ip.scale_jacobian) {
      for (int j = 0; j < 4; ++j) {
        if (scalevec[j] == 0.0) scalevec[j] = 1.0;
        invscalevec[j] = kmath::div(1.0, scalevec[j]);
      }
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
          if (i != j) jac[i][j] = jac[i][j] * (scalevec[j] * invscalevec[i]);
    }
    double ijac[4][4];
    invert4(jac, ijac);
    double xiapp = 1.0;
    while (true) {
      for (int k = 0; k < 4; ++k) xxx[k] = ppp[k + sh];
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
          if (ip.scale_jacobian) xxx[i] -= xiapp * (ijac[i][j] * scalevec[i] * invscalevec[j]) * f1[j];
          else xxx[i] -= xiapp * ijac[i][j] * f1[j];
        }
      for (int k = 0; k < 4; ++k) pp[k + sh] = xxx[k];
      fret = apply_constraints(pp, uu, uu00, g, gam, rad, ip, whichprim);
      fill_rad_state(pp, g, gam, op, !slim, state);
      if (ip.lag_opac) lag_opac(state, state00);
      bool okcheck = false;
      double edenmin = kmath::div(ppp[sh], ip.max_en_change_down);
      double edenmax = ppp[sh] * ip.max_en_change_up;
      if (xxx[0] > edenmin && xxx[0] < edenmax && fret >= -1) okcheck = true;
      double tgasold = t_from_urho(op.c, ppp[UU], ppp[RHO], gam);
      double tgasnew = t_from_urho(op.c, pp[UU], pp[RHO], gam);
      if (okcheck && (tgasnew > tgasold * ip.max_tgas_change || tgasnew < kmath::div(tgasold, ip.max_tgas_change))) okcheck = false;
      double tradnew = lte_T_from_E(op.c, pp[EE]);
      double tradold = lte_T_from_E(op.c, ppp[EE]);
      if (okcheck && (tradnew > tradold * ip.max_trad_change || tradnew < kmath::div(tradold, ip.max_trad_change))) okcheck = false;
      if (okcheck) break;
      if (xxx[0] <= 0.0) {
        xiapp *= kmath::div(ppp[sh], (ppp[sh] + kmath::fabs(xxx[0])));
        xiapp *= 1.0e-1;
      } else {
        xiapp /= ip.damping_factor;
      }
      // !(x >= m) is x < m for every number and also true for NaN: a NaN
      // damping factor (a NaN start state) fails the rung instead of looping
      if (!(xiapp >= ip.max_damping)) {
        failed = true;
        break;
      }
    }
    if (!failed) {
      double f3[4];
      f3[0] = kmath::fabs(kmath::div((pp[sh] - ppp[sh]), ppp[sh]));
      for (int i = 1; i < 4; ++i) {
        f3[i] = pp[i + sh] - ppp[i + sh];
        f3[i] = kmath::fabs(kmath::div(f3[i], kmath::fmax(ip.eps, kmath::fabs(ppp[i + sh]))));
      }
      double convrel = (whicheq == EQ_ENTROPY) ? ip.convrelentr : ip.convrel;
      double convrelerr = (whicheq == EQ_ENTROPY) ? ip.convrelentrerr : ip.convrelerr;
      bool convrelcheck = true;
      for (int ib = 0; ib < 4; ++ib) {
        if (f3[ib] > convrel) {
          convrelcheck = false;
          break;
        }
      }
      if (convrelcheck || errbase <= convrelerr) {
        success = true;
        break;
      }
    }
    if (iter > ip.maxiter || failed) break;
  }
  if (!success) return 0;
  if (iter > ip.maxiter) return 0;
  for (int i = 0; i < NV; ++i) pp_out[i] = pp[i];
  *iters_out = iter;
  return 1;
}
// the reference's core (koral/solve/implicit.zig:642): 1 on success (pp_out,
// *iters_out written), 0 on failure
KC_HD int solve_4dprim_core(const double uu00[NV], const RadState& state00, const double pp0in[NV], const Geom& g,
                            double dt, double gam, const RadParams& rad, const OpacParams& op, double opdamp,
                            const ImplicitParams& ip, int whichprim, int whicheq, int whichframe, double pp_out[NV],
                            int* iters_out) {
  return solve_4dprim_core_t<false>(uu00, state00, pp0in, g, dt, gam, rad, op, opdamp, ip, whichprim, whicheq,
                                    whichframe, pp_out, iters_out, nullptr, 0);
}

// The per-solve preamble of C solve_implicit_lab (implicit.zig:927-961): the
// reference conserveds uu00, the full reference fill state00, the bisection
// warm start pp0 and the starting fluid. Split out so the batched solver can
// run it once and keep it resident across rung retries.
struct ImplicitPre {
  double uu00[NV];
  double pp0[NV];
  RadState state00;
  int startwith;
};
KC_HD void implicit_prepare(const double pp00[NV], const Geom& g, double dt, double gam, const OpacParams& op,
                            const ImplicitParams& ip, ImplicitPre& pre) {
  p2u(pp00, pre.uu00, g, gam);
  double ehat = -calc_ff_rtt(pp00, g, nullptr);
  fill_rad_state(pp00, g, gam, op, true, pre.state00);
  for (int i = 0; i < NV; ++i) pre.pp0[i] = pp00[i];
  if (ip.start_with_bisect) solve_1d_prim(pp00, pre.state00, g, dt, gam, op, pre.pp0);
  pre.startwith = (ehat < ip.threshold * pp00[UU]) ? PRIM_RAD : PRIM_MHD;
}

// rung table of the full ladder (implicit.zig:963)
KC_HD void implicit_rung(int ir, int startwith, int& p, int& e, int& fr) {
  int swapped = (startwith == PRIM_RAD) ? PRIM_MHD : PRIM_RAD;
  switch (ir) {
    case 0: p = startwith; e = EQ_ENERGY; fr = FRAME_LAB; break;
    case 1: p = startwith; e = EQ_ENERGY; fr = FRAME_FF; break;
    case 2: p = swapped; e = EQ_ENERGY; fr = FRAME_LAB; break;
    case 3: p = swapped; e = EQ_ENERGY; fr = FRAME_FF; break;
    case 4: p = startwith; e = EQ_ENTROPY; fr = FRAME_FF; break;
    default: p = swapped; e = EQ_ENTROPY; fr = FRAME_FF; break;
  }
}

// the rung ladder of solve_implicit_lab (implicit.zig:963) from a prepared
// state: on success pp and uu are overwritten, on failure untouched
KC_HDN ImplicitResult implicit_ladder(double uu[NV], double pp[NV], const Geom& g, double dt, double gam,
                                      const RadParams& rad, const OpacParams& op, const ImplicitParams& ip,
                                      const ImplicitPre& pre) {
  ImplicitResult res;
  res.ok = 0;
  res.rung = -1;
  res.iters = 0;
  res.whichprim = PRIM_RAD;
  res.whicheq = EQ_ENERGY;
  res.whichframe = FRAME_LAB;
  for (int level = 0; level <= ip.opdamp_maxlevels; ++level) {
    double od = 1.0;  // the level's opdamp (implicit.zig:955)
    for (int i = 0; i < level; ++i) od /= ip.opdamp_factor;
    KC_ROLLED
    for (int ir = 0; ir < 6; ++ir) {
      int p, e, fr;
      implicit_rung(ir, pre.startwith, p, e, fr);
      double ppw[NV];
      int iters = 0;
      if (solve_4dprim_core(pre.uu00, pre.state00, pre.pp0, g, dt, gam, rad, op, od, ip, p, e, fr, ppw, &iters)) {
        for (int i = 0; i < NV; ++i) pp[i] = ppw[i];
        p2u(ppw, uu, g, gam);
        res.ok = 1;
        res.rung = ir;
        res.iters = iters;
        res.whichprim = p;
        res.whicheq = e;
        res.whichframe = fr;
        return res;
      }
    }
  }
  return res;
}

// C solve_implicit_lab (implicit.zig:927) — the rung ladder; on success pp
// and uu are overwritten, on failure untouched.
KC_HDN ImplicitResult solve_implicit_lab(double uu[NV], double pp[NV], const Geom& g, double dt, double gam,
                                         const RadParams& rad, const OpacParams& op, const ImplicitParams& ip) {
  ImplicitPre pre;
  implicit_prepare(pp, g, dt, gam, op, ip, pre);
  return implicit_ladder(uu, pp, g, dt, gam, rad, op, ip, pre);
}

// The first-rung residual the Newton core evaluates at a start state before
// its first Jacobian (the opening of solve_4dprim_core: constraints, state
// fill, residual) and the constrained start in pp; +inf when the constraints
// reject the start.
KC_HD double implicit_start_residual(const double uu00[NV], const RadState& state00, const double start[NV],
                                     const Geom& g, double dt, double gam, const RadParams& rad,
                                     const OpacParams& op, double opdamp, const ImplicitParams& ip, int whichprim,
                                     double pp[NV]) {
  double uu[NV], f[4];
  for (int i = 0; i < NV; ++i) {
    uu[i] = uu00[i];
    pp[i] = start[i];
  }
  if (apply_constraints(pp, uu, uu00, g, gam, rad, ip, whichprim) < -1) return 1.0e300;
  RadState st;
  fill_rad_state(pp, g, gam, op, false, st);
  if (ip.lag_opac) lag_opac(st, state00);
  return implicit_residual(uu, pp, st, uu00, state00, dt, g, op, opdamp, whichprim, EQ_ENERGY, FRAME_LAB, f);
}

// The opening of rung 0 of the ladder (level 0, start fluid, energy equation,
// lab frame) from a prepared state: returns 1 when the core's first exit is
// taken there (first residual below conv), with pp and uu finished exactly as
// implicit_ladder finishes them (the core's iteration count is then 1), else 0
// with pp and uu untouched. The split form of the implicit pass runs this for
// every cell and the full ladder only for the cells it leaves.
KC_HDN int implicit_first_exit(double uu[NV], double pp[NV], const Geom& g, double dt, double gam,
                               const RadParams& rad, const OpacParams& op, const ImplicitParams& ip,
                               const ImplicitPre& pre) {
  int p, e, fr;
  implicit_rung(0, pre.startwith, p, e, fr);
  double pc[NV];
  double e0 = implicit_start_residual(pre.uu00, pre.state00, pre.pp0, g, dt, gam, rad, op, 1.0, ip, p, pc);
  if (!(e0 < ip.conv)) return 0;
  for (int i = 0; i < NV; ++i) pp[i] = pc[i];
  p2u(pc, uu, g, gam);
  return 1;
}

// The same ladder started from a learned state in place of the bisection warm
// start (the learned-guess form; it has no counterpart in the reference).
// The start fluid is decided as solve_implicit_lab decides it. A cell the
// pre-solve state already satisfies (first-rung residual below conv, the
// core's first exit) is finished there, as the core would finish it, so a
// prediction error never costs such a cell an iteration; the others run the
// ladder from whichever of the pre-solve and the learned state has the
// smaller first-rung residual (starting every such cell from the learned
// state measured slower: the prediction is worse than the pre-solve state for
// a part of them).
// The learned start's preamble: the reference conserveds and state of the
// pre-solve primitives, the start fluid, and the core's first exit on rung 0
// (lab frame, energy equation) at the pre-solve state; returns 1 when that exit
// is taken (uu, pp written), else 0 with pre.pp0 the one of the pre-solve and
// the learned state that has the smaller rung-0 first residual.
KC_HDN int implicit_prepare_from(double uu[NV], double pp[NV], const Geom& g, double dt, double gam,
                                 const RadParams& rad, const OpacParams& op, const ImplicitParams& ip,
                                 const double guess[NV], ImplicitPre& pre) {
  p2u(pp, pre.uu00, g, gam);
  double ehat = -calc_ff_rtt(pp, g, nullptr);
  fill_rad_state(pp, g, gam, op, true, pre.state00);
  pre.startwith = (ehat < ip.threshold * pp[UU]) ? PRIM_RAD : PRIM_MHD;
  double pc[NV];
  double e0 = implicit_start_residual(pre.uu00, pre.state00, pp, g, dt, gam, rad, op, 1.0, ip, pre.startwith, pc);
  if (e0 < ip.conv) {
    for (int i = 0; i < NV; ++i) pp[i] = pc[i];
    p2u(pc, uu, g, gam);
    return 1;
  }
  double e1 = implicit_start_residual(pre.uu00, pre.state00, guess, g, dt, gam, rad, op, 1.0, ip, pre.startwith, pc);
  bool learned = e1 < e0;
  for (int i = 0; i < NV; ++i) pre.pp0[i] = learned ? guess[i] : pp[i];
  return 0;
}
// the result of the core's first exit on rung 0
KC_HD ImplicitResult implicit_first_exit_result(int startwith) {
  ImplicitResult res;
  res.ok = 1;
  res.rung = 0;
  res.iters = 1;
  res.whichprim = startwith;
  res.whicheq = EQ_ENERGY;
  res.whichframe = FRAME_LAB;
  return res;
}
KC_HDN ImplicitResult solve_implicit_lab_from(double uu[NV], double pp[NV], const Geom& g, double dt, double gam,
                                              const RadParams& rad, const OpacParams& op, const ImplicitParams& ip,
                                              const double guess[NV]) {
  ImplicitPre pre;
  if (implicit_prepare_from(uu, pp, g, dt, gam, rad, op, ip, guess, pre)) return implicit_first_exit_result(pre.startwith);
  return implicit_ladder(uu, pp, g, dt, gam, rad, op, ip, pre);
}

}  // namespace kp
