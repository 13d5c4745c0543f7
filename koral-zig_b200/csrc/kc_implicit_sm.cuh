// kc_implicit_sm.cuh — the implicit radiation-gas solve of
// koral/solve/implicit.zig:927 (solveImplicitLab: the rung ladder over
// solve4dPrimCore :642, with the 1-D bisection warm start :473) restated as a
// per-lane state machine for a persistent, lane-refilling kernel.
//
// The per-cell arithmetic is exactly that of kp::solve_implicit_lab (the same
// functions, on the same values, in the same order), so results are bit for
// bit identical; only the schedule differs. Every trip of the kernel's loop,
// each lane advances its cell's control flow (cheap, divergent) up to the next
// expensive evaluation, then the whole warp performs one evaluation together:
// a single call site for constraints + fill_rad_state + residual (or the
// bisection's slim fill + four-force). Lanes whose cell is finished take the
// next cell from a global counter at the top of a trip, so uneven iteration
// counts, rung retries and bisection lengths do not leave lanes idle.
#pragma once
#include "kc_dev.cuh"

namespace kc {

using namespace kp;

enum : int { EV_NONE = 0, EV_FILL00, EV_F1D, EV_CF, EV_R, EV_FD };

enum : int {
  S_IDLE = 0,
  S_DONE,  // no more cells for this lane
  S_START,
  S_PREP_FILLED,
  S_B_LO,
  S_B_HI,
  S_B_EXPAND,
  S_B_EXP_LO,
  S_B_EXP_HI,
  S_B_AFTER_EXPAND,
  S_B_BISECT,
  S_B_BIS_POST,
  S_STARTWITH,
  S_RUNG_INIT,
  S_C_INIT_POST,
  S_C_ITER,
  S_C_BASE_POST,
  S_C_FD_TRY,
  S_C_FD_POST,
  S_C_AFTER_FD,
  S_C_DAMP,
  S_C_DAMP_POST,
  S_C_CONV,
  S_C_END,
  S_RUNG_FAIL,
  S_FINISH
};

struct ImpParams {
  double gam;
  RadParams rp;
  OpacParams op;
  ImplicitParams ip;
};

// one lane's solve in flight
struct ImpLane {
  long cell;
  int st;
  Geom g;
  double dt;
  double pp00[NV], uu00[NV], pp0[NV];
  RadState state00, state;
  double ehat_s;
  int startwith;
  // bisection (solve_1d_prim)
  int b_prim, b_iter;
  double b_dtau, b_tot, b_ratio, b_xlo, b_xhi, b_errlo, b_errhi, b_xmid, b_x, b_val;
  // rung ladder
  int level, ir, p, e, fr;
  double od;
  // Newton core (solve_4dprim_core)
  double uu[NV], pp[NV], ppp[NV];
  double f1[4], f2[4], jac[4][4], ijac[4][4], scalevec[4], invscalevec[4], xxx[4];
  int sh, fret, iter, j;
  bool slim, failed, success;
  double conv, sign, del, xiapp, errbase, errx;
  // result
  int ok, rung, iters;
};

// the f1d_err state at L.b_x (implicit.zig:431): the trial pp into L.pp
__device__ __forceinline__ void f1d_setup(ImpLane& L) {
  double ugas, ehat;
  if (L.b_prim == PRIM_RAD) {
    ehat = L.b_x * L.b_ratio;
    ugas = L.b_tot - ehat;
  } else {
    ugas = L.b_x;
    ehat = L.b_tot - ugas;
  }
  for (int i = 0; i < NV; ++i) L.pp[i] = L.pp00[i];
  L.pp[UU] = ugas;
  L.pp[EE] = ehat / L.b_ratio;
}

// The warp-wide evaluation: one call site for every lane's expensive work.
__device__ __noinline__ void imp_eval(ImpLane& L, int kind, const ImpParams& P) {
  if (kind == EV_CF || kind == EV_FD) L.fret = apply_constraints(L.pp, L.uu, L.uu00, L.g, P.gam, P.rp, P.ip, L.p);
  bool gated = kind == EV_FD && L.fret < -1;
  if (kind != EV_NONE && kind != EV_R && !gated) {
    bool full = kind == EV_FILL00 || ((kind == EV_CF || kind == EV_FD) && !L.slim);
    const double* src = kind == EV_FILL00 ? L.pp00 : L.pp;
    RadState& dst = kind == EV_FILL00 ? L.state00 : L.state;
    fill_rad_state(src, L.g, P.gam, P.op, full, dst);  // the state fill does not read the damping
    if ((kind == EV_CF || kind == EV_FD) && P.ip.lag_opac) lag_opac(L.state, L.state00);
  }
  if (kind == EV_F1D) {
    // the return value of f1d_err (implicit.zig:431)
    double giff[4], gilab[4];
    calc_gi_from_state(L.state, L.pp[VX], L.pp[VY], L.pp[VZ], L.g, P.op, false, giff, gilab);
    if (L.b_prim == PRIM_RAD) L.b_val = L.b_x * L.b_ratio - L.pp00[EE] / L.b_ratio + L.b_dtau * giff[0];
    else L.b_val = L.b_x - L.pp00[UU] - L.b_dtau * giff[0];
  }
  if (kind == EV_R || (kind == EV_FD && !gated))
    L.errx = implicit_residual(L.uu, L.pp, L.state, L.uu00, L.state00, L.dt, L.g, P.op, L.od, L.p, L.e, L.fr,
                               kind == EV_R ? L.f1 : L.f2);
}

// Advance one lane's control flow from its state to the next evaluation it
// needs; returns that evaluation's kind (EV_NONE when the lane is idle, done,
// or has just finished a cell).
__device__ __noinline__ int imp_advance(ImpLane& L, const ImpParams& P) {
  const ImplicitParams& ip = P.ip;
  for (;;) {
    switch (L.st) {
      case S_IDLE:
      case S_DONE:
      case S_FINISH:
        return EV_NONE;
      case S_START:
        // implicit_prepare (implicit.zig:927-961)
        p2u(L.pp00, L.uu00, L.g, P.gam);
        L.ehat_s = -calc_ff_rtt(L.pp00, L.g, nullptr);
        L.st = S_PREP_FILLED;
        return EV_FILL00;
      case S_PREP_FILLED: {
        for (int i = 0; i < NV; ++i) L.pp0[i] = L.pp00[i];
        if (!ip.start_with_bisect) {
          L.st = S_STARTWITH;
          break;
        }
        // solve_1d_prim set-up (implicit.zig:473)
        double ehat = L.state00.ehat;
        L.b_dtau = L.dt / L.state00.ucon[0];
        L.b_tot = ehat + L.pp00[UU];
        L.b_prim = (ehat < 1.0e-3 * L.pp00[UU]) ? PRIM_RAD : PRIM_MHD;
        double tgas = L.state00.tgas;
        L.b_ratio = ehat / L.pp00[EE];
        const double fac = 3.0;
        const double fac1 = fac + 1.0;
        double pp_uu = L.pp00[UU];
        double pp_ee = L.pp00[EE];
        if (tgas > 1.0e14) {
          pp_uu = L.pp00[UU] * 1.0e14 / tgas;
          pp_ee = (L.b_tot - pp_uu) / L.b_ratio;
        }
        if (L.b_prim == PRIM_MHD) {
          L.b_xlo = pp_uu / 1.05;
          L.b_xhi = kmath::fmin(pp_uu * 1.05, (pp_uu + fac * L.b_tot) / fac1);
        } else {
          L.b_xlo = pp_ee / 1.05;
          L.b_xhi = kmath::fmin(pp_ee * 1.05, (pp_ee + fac * L.b_tot / L.b_ratio) / fac1);
        }
        L.b_x = L.b_xlo;
        f1d_setup(L);
        L.st = S_B_LO;
        return EV_F1D;
      }
      case S_B_LO:
        L.b_errlo = L.b_val;
        L.b_x = L.b_xhi;
        f1d_setup(L);
        L.st = S_B_HI;
        return EV_F1D;
      case S_B_HI:
        L.b_errhi = L.b_val;
        L.b_iter = 0;
        L.st = S_B_EXPAND;
        break;
      case S_B_EXPAND: {
        if (!(L.b_errlo * L.b_errhi > 0.0)) {
          L.st = S_B_AFTER_EXPAND;
          break;
        }
        const double fac = 3.0;
        const double fac1 = fac + 1.0;
        L.b_iter += 1;
        if (L.b_errlo > 0.0) {
          L.b_xhi = L.b_xlo;
          L.b_errhi = L.b_errlo;
          L.b_xlo /= fac;
          L.b_x = L.b_xlo;
          L.st = S_B_EXP_LO;
        } else {
          L.b_xlo = L.b_xhi;
          L.b_errlo = L.b_errhi;
          if (L.b_prim == PRIM_RAD) L.b_xhi = kmath::fmin(L.b_xhi * fac, (L.b_xhi + fac * L.b_tot / L.b_ratio) / fac1);
          else L.b_xhi = kmath::fmin(L.b_xhi * fac, (L.b_xhi + fac * L.b_tot) / fac1);
          L.b_x = L.b_xhi;
          L.st = S_B_EXP_HI;
        }
        f1d_setup(L);
        return EV_F1D;
      }
      case S_B_EXP_LO:
      case S_B_EXP_HI: {
        if (L.st == S_B_EXP_LO) L.b_errlo = L.b_val;
        else L.b_errhi = L.b_val;
        const int maxiter = 50;
        if (kmath::isnan(L.b_errlo) || kmath::isnan(L.b_errhi)) L.b_iter = maxiter;
        L.st = (L.b_iter >= maxiter) ? S_B_AFTER_EXPAND : S_B_EXPAND;
        break;
      }
      case S_B_AFTER_EXPAND:
        if (L.b_iter >= 50) {
          for (int i = 0; i < NV; ++i) L.pp0[i] = L.pp00[i];
          L.st = S_STARTWITH;
        } else {
          L.st = S_B_BISECT;
        }
        break;
      case S_B_BISECT:
        L.b_iter += 1;
        L.b_xmid = 0.5 * (L.b_xlo + L.b_xhi);
        L.b_x = L.b_xmid;
        f1d_setup(L);
        L.st = S_B_BIS_POST;
        return EV_F1D;
      case S_B_BIS_POST: {
        double errmid = L.b_val;
        if (errmid * L.b_errlo > 0.0) {
          L.b_xlo = L.b_xmid;
          L.b_errlo = errmid;
        } else {
          L.b_xhi = L.b_xmid;
          L.b_errhi = errmid;
        }
        if (kmath::isnan(L.b_xmid) || kmath::isnan(errmid)) {
          for (int i = 0; i < NV; ++i) L.pp0[i] = L.pp00[i];
          L.st = S_STARTWITH;
          break;
        }
        const double conv = 1.0e-3;
        if (!(kmath::fabs((L.b_xhi - L.b_xlo) / L.b_xmid) > conv)) {
          for (int i = 0; i < NV; ++i) L.pp0[i] = L.pp00[i];
          if (L.b_prim == PRIM_RAD) {
            L.pp0[EE] = L.b_xmid;
            L.pp0[UU] = L.b_tot - L.b_xmid * L.b_ratio;
          } else {
            L.pp0[UU] = L.b_xmid;
            L.pp0[EE] = (L.b_tot - L.b_xmid) / L.b_ratio;
          }
          L.st = S_STARTWITH;
        } else {
          L.st = S_B_BISECT;
        }
        break;
      }
      case S_STARTWITH:
        L.startwith = (L.ehat_s < ip.threshold * L.pp00[UU]) ? PRIM_RAD : PRIM_MHD;
        L.level = 0;
        L.ir = 0;
        L.st = S_RUNG_INIT;
        break;
      case S_RUNG_INIT: {
        double od = 1.0;
        for (int i = 0; i < L.level; ++i) od /= ip.opdamp_factor;
        L.od = od;
        implicit_rung(L.ir, L.startwith, L.p, L.e, L.fr);
        for (int i = 0; i < NV; ++i) {
          L.uu[i] = L.uu00[i];
          L.pp[i] = L.pp0[i];
        }
        L.sh = (L.p == PRIM_MHD) ? UU : EE;
        L.conv = (L.e == EQ_ENTROPY) ? ip.entrconv : ip.conv;
        L.slim = L.e != EQ_ENTROPY;
        L.iter = 0;
        L.failed = false;
        L.success = false;
        L.st = S_C_INIT_POST;
        return EV_CF;
      }
      case S_C_INIT_POST:
        L.st = S_C_ITER;
        break;
      case S_C_ITER:
        L.iter += 1;
        for (int i = 0; i < NV; ++i) L.ppp[i] = L.pp[i];
        if (L.fret < -1) {
          L.st = S_RUNG_FAIL;
          break;
        }
        L.st = S_C_BASE_POST;
        return EV_R;
      case S_C_BASE_POST:
        L.errbase = L.errx;
        if (L.errbase < L.conv) {
          L.success = true;
          L.st = S_C_END;
          break;
        }
        L.j = 0;
        L.sign = -1.0;
        L.st = S_C_FD_TRY;
        break;
      case S_C_FD_TRY:
        L.del = fd_del(L.j, L.sign, L.ppp, L.sh, ip.eps, L.g);
        L.pp[L.j + L.sh] = L.ppp[L.j + L.sh] + L.del;
        L.st = S_C_FD_POST;
        return EV_FD;
      case S_C_FD_POST:
        if (L.fret < -1) {
          if (L.sign > 0.0) {
            L.failed = true;
            L.st = S_C_AFTER_FD;
            break;
          }
          L.pp[L.j + L.sh] = L.ppp[L.j + L.sh];
          L.sign *= -1.0;
          L.st = S_C_FD_TRY;
          break;
        }
        for (int i = 0; i < 4; ++i) L.jac[i][L.j] = (L.f2[i] - L.f1[i]) / L.del;
        L.pp[L.j + L.sh] = L.ppp[L.j + L.sh];
        L.j += 1;
        if (L.j < 4) {
          L.sign = -1.0;
          L.st = S_C_FD_TRY;
        } else {
          L.st = S_C_AFTER_FD;
        }
        break;
      case S_C_AFTER_FD:
        if (L.failed) {
          L.st = S_C_END;
          break;
        }
        L.scalevec[0] = L.pp[L.sh];
        L.scalevec[1] = 1.0;
        L.scalevec[2] = 1.0;
        L.scalevec[3] = 1.0;
        if (ip.scale_jacobian) {
          for (int jj = 0; jj < 4; ++jj) {
            if (L.scalevec[jj] == 0.0) L.scalevec[jj] = 1.0;
            L.invscalevec[jj] = 1.0 / L.scalevec[jj];
          }
          for (int i = 0; i < 4; ++i)
            for (int jj = 0; jj < 4; ++jj)
              if (i != jj) L.jac[i][jj] = L.jac[i][jj] * (L.scalevec[jj] * L.invscalevec[i]);
        }
        invert4(L.jac, L.ijac);
        L.xiapp = 1.0;
        L.st = S_C_DAMP;
        break;
      case S_C_DAMP:
        for (int k = 0; k < 4; ++k) L.xxx[k] = L.ppp[k + L.sh];
        for (int i = 0; i < 4; ++i)
          for (int jj = 0; jj < 4; ++jj) {
            if (ip.scale_jacobian) L.xxx[i] -= L.xiapp * (L.ijac[i][jj] * L.scalevec[i] * L.invscalevec[jj]) * L.f1[jj];
            else L.xxx[i] -= L.xiapp * L.ijac[i][jj] * L.f1[jj];
          }
        for (int k = 0; k < 4; ++k) L.pp[k + L.sh] = L.xxx[k];
        L.st = S_C_DAMP_POST;
        return EV_CF;
      case S_C_DAMP_POST: {
        const Consts& c = P.op.c;
        bool okcheck = false;
        double edenmin = L.ppp[L.sh] / ip.max_en_change_down;
        double edenmax = L.ppp[L.sh] * ip.max_en_change_up;
        if (L.xxx[0] > edenmin && L.xxx[0] < edenmax && L.fret >= -1) okcheck = true;
        double tgasold = t_from_urho(c, L.ppp[UU], L.ppp[RHO], P.gam);
        double tgasnew = t_from_urho(c, L.pp[UU], L.pp[RHO], P.gam);
        if (okcheck && (tgasnew > tgasold * ip.max_tgas_change || tgasnew < tgasold / ip.max_tgas_change))
          okcheck = false;
        double tradnew = lte_T_from_E(c, L.pp[EE]);
        double tradold = lte_T_from_E(c, L.ppp[EE]);
        if (okcheck && (tradnew > tradold * ip.max_trad_change || tradnew < tradold / ip.max_trad_change))
          okcheck = false;
        if (okcheck) {
          L.st = S_C_CONV;
          break;
        }
        if (L.xxx[0] <= 0.0) {
          L.xiapp *= L.ppp[L.sh] / (L.ppp[L.sh] + kmath::fabs(L.xxx[0]));
          L.xiapp *= 1.0e-1;
        } else {
          L.xiapp /= ip.damping_factor;
        }
        if (!(L.xiapp >= ip.max_damping)) {  // NaN fails the rung (see solve_4dprim_core)
          L.failed = true;
          L.st = S_C_CONV;
        } else {
          L.st = S_C_DAMP;
        }
        break;
      }
      case S_C_CONV: {
        if (!L.failed) {
          double f3[4];
          f3[0] = kmath::fabs((L.pp[L.sh] - L.ppp[L.sh]) / L.ppp[L.sh]);
          for (int i = 1; i < 4; ++i) {
            f3[i] = L.pp[i + L.sh] - L.ppp[i + L.sh];
            f3[i] = kmath::fabs(f3[i] / kmath::fmax(ip.eps, kmath::fabs(L.ppp[i + L.sh])));
          }
          double convrel = (L.e == EQ_ENTROPY) ? ip.convrelentr : ip.convrel;
          double convrelerr = (L.e == EQ_ENTROPY) ? ip.convrelentrerr : ip.convrelerr;
          bool convrelcheck = true;
          for (int ib = 0; ib < 4; ++ib) {
            if (f3[ib] > convrel) {
              convrelcheck = false;
              break;
            }
          }
          if (convrelcheck || L.errbase <= convrelerr) {
            L.success = true;
            L.st = S_C_END;
            break;
          }
        }
        L.st = (L.iter > ip.maxiter || L.failed) ? S_C_END : S_C_ITER;
        break;
      }
      case S_C_END:
        if (!L.success || L.iter > ip.maxiter) {
          L.st = S_RUNG_FAIL;
          break;
        }
        // solve_implicit_lab success (implicit.zig:990)
        p2u(L.pp, L.uu, L.g, P.gam);
        L.ok = 1;
        L.rung = L.ir;
        L.iters = L.iter;
        L.st = S_FINISH;
        return EV_NONE;
      case S_RUNG_FAIL:
        L.ir += 1;
        if (L.ir >= 6) {
          L.ir = 0;
          L.level += 1;
          if (L.level > ip.opdamp_maxlevels) {
            L.ok = 0;
            L.rung = -1;
            L.iters = 0;
            L.st = S_FINISH;
            return EV_NONE;
          }
        }
        L.st = S_RUNG_INIT;
        break;
      default:
        L.ok = 0;
        L.rung = -1;
        L.iters = 0;
        L.st = S_FINISH;
        return EV_NONE;
    }
  }
}

// The persistent, lane-refilling solve over n cells. Src supplies
// `bool load(long i, ImpLane& L)` (false: nothing to solve, cell skipped) and
// `void store(const ImpLane& L)`; `counter` must start at 0 and is advanced by
// whole warps. Launch with a multiple of 32 threads per block.
template <class Src>
__device__ void imp_persistent(Src& src, long n, unsigned long long* counter, const ImpParams& P) {
  ImpLane L;
  L.st = S_IDLE;
  L.od = 1.0;
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  for (;;) {
    __syncwarp(full);
    unsigned need = __ballot_sync(full, L.st == S_IDLE);
    if (need) {
      int leader = __ffs(need) - 1;
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(need));
      base = __shfl_sync(full, base, leader);
      if (L.st == S_IDLE) {
        unsigned long long mine = base + __popc(need & ((1u << lane) - 1u));
        if (mine < (unsigned long long)n) {
          L.cell = (long)mine;
          L.st = src.load(L.cell, L) ? S_START : S_IDLE;
        } else {
          L.st = S_DONE;
        }
      }
    }
    if (__all_sync(full, L.st == S_DONE)) break;
    int kind = imp_advance(L, P);
    if (L.st == S_FINISH) {
      src.store(L);
      L.st = S_IDLE;
    }
    __syncwarp(full);
    if (kind != EV_NONE) imp_eval(L, kind, P);
  }
}

// The step's implicit operator (sim.zig:1715 opImplicit) as a persistent
// solve: work item i is domain cell (ix, iy, iz) outside the polar band.
struct ImpStepSrc {
  DevState s;
  DevScalars* sc;
  double dt;
  long nx, nyb, y0;
  __device__ bool load(long i, ImpLane& L) {
    long ix = i % nx, q = i / nx, iy = y0 + q % nyb, iz = q / nyb;
    long c = cidx(s.gr, ix, iy, iz);
    L.cell = c;
    load_cell(s.p, s.gr.nc, c, L.pp00);
    geom_cell(s, ix, iy, iz, L.g);
    L.dt = dt;
    return true;
  }
  __device__ void store(const ImpLane& L) {
    long nc = s.gr.nc, c = L.cell;
    if (L.ok) {
      store_cell(s.u, nc, c, L.uu);
      store_cell(s.p, nc, c, L.pp);
      s.flags[5 * nc + c] = 0;
      atomicAdd(&sc->n_iters, (unsigned long long)L.iters);
      atomicAdd(&sc->n_solves, 1ULL);
    } else {
      s.flags[5 * nc + c] = -1;
      atomicAdd(&sc->n_fail, 1ULL);
    }
  }
};

}  // namespace kc
