// orc_golden.cpp — TEST INFRASTRUCTURE (the CPU oracle), not product code.
//
// Runs the shared per-point restatement (include/koral/*.h) on the input side
// of the reference's per-function golden records (KGLD, produced by
// koral-zig's oracle/harness_*.c from C KORAL) and writes the outputs in the
// record's own output layout, so the tests compare them with the reference
// tolerances of koral/tests/golden/*_golden_tests.zig. Only tests/ loads this.
#include <string.h>

#include "../include/koral/kparams.h"
#include "../include/koral/kmetric.h"

using namespace kp;

namespace {

// koral/testing/golden.zig:226 (sym10) + :241 (geomFromRecord)
void geom_from_record(const double* v, int len, Geom& g) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 5; ++j) {
      g.gg[i][j] = 0.0;
      g.GG[i][j] = 0.0;
    }
  int n = 0;
  for (int i = 0; i < 4; ++i)
    for (int j = i; j < 4; ++j) {
      g.gg[i][j] = v[n];
      g.gg[j][i] = v[n];
      g.GG[i][j] = v[10 + n];
      g.GG[j][i] = v[10 + n];
      ++n;
    }
  g.gdet = (len >= 23) ? v[20] : 1.0;
  g.gttpert = (len >= 23) ? v[22] : 0.0;
  g.alpha = (len >= 23) ? v[21] : kmath::sqrt(-1.0 / g.GG[0][0]);
  for (int i = 0; i < 4; ++i) g.xx[i] = 0.0;
}

const double kGam = 5.0 / 3.0;

}  // namespace

extern "C" int orc_golden(const char* name, long nrec, const double* in, int nin, double* out, int nout) {
  const FloorParams fl = floor_params_puffy();
  const RadParams rp = rad_params_puffy();
  const OpacParams op = opac_params_puffy(10.0);
  const ImplicitParams ip = implicit_params_puffy();
  for (long r = 0; r < nrec; ++r) {
    const double* a = in + r * nin;
    double* o = out + r * nout;
    Geom g;
    if (!strcmp(name, "p2u")) {
      geom_from_record(a, 23, g);
      double uu[NV];
      p2u(a + 23, uu, g, kGam);
      for (int i = 0; i < NV; ++i) o[i] = uu[i];
    } else if (!strcmp(name, "u2p_solver")) {
      geom_from_record(a, 23, g);
      double pp[NV];
      for (int i = 0; i < NV; ++i) pp[i] = a[36 + i];
      o[0] = u2p_solver_w(a + 23, pp, g, ETYPE_HOT, kGam);
      for (int i = 0; i < 9; ++i) o[1 + i] = pp[i];
      for (int i = 0; i < NV; ++i) pp[i] = a[36 + i];
      o[10] = u2p_solver_w(a + 23, pp, g, ETYPE_ENTROPY, kGam);
      for (int i = 0; i < 9; ++i) o[11 + i] = pp[i];
    } else if (!strcmp(name, "u2p_cascade")) {
      // geom23 uu13 pp13 -> pp13 entropy_used hd_fixup rad_fixup: one cell of
      // calcU2p's inversion (koral/sim.zig:972-994)
      geom_from_record(a, 23, g);
      double uu[NV], pp[NV];
      for (int i = 0; i < NV; ++i) {
        uu[i] = a[23 + i];
        pp[i] = a[36 + i];
      }
      U2pMhdRes res = u2p_mhd(uu, pp, g, kGam, fl);
      U2pRadRes rr = u2p_rad(uu, pp, g, rp);
      int guards = 0;
      check_floors_mhd(pp, g, kGam, fl, guards);
      check_floors_rad(pp, g, rp);
      for (int i = 0; i < NV; ++i) o[i] = pp[i];
      o[13] = res.entropy_used;
      o[14] = res.fixup;
      o[15] = rr.corrected ? -1 : 0;
    } else if (!strcmp(name, "floors")) {
      geom_from_record(a, 23, g);
      double pp[NV];
      for (int i = 0; i < NV; ++i) pp[i] = a[23 + i];
      int guards = 0;
      o[0] = check_floors_mhd(pp, g, kGam, fl, guards);
      for (int i = 0; i < NV; ++i) o[1 + i] = pp[i];
    } else if (!strcmp(name, "physics_tij")) {
      geom_from_record(a, 20, g);
      const double* pp = a + 20;
      double t[4][4], ucon[4], ucov[4], bcon[4], bcov[4], bsq;
      calc_tij(pp, g, kGam, t);
      ucon_ucov_from_prims(pp[VX], pp[VY], pp[VZ], g, ucon, ucov);
      double B[3] = {pp[B1], pp[B2], pp[B3]};
      bcon_bcov_bsq(B, ucon, ucov, g, bcon, bcov, bsq);
      int n = 0;
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) o[n++] = t[i][j];
      for (int i = 0; i < 4; ++i) o[n++] = ucon[i];
      for (int i = 0; i < 4; ++i) o[n++] = ucov[i];
      for (int i = 0; i < 4; ++i) o[n++] = bcon[i];
      for (int i = 0; i < 4; ++i) o[n++] = bcov[i];
      o[n++] = bsq;
    } else if (!strcmp(name, "relele_convvels")) {
      geom_from_record(a, 20, g);
      double uin[4] = {0.0, a[22], a[23], a[24]}, uo[4] = {0, 0, 0, 0};
      int e = convert(uin, (int)a[20], (int)a[21], g, RECOMPUTE_UT, uo);
      for (int i = 0; i < 4; ++i) o[i] = e ? kmath::nan() : uo[i];
    } else if (!strcmp(name, "relele_boost")) {
      geom_from_record(a, 20, g);
      double l[4][4], b1[4], b2[4];
      lorentz_lab2ff(a[20], a[21], a[22], g, l);
      boost2_lab2ff(a + 23, a[20], a[21], a[22], g, b1);
      boost2_ff2lab(a + 23, a[20], a[21], a[22], g, b2);
      int n = 0;
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) o[n++] = l[i][j];
      for (int i = 0; i < 4; ++i) o[n++] = b1[i];
      for (int i = 0; i < 4; ++i) o[n++] = b2[i];
    } else if (!strcmp(name, "recon")) {
      int param = (int)a[10];
      int scheme = 2 - param;
      if (scheme < 0) scheme = 0;
      Faces f = reconstruct(scheme, a, a + 5, a[11]);
      o[0] = f.left;
      o[1] = f.right;
    } else if (!strcmp(name, "wavespeed")) {
      geom_from_record(a, 23, g);
      bool act[3] = {true, true, false};
      double aa[6];
      gas_wavespeeds_lr(a + 23, g, kGam, act, aa);
      for (int i = 0; i < 4; ++i) o[i] = aa[i];
    } else if (!strcmp(name, "fluxprime")) {
      geom_from_record(a, 23, g);
      double ff[NV];
      int e = f_flux_prime(a + 24, (int)a[23], g, kGam, ff);
      for (int i = 0; i < NV; ++i) o[i] = e ? kmath::nan() : ff[i];
    } else if (!strcmp(name, "rad_rij")) {
      geom_from_record(a, 20, g);
      double rij[4][4], ucon[4];
      calc_rij(a + 20, g, rij);
      double rtt = calc_ff_rtt(a + 20, g, ucon);
      int n = 0;
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) o[n++] = rij[i][j];
      o[n++] = rtt;
      for (int i = 0; i < 4; ++i) o[n++] = ucon[i];
    } else if (!strcmp(name, "rad_u2prad")) {
      geom_from_record(a, 23, g);
      double uu[NV], pp[NV];
      for (int i = 0; i < NV; ++i) {
        uu[i] = 0.0;
        pp[i] = 0.0;
      }
      for (int i = 0; i < 4; ++i) {
        uu[EE + i] = a[23 + i];
        pp[EE + i] = a[27 + i];
      }
      U2pRadRes res = u2p_rad(uu, pp, g, rp);
      o[0] = res.ret;
      o[1] = res.corrected ? 1.0 : 0.0;
      for (int i = 0; i < 4; ++i) o[2 + i] = pp[EE + i];
    } else if (!strcmp(name, "rad_wavespeeds")) {
      geom_from_record(a, 20, g);
      bool act[3] = {true, true, false};
      double aval[12];
      rad_wavespeeds(a + 20, g, a + 33, act, aval);
      o[0] = aval[0];
      o[1] = aval[1];
      o[2] = aval[2];
      o[3] = aval[3];
      o[4] = aval[6];
      o[5] = aval[7];
      o[6] = aval[8];
      o[7] = aval[9];
    } else if (!strcmp(name, "rad_floors")) {
      geom_from_record(a, 23, g);
      double pp[NV];
      for (int i = 0; i < NV; ++i) pp[i] = a[23 + i];
      o[0] = check_floors_rad(pp, g, rp);
      for (int i = 0; i < NV; ++i) o[1 + i] = pp[i];
    } else if (!strcmp(name, "rad_thermo")) {
      geom_from_record(a, 23, g);
      RadState st;
      fill_rad_state(a + 23, g, kGam, op, true, st);
      o[0] = st.tgas;
      o[1] = st.te;
      o[2] = st.ne;
      o[3] = st.ehat;
      o[4] = st.tradbb;
      o[5] = st.kappaes;
      o[6] = st.opac.gas_abs;
      o[7] = st.opac.rad_abs;
      o[8] = st.opac.gas_num;
      o[9] = st.opac.rad_num;
      o[10] = st.opac.gas_ross;
      o[11] = st.opac.rad_ross;
      o[12] = st.kappa;
    } else if (!strcmp(name, "rad_opac")) {
      geom_from_record(a, 23, g);
      RadState st;
      fill_rad_state(a + 23, g, kGam, op, true, st);
      double kes = calc_kappaes_standalone(a + 23, kGam, op);
      o[0] = st.kappa;
      o[1] = kes;
      o[2] = st.kappa + kes;
    } else if (!strcmp(name, "rad_gi")) {
      geom_from_record(a, 23, g);
      const double* pp = a + 23;
      RadState st;
      fill_rad_state(pp, g, kGam, op, true, st);
      double giff[4], gilab[4];
      calc_gi_from_state(st, pp[VX], pp[VY], pp[VZ], g, op, true, giff, gilab);
      for (int i = 0; i < 4; ++i) {
        o[i] = gilab[i];
        o[4 + i] = giff[i];
      }
      // the test's force scale (koral/tests/golden/opac_golden_tests.zig:108)
      RadState sens = st;
      sens.trad = 2.0 * st.te;
      double b = op.c.sigma_rad_over_pi * st.te * st.te * st.te * st.te;
      if (nout > 8)
        o[8] = (st.opac.rad_ross + st.kappaes) * st.ehat + st.opac.gas_abs * op.c.fourpi * b +
               kmath::fabs(compton_gi_coeff(op.c, sens));
    } else if (!strcmp(name, "rad_implicit")) {
      geom_from_record(a, 23, g);
      double dt = a[23];
      double pp[NV], uu[NV];
      for (int i = 0; i < NV; ++i) pp[i] = a[24 + i];
      ImplicitResult res = solve_implicit_lab(uu, pp, g, dt, kGam, rp, op, ip);
      o[0] = res.ok ? 0.0 : -1.0;
      o[1] = res.whichprim;
      o[2] = res.whicheq;
      o[3] = res.whichframe;
      o[4] = res.iters;
      for (int i = 0; i < NV; ++i) o[5 + i] = pp[i];
      if (nout > 18) o[18] = res.rung;
    } else if (!strcmp(name, "implicit_resid")) {
      // in: geom23 dt pp00[13] cand[13] prim eq frame -> err
      // (koral/tests/golden/implicit_golden_tests.zig:33 trueResidual)
      geom_from_record(a, 23, g);
      double dt = a[23];
      const double* pp00 = a + 24;
      const double* cand = a + 37;
      double uu00[NV], uux[NV], f[4];
      RadState st00, stx;
      p2u(pp00, uu00, g, kGam);
      fill_rad_state(pp00, g, kGam, op, true, st00);
      p2u(cand, uux, g, kGam);
      fill_rad_state(cand, g, kGam, op, true, stx);
      o[0] = implicit_residual(uux, cand, stx, uu00, st00, dt, g, op, op.opdamp, (int)a[50], (int)a[51], (int)a[52], f);
    } else if (!strcmp(name, "metric_points")) {
      // coords, x0..x3 -> gg16 GG16 gdet dlgdet3 Kr64 gttpert
      int id = (int)a[0];
      int co = id == 1 ? BL : id == 2 ? KS : id == 4 ? MINK : MKS2;
      MetricParams mp = {0.0, 0.1, 0.9};
      CoordData d;
      metric_compute(co, mp, a + 1, d);
      int n = 0;
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) o[n++] = d.gcov[i][j];
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) o[n++] = d.gcon[i][j];
      o[n++] = d.gdet;
      for (int i = 0; i < 3; ++i) o[n++] = d.dlgdet[i];
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
          for (int k = 0; k < 4; ++k) o[n++] = d.kris[i][j][k];
      o[n++] = d.gttpert;
    } else if (!strcmp(name, "coco_dxdx")) {
      auto cid = [](double v) { int id = (int)v; return id == 1 ? BL : id == 2 ? KS : id == 4 ? MINK : MKS2; };
      MetricParams mp = {0.0, 0.1, 0.9};
      int from = cid(a[0]), to = cid(a[1]);
      double y[4], m[4][4];
      coco_full(a + 2, from, to, mp, y);
      dxdx(a + 2, from, to, mp, m);
      for (int i = 0; i < 4; ++i) o[i] = y[i];
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) o[4 + i * 4 + j] = m[i][j];
    } else if (!strcmp(name, "frames_transpall")) {
      // trans_pall_coco between the record's coordinate systems
      // (koral/frames.zig:300 transPallCoco, state_golden_tests.zig:94): in =
      // from, to, x1..x3, pp[13], geometry of `from` (20), of `to` (20)
      auto cid = [](double v) { int id = (int)v; return id == 1 ? BL : id == 2 ? KS : id == 4 ? MINK : MKS2; };
      MetricParams mp = {0.0, 0.1, 0.9};
      int from = cid(a[0]), to = cid(a[1]);
      double x[4] = {0.0, a[2], a[3], a[4]};
      Geom g1, g2;
      geom_from_record(a + 18, 20, g1);
      for (int i = 0; i < 4; ++i) g1.xx[i] = x[i];
      geom_from_record(a + 38, 20, g2);
      double pp[NV], jac[4][4];
      for (int i = 0; i < NV; ++i) pp[i] = a[5 + i];
      dxdx(x, from, to, mp, jac);
      int e = from == to ? 0 : trans_pmhd_coco_j(pp, g1, g2, jac, pp);
      if (!e && from != to) e = trans_prad_coco_j(pp, g1, g2, jac, pp);
      for (int i = 0; i < NV; ++i) o[i] = e ? kmath::nan() : pp[i];
    } else if (!strcmp(name, "krzysie_grid")) {
      // PUFFY 384x360 grid (koral/tests/golden/metric_golden_tests.zig:133)
      MetricParams mp = {0.0, 0.1, 0.9};
      Grid gr = grid_init(384, 360, 1, 3, kmath::log(1.85 - 0.1), kmath::log(500.0 - 0.1), 0.001, 1.0 - 0.001,
                          -KP_PI / 4.0, KP_PI / 4.0);
      long ix = (long)a[0], iy = (long)a[1];
      o[0] = grid_xc(gr, ix);
      o[1] = grid_yc(gr, iy);
      double x[4] = {0.0, grid_xc(gr, ix), grid_yc(gr, iy), grid_zc(gr, 0)};
      CoordData d;
      metric_compute(MKS2, mp, x, d);
      apply_kris_correction(MKS2, mp, gr, d, ix, iy, 0);
      int n = 2;
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
          for (int k = 0; k < 4; ++k) o[n++] = d.kris[i][j][k];
    } else {
      return -1;
    }
  }
  return 0;
}

// solveImplicitLab over n independent cells on `nthreads` host threads, cells
// handed out in chunks from an atomic ticket (the scheme of the reference's
// tools/bench_implicit.zig:53-94). geom23 as the golden records; pp in/out;
// res per cell {ok, rung, iters}. The CPU baseline of the implicit microbench.
#include <atomic>
#include <thread>
#include <vector>
extern "C" int orc_implicit_batch_mt(long n, const double* geom23, const double* dt, double* pp, int* res,
                                     int nthreads) {
  const RadParams rp = rad_params_puffy();
  const OpacParams op = opac_params_puffy(10.0);
  const ImplicitParams ip = implicit_params_puffy();
  std::atomic<long> next(0);
  const long chunk = 64;
  auto work = [&]() {
    for (long c0 = next.fetch_add(chunk); c0 < n; c0 = next.fetch_add(chunk)) {
      for (long c = c0; c < n && c < c0 + chunk; ++c) {
        Geom g;
        geom_from_record(geom23 + c * 23, 23, g);
        double uu[NV];
        ImplicitResult r = solve_implicit_lab(uu, pp + c * NV, g, dt[c], kGam, rp, op, ip);
        res[c * 3 + 0] = r.ok;
        res[c * 3 + 1] = r.rung;
        res[c * 3 + 2] = r.iters;
      }
    }
  };
  if (nthreads < 1) nthreads = 1;
  std::vector<std::thread> th;
  for (int t = 0; t < nthreads; ++t) th.emplace_back(work);
  for (auto& t : th) t.join();
  return 0;
}
