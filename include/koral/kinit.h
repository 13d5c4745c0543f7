// kinit.h — host-side PUFFY initial primitives (the limotorus of
// Penna+13 with the broken-power-law angular momentum, atmospheres, the LTE
// gas/radiation pressure split, the BL -> MKS2 transform and the A_phi seed).
// Restates koral/problems/puffy/puffy.zig:316-819 and the GK21 quadrature of
// koral/math/quad.zig (QUADPACK dqk21 nodes and weights). The per-(x1,x2)
// profile is computed once and replicated over the phi cells: the metric is
// axisymmetric, so every phi cell of a column gets the same bits. Everything
// here is host-and-device code (KC_HDI): the oracle runs it on the host, the
// engine runs the torus solve one thread per column and the per-cell
// preparation one thread per cell on the device.
#pragma once
#include <stdint.h>

#include "kopts.h"

namespace kcinit {

using namespace kp;

// PUFFY problem constants (puffy.zig:84 Physics defaults, :316 lt)
struct PuffyPhysics {
  double rhoatmmin = 1.0e-24;
  double maxbeta = 1.0 / 20.0;
  double lt_kappa = 6.0e1;
  double atm_tgas = 1.0e10;
  double atm_trad_init = 3.0e5;
  double lt_xi = 0.995, lt_r1 = 20.0, lt_r2 = 350.0, lt_gamma = 4.0 / 3.0, lt_rin = 35.0;
  double mass = 10.0;
};

constexpr double kXacc = 5.0 * 2.220446049250313e-16;  // 5 DBL_EPSILON
constexpr double kPi2 = KP_PI / 2.0;

struct Gd {
  double gdtt, gdtp, gdpp;
};
// tools.c compute_gd (puffy.zig:345)
KC_HDI Gd compute_gd(double r, double th, double a) {
  double ac = a * kmath::cos(th);
  double sigma = ac * ac + r * r;
  double s2 = kmath::sin(th) * kmath::sin(th);
  double tmp = 2.0 * r * s2 / sigma;
  Gd g;
  g.gdtt = -1.0 + 2.0 * r / sigma;
  g.gdtp = -a * tmp;
  g.gdpp = (r * r + a * a * (1.0 + tmp)) * s2;
  return g;
}
// puffy.zig:358 lK
KC_HDI double lK(double r, double a) {
  double curly_f = 1.0 - 2.0 * a / kmath::pow(r, 1.5) + (a / r) * (a / r);
  double curly_g = 1.0 - 2.0 / r + a / kmath::pow(r, 1.5);
  return kmath::sqrt(r) * curly_f / curly_g;
}
KC_HDI double l3d(double lam, double a, double lb1, double lb2, double xi) {
  double arg = lam <= lb1 ? lb1 : (lam >= lb2 ? lb2 : lam);
  return xi * lK(arg, a);
}
// HARM rtbis (puffy.zig:374)
template <class F>
KC_HDI double rtbis(const F& func, double x1, double x2, double xacc) {
  double f = func(x1);
  double fmid = func(x2);
  (void)fmid;
  double dx, rtb;
  if (f < 0.0) {
    dx = x2 - x1;
    rtb = x1;
  } else {
    dx = x1 - x2;
    rtb = x2;
  }
  for (int j = 1; j <= 100; ++j) {
    dx *= 0.5;
    double xmid = rtb + dx;
    fmid = func(xmid);
    if (fmid <= 0.0) rtb = xmid;
    if (kmath::fabs(dx) < xacc || fmid == 0.0) return rtb;
  }
  return 0.0;
}
KC_HDI double lam_bl(double R, const Gd& gd, double a, double lb1, double lb2, double xi) {
  auto f = [&](double lam) {
    double l = l3d(lam, a, lb1, lb2, xi);
    return lam * lam + l * (l * gd.gdtp + gd.gdpp) / (l * gd.gdtt + gd.gdtp);
  };
  return rtbis(f, R, 10.0 * R, kXacc);
}
KC_HDI double omega3d(double l, const Gd& gd) { return -(gd.gdtt * l + gd.gdtp) * (1.0 / (gd.gdpp + gd.gdtp * l)); }
KC_HDI double compute_agrav(double om, const Gd& gd) {
  return kmath::sqrt(kmath::fabs(1.0 / (gd.gdtt + 2.0 * om * gd.gdtp + om * om * gd.gdpp)));
}
KC_HDI double find_rml(double lam, double a, double lb1, double lb2, double xi) {
  double lamsq = lam * lam;
  auto f = [&](double x) {
    Gd gd = compute_gd(x, kPi2, a);
    double lx = lam_bl(x, gd, a, lb1, lb2, xi);
    return lamsq - lx * lx;
  };
  return rtbis(f, 6.0, 10.0 * lamsq, kXacc);
}
// tools.c lnf_integrand (puffy.zig:435)
struct LnfIntegrand {
  double a, lb1, lb2, xi;
  KC_HDI double operator()(double r) const {
    double r2 = r * r, r3 = r2 * r, a2 = a * a;
    Gd gd = compute_gd(r, kPi2, a);
    double lam = lam_bl(r, gd, a, lb1, lb2, xi);
    double lam2 = lam * lam;
    double l = l3d(lam, a, lb1, lb2, xi);
    double term1 = (r - 2.0) * l, term2 = 2.0 * a, term3 = r3 + a2 * (r + 2.0), term4 = term2 * l;
    double om_num = term1 + term2, om_den = term3 - term4;
    double om = om_num / om_den;
    double dl_dr = 0.0;
    if (lam <= lb1 || lam >= lb2) {
      dl_dr = 0.0;
    } else {
      double oneplusx = 1.0 - 2.0 / lam + a * kmath::pow(lam, -1.5);
      double dx_dlam = 2.0 * kmath::pow(lam, -2.0) - 1.5 * a * kmath::pow(lam, -2.5);
      double lamroot = kmath::sqrt(lam);
      double dlk_dlam = (oneplusx * 0.5 * (1.0 / lamroot) + (a - lamroot) * dx_dlam) / (oneplusx * oneplusx);
      double dd = term3 - 2.0 * term4 - lam2 * (r - 2.0);
      double ee = l * (3.0 * r2 + a2 - lam2);
      dl_dr = ee / (2.0 * lam * om_num / (xi * dlk_dlam) - dd);
    }
    double dom_dr = (om_den * (l + (r - 2.0) * dl_dr) - om_num * (3.0 * r2 + a2 + 2.0 * a * dl_dr)) / (om_den * om_den);
    return -l / (1.0 - om * l) * dom_dr;
  }
};

// ---- adaptive Gauss-Kronrod 21 (koral/math/quad.zig; QUADPACK dqk21) --------
template <class F>
KC_HDI void gk21(const F& f, double a, double b, double& value, double& abserr) {
  const double kXgk[11] = {
      0.995657163025808080735527280689003, 0.973906528517171720077964012084452,
      0.930157491355708226001207180059508, 0.865063366688984510732096688423493,
      0.780817726586416897063717578345042, 0.679409568299024406234327365114874,
      0.562757134668604683339000099272694, 0.433395394129247190799265943165784,
      0.294392862701460198131126603103866, 0.148874338981631210884826001129720,
      0.000000000000000000000000000000000};
  const double kWgk[11] = {
      0.011694638867371874278064396062192, 0.032558162307964727478818972459390,
      0.054755896574351996031381300244580, 0.075039674810919952767043140916190,
      0.093125454583697605535065465083366, 0.109387158802297641899210590325805,
      0.123491976262065851077958109831074, 0.134709217311473325928054001771707,
      0.142775938577060080797094273138717, 0.147739104901338491374841515972068,
      0.149445554002916905664936468389821};
  const double kWg[5] = {
      0.066671344308688137593568809893332, 0.149451349150580593145776339657697,
      0.219086362515982043995534934228163, 0.269266719309996355091226921569469,
      0.295524224714752870173892994651338};
  double c = 0.5 * (a + b), h = 0.5 * (b - a);
  double fc = f(c);
  double resg = 0.0, resk = kWgk[10] * fc;
  for (int j = 0; j < 5; ++j) {
    int jtw = 2 * j + 1;
    double x = h * kXgk[jtw];
    double fsum = f(c - x) + f(c + x);
    resg += kWg[j] * fsum;
    resk += kWgk[jtw] * fsum;
  }
  for (int j = 0; j < 5; ++j) {
    int jtw = 2 * j;
    double x = h * kXgk[jtw];
    resk += kWgk[jtw] * (f(c - x) + f(c + x));
  }
  value = resk * h;
  abserr = kmath::fabs((resk - resg) * h);
}
// the segment table of the adaptive quadrature: 4 x kMaxSeg doubles of scratch
constexpr int kMaxSeg = 512;
template <class F>
KC_HDI bool integrate(const F& f, double a, double b, double epsabs, double epsrel, double& out, double* seg) {
  if (a == b) {
    out = 0.0;
    return true;
  }
  const int maxseg = kMaxSeg;
  double *sa = seg, *sb = seg + kMaxSeg, *sv = seg + 2 * kMaxSeg, *se = seg + 3 * kMaxSeg;
  int nseg = 1;
  gk21(f, a, b, sv[0], se[0]);
  sa[0] = a;
  sb[0] = b;
  while (true) {
    double total = 0.0, toterr = 0.0;
    int worst = 0;
    for (int i = 0; i < nseg; ++i) {
      total += sv[i];
      toterr += se[i];
      if (se[i] > se[worst]) worst = i;
    }
    if (toterr <= kmath::fmax(epsabs, epsrel * kmath::fabs(total))) {
      out = total;
      return true;
    }
    if (nseg == maxseg) {
      out = total;
      return false;
    }
    double lo = sa[worst], hi = sb[worst];
    double mid = 0.5 * (lo + hi);
    double lv, le, rv, re;
    gk21(f, lo, mid, lv, le);
    gk21(f, mid, hi, rv, re);
    sa[worst] = lo;
    sb[worst] = mid;
    sv[worst] = lv;
    se[worst] = le;
    sa[nseg] = mid;
    sb[nseg] = hi;
    sv[nseg] = rv;
    se[nseg] = re;
    nseg += 1;
  }
}

struct TorusConsts {
  double lb1, lb2, lamin, lin, omin, agravin;
};
KC_HDI TorusConsts torus_consts(double a, const PuffyPhysics& ph) {
  TorusConsts tc;
  Gd gd = compute_gd(ph.lt_r1, kPi2, a);
  tc.lb1 = lam_bl(ph.lt_r1, gd, a, 0.0, 200000.0, ph.lt_xi);
  gd = compute_gd(ph.lt_r2, kPi2, a);
  tc.lb2 = lam_bl(ph.lt_r2, gd, a, tc.lb1, 200000.0, ph.lt_xi);
  gd = compute_gd(ph.lt_rin, kPi2, a);
  tc.lamin = lam_bl(ph.lt_rin, gd, a, tc.lb1, tc.lb2, ph.lt_xi);
  tc.lin = l3d(tc.lamin, a, tc.lb1, tc.lb2, ph.lt_xi);
  tc.omin = omega3d(tc.lin, gd);
  tc.agravin = compute_agrav(tc.omin, gd);
  return tc;
}
struct DsVels {
  double rho, uu, ell;
};
// tools.c init_dsandvels_limotorus (puffy.zig:572); seg: 4 kMaxSeg doubles
KC_HDI DsVels init_dsandvels_s(double r, double th, double a, const TorusConsts& tc, const PuffyPhysics& ph,
                               double* seg) {
  DsVels o = {-1.0, 0.0, 0.0};
  double R = r * kmath::sin(th);
  if (R < ph.lt_rin) return o;
  Gd gd = compute_gd(r, th, a);
  double lam = lam_bl(R, gd, a, tc.lb1, tc.lb2, ph.lt_xi);
  double l = l3d(lam, a, tc.lb1, tc.lb2, ph.lt_xi);
  double om = omega3d(l, gd);
  double agrav = compute_agrav(om, gd);
  double rml = find_rml(lam, a, tc.lb1, tc.lb2, ph.lt_xi);
  LnfIntegrand integrand = {a, tc.lb1, tc.lb2, ph.lt_xi};
  double q;
  bool conv = integrate(integrand, ph.lt_rin, rml, 0.0, 1.0e-12, q, seg);
  double lnf3d = conv ? q : -kmath::inf();
  double f3d = kmath::exp(-lnf3d);
  const double f3din = 1.0;
  double hh = f3din * agrav / (f3d * tc.agravin);
  double eps = (-1.0 + hh) * (1.0 / ph.lt_gamma);
  double rho = (eps < 0.0) ? -1.0
                           : kmath::pow((-1.0 + ph.lt_gamma) * eps * (1.0 / ph.lt_kappa), 1.0 / (-1.0 + ph.lt_gamma));
  o.rho = rho;
  o.ell = l;
  o.uu = ph.lt_kappa * kmath::pow(rho, ph.lt_gamma) / (ph.lt_gamma - 1.0);
  return o;
}

// the same with the calling host thread's own scratch
inline DsVels init_dsandvels(double r, double th, double a, const TorusConsts& tc, const PuffyPhysics& ph) {
  static thread_local double seg[4 * kMaxSeg];
  return init_dsandvels_s(r, th, a, tc, ph, seg);
}

// prepinit.c T from P = bbb T + aaa T^4 (puffy.zig:660)
KC_HDI double t_from_ptot(double P, double aaa, double bbb) {
  const double third = 0.3333333333333333, twothird = 0.6666666666666666;
  double naw1 = kmath::cbrt(9.0 * aaa * (bbb * bbb) -
                            kmath::sqrt(3.0) * kmath::sqrt(27.0 * (aaa * aaa) * kmath::pow(bbb, 4.0) +
                                                           256.0 * kmath::pow(aaa, 3.0) * kmath::pow(P, 3.0)));
  double c23 = kmath::pow(twothird, third);
  double c2 = kmath::pow(2.0, third);
  double c3 = kmath::pow(3.0, twothird);
  return -kmath::sqrt((-4.0 * c23 * P) / naw1 + naw1 / (c2 * c3 * aaa)) / 2.0 +
         kmath::sqrt((4.0 * c23 * P) / naw1 - naw1 / (c2 * c3 * aaa) +
                     (2.0 * bbb) / (aaa * kmath::sqrt((-4.0 * c23 * P) / naw1 + naw1 / (c2 * c3 * aaa)))) /
             2.0;
}

// splitmix64 finalizer (puffy.zig:684)
KC_HDI uint64_t mix64(uint64_t z) {
  z = z + 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
// decomposition-invariant cell noise in [-1, 1) (puffy.zig:696 perturbXi);
// seed 0 is the reference's field, other seeds mix into the x1 word
KC_HDI double perturb_xi(const double x[4], uint64_t seed) {
  uint64_t b1 = kmath::to_bits(x[1]) ^ seed, b2 = kmath::to_bits(x[2]), b3 = kmath::to_bits(x[3]);
  uint64_t u = mix64(mix64(mix64(b1) ^ b2) ^ b3);
  return 2.0 * ((double)(u >> 11) * 0x1.0p-53) - 1.0;
}

// atmosphere (relele.c:518/718 atmtype 0, puffy.zig:617-650)
KC_HDI void set_atmospheres(double pp[NV], const Geom& geo, const Geom& gbl, double uintatmmin, double eradatmmin,
                            const PuffyPhysics& ph) {
  double ucon[4];
  normal_obs_velr(geo, ucon);
  pp[VX] = ucon[1];
  pp[VY] = ucon[2];
  pp[VZ] = ucon[3];
  double r = gbl.xx[1];
  const double rout = 2.0;
  pp[RHO] = ph.rhoatmmin * kmath::pow(r / rout, -1.5);
  pp[UU] = uintatmmin * kmath::pow(r / rout, -2.5);
  pp[B1] = 0.0;
  pp[B2] = 0.0;
  pp[B3] = 0.0;
  pp[EE] = eradatmmin;
  pp[FX] = ucon[1];
  pp[FY] = ucon[2];
  pp[FZ] = ucon[3];
}

// prepinit.c per-cell initial primitives (puffy.zig:715 prepInitCellWith)
// with the optional interior perturbations; A_phi is left in B3.
KC_HDI int prep_init_cell(const Geom& geo, const Geom& gbl, const double jb2m[4][4], const DsVels& dv,
                          const SimParams& sp, const PuffyPhysics& ph, double perturb, double perturb_rho, uint64_t seed,
                          double pp[NV]) {
  const Consts& con = sp.op.c;
  double uintatmmin = u_from_trho(con, ph.atm_tgas, ph.rhoatmmin, sp.gam);
  double eradatmmin = lte_E_from_T(con, ph.atm_trad_init) / 10.0 * 6.62 / ph.mass;
  double rho = dv.rho;
  double ell = dv.ell;
  for (int i = 0; i < NV; ++i) pp[i] = 0.0;
  if (rho < 0.0) {
    set_atmospheres(pp, geo, gbl, uintatmmin, eradatmmin, ph);
    pp[ENTR] = -1.0;
    return E_OK;
  }
  pp[ENTR] = 1.0;
  double ppback[NV];
  for (int i = 0; i < NV; ++i) ppback[i] = 0.0;
  set_atmospheres(ppback, geo, gbl, uintatmmin, eradatmmin, ph);
  double uint_ = ph.lt_kappa * kmath::pow(rho, ph.lt_gamma) / (ph.lt_gamma - 1.0);
  if (perturb != 0.0) uint_ *= 1.0 + perturb * perturb_xi(geo.xx, seed);
  if (perturb_rho != 0.0) rho *= 1.0 + perturb_rho * perturb_xi(geo.xx, seed ^ 0x5DEECE66DULL);
  ell *= -1.0;
  double ulph = kmath::sqrt(-1.0 / (gbl.GG[0][0] / ell / ell + 2.0 / ell * gbl.GG[0][3] + gbl.GG[3][3]));
  double ult = ulph / ell;
  double ucov[4] = {ult, 0.0, 0.0, ulph}, ucon[4];
  raise_vec(ucov, gbl, ucon);
  int e = convert(ucon, VEL4, VELR, gbl, TRUST_UT, ucon);
  if (e) return e;
  pp[RHO] = kmath::fmax(rho, ppback[RHO]);
  pp[UU] = kmath::fmax(uint_, ppback[UU]);
  pp[VX] = ucon[1];
  pp[VY] = ucon[2];
  pp[VZ] = ucon[3];
  // LTE split P = (gam-1) uint = bbb T + aaa T^4
  double P = (sp.gam - 1.0) * uint_;
  double aaa = con.four_sigmarad / 3.0;
  double bbb = con.kb_over_mugas_mp * rho;
  double t4 = t_from_ptot(P, aaa, bbb);
  double E = lte_E_from_T(con, t4);
  uint_ = u_from_trho(con, t4, rho, sp.gam);
  pp[UU] = kmath::fmax(uint_, ppback[UU]);
  pp[EE] = kmath::fmax(E, ppback[EE]);
  pp[FX] = 0.0;
  pp[FY] = 0.0;
  pp[FZ] = 0.0;
  // prad_ff2lab (radiation.zig:139) in BL
  {
    double rff[4][4], rlab[4][4], rud[4][4];
    calc_rij(pp, gbl, rff);
    boost22_ff2lab(rff, pp[VX], pp[VY], pp[VZ], gbl, rlab);
    lower_second(rlab, gbl, rud);
    double uu[NV];
    for (int i = 0; i < NV; ++i) uu[i] = 0.0;
    double gdetu = gbl.gdet;
    uu[EE] = gdetu * rud[0][0];
    uu[FX] = gdetu * rud[0][1];
    uu[FY] = gdetu * rud[0][2];
    uu[FZ] = gdetu * rud[0][3];
    u2p_rad(uu, pp, gbl, sp.rp);
  }
  // BL -> MKS2 (frames.zig:300 transPallCoco)
  e = trans_pmhd_coco_j(pp, gbl, geo, jb2m, pp);
  if (e) return e;
  e = trans_prad_coco_j(pp, gbl, geo, jb2m, pp);
  if (e) return e;
  // A_phi seed with QUADLOOPS (puffy.zig:808)
  double base = pp[RHO] * gbl.xx[1] / 4.0e-22;
  double acov3 = kmath::fmax(base * base - 0.02, 0.0) * 0x1.bd0d0f57f40b8p-39;  // sqrt(1e-23)
  acov3 *= kmath::sin((KP_PI / 2.0 - gbl.xx[2]) / 0.1);
  pp[B1] = 0.0;
  pp[B2] = 0.0;
  pp[B3] = acov3;
  return E_OK;
}

}  // namespace kcinit
