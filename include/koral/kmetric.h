// kmetric.h — the MKS2/KS/BL metric in forward-mode dual numbers, its
// determinant/inverse/Christoffels, the Christoffel trace correction, the
// coordinate point transforms and Jacobians, and the per-cell/per-face
// geometry blocks the engine caches. Host-side restatement (also device-safe)
// of koral/math/dual.zig, koral/math/linalg.zig, koral/metric/{forms,metric,
// precompute,coco}.zig.
#pragma once
#include "kcore.h"

namespace kp {

struct MetricParams {
  double a, mksr0, mksh0;
};

// ---- Dual(3) (koral/math/dual.zig:26) ---------------------------------------
struct D3 {
  double v, d[3];
};
KC_HD D3 dconst(double x) {
  D3 r;
  r.v = x;
  r.d[0] = r.d[1] = r.d[2] = 0.0;
  return r;
}
KC_HD D3 dvar(double x, int slot) {
  D3 r = dconst(x);
  r.d[slot] = 1.0;
  return r;
}
KC_HD D3 dadd(const D3& a, const D3& b) {
  D3 r;
  r.v = a.v + b.v;
  for (int i = 0; i < 3; ++i) r.d[i] = a.d[i] + b.d[i];
  return r;
}
KC_HD D3 dsub(const D3& a, const D3& b) {
  D3 r;
  r.v = a.v - b.v;
  for (int i = 0; i < 3; ++i) r.d[i] = a.d[i] - b.d[i];
  return r;
}
KC_HD D3 dmul(const D3& a, const D3& b) {
  D3 r;
  r.v = a.v * b.v;
  for (int i = 0; i < 3; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
KC_HD D3 ddiv(const D3& a, const D3& b) {
  double inv = 1.0 / b.v;
  double q = a.v * inv;
  D3 r;
  r.v = q;
  for (int i = 0; i < 3; ++i) r.d[i] = (a.d[i] - q * b.d[i]) * inv;
  return r;
}
KC_HD D3 dscale(const D3& a, double c) {
  D3 r;
  r.v = a.v * c;
  for (int i = 0; i < 3; ++i) r.d[i] = a.d[i] * c;
  return r;
}
KC_HD D3 daddc(const D3& a, double c) {
  D3 r = a;
  r.v = a.v + c;
  return r;
}
KC_HD D3 dsq(const D3& a) { return dmul(a, a); }
KC_HD D3 dchain(const D3& a, double v, double dv) {
  D3 r;
  r.v = v;
  for (int i = 0; i < 3; ++i) r.d[i] = a.d[i] * dv;
  return r;
}
KC_HD D3 dsin(const D3& a) { return dchain(a, kmath::sin(a.v), kmath::cos(a.v)); }
KC_HD D3 dcos(const D3& a) { return dchain(a, kmath::cos(a.v), -kmath::sin(a.v)); }
KC_HD D3 dtan(const D3& a) {
  double t = kmath::tan(a.v);
  return dchain(a, t, 1.0 + t * t);
}
KC_HD D3 dexp(const D3& a) {
  double e = kmath::exp(a.v);
  return dchain(a, e, e);
}

// ---- metric forms (koral/metric/forms.zig) ----------------------------------
// Kerr-Schild (forms.zig:57)
KC_HD void gcov_ks(const D3 x[4], const MetricParams& mp, D3 g[4][4]) {
  double a = mp.a;
  D3 r = x[1];
  D3 sth = dsin(x[2]);
  D3 cth = dcos(x[2]);
  D3 s2 = dsq(sth);
  D3 sigma = dadd(dsq(r), dscale(dsq(cth), a * a));
  D3 two_r_sigma = ddiv(dscale(r, 2.0), sigma);
  D3 one_p = daddc(two_r_sigma, 1.0);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) g[i][j] = dconst(0.0);
  g[0][0] = daddc(two_r_sigma, -1.0);
  g[0][1] = two_r_sigma;
  g[0][3] = ddiv(dscale(dmul(r, s2), -2.0 * a), sigma);
  g[1][1] = one_p;
  g[1][3] = dscale(dmul(one_p, s2), -a);
  g[2][2] = sigma;
  g[3][3] = dmul(s2, dadd(sigma, dscale(dmul(one_p, s2), a * a)));
  g[1][0] = g[0][1];
  g[3][0] = g[0][3];
  g[3][1] = g[1][3];
}
// Boyer-Lindquist (forms.zig:33)
KC_HD void gcov_bl(const D3 x[4], const MetricParams& mp, D3 g[4][4]) {
  double a = mp.a;
  D3 r = x[1];
  D3 sth = dsin(x[2]);
  D3 cth = dcos(x[2]);
  D3 s2 = dsq(sth);
  D3 sigma = dadd(dsq(r), dscale(dsq(cth), a * a));
  D3 delta = daddc(dmul(daddc(r, -2.0), r), a * a);
  D3 two_r_sigma = ddiv(dscale(r, 2.0), sigma);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) g[i][j] = dconst(0.0);
  g[0][0] = daddc(two_r_sigma, -1.0);
  g[0][3] = ddiv(dscale(dmul(r, s2), -2.0 * a), sigma);
  g[1][1] = ddiv(sigma, delta);
  g[2][2] = sigma;
  g[3][3] = dmul(s2, dadd(daddc(dsq(r), a * a), ddiv(dscale(dmul(r, s2), 2.0 * a * a), sigma)));
  g[3][0] = g[0][3];
}

#define KP_PI 3.141592653589793
// cot(pi H0 / 2) (forms.zig:88)
KC_HD double mks2_cot(double h0) { return 1.0 / kmath::tan(0.5 * KP_PI * h0); }
// point-transform flavor theta(x2) (forms.zig:93)
KC_HD D3 mks2_theta(const D3& x2, double h0) {
  D3 u = dscale(daddc(x2, -0.5), h0 * KP_PI);
  return daddc(dscale(dtan(u), 0.5 * KP_PI * mks2_cot(h0)), 0.5 * KP_PI);
}
// metric flavor theta(x2) (forms.zig:100)
KC_HD D3 mks2_theta_metric(const D3& x2, double h0) {
  D3 u = dscale(daddc(x2, -0.5), h0 * KP_PI);
  return dscale(daddc(dscale(dtan(u), mks2_cot(h0)), 1.0), 0.5 * KP_PI);
}
// metric flavor dtheta/dx2 (forms.zig:107)
KC_HD D3 mks2_dtheta_dx2_metric(const D3& x2, double h0) {
  D3 u = dscale(daddc(x2, -0.5), h0 * KP_PI);
  D3 t = dtan(u);
  return dscale(daddc(dsq(t), 1.0), 0.5 * h0 * KP_PI * KP_PI * mks2_cot(h0));
}
// MKS2 = pushforward of KS (forms.zig:122)
KC_HD void gcov_mks2(const D3 x[4], const MetricParams& mp, D3 g[4][4]) {
  D3 j1 = dexp(x[1]);
  D3 r = daddc(j1, mp.mksr0);
  D3 th = mks2_theta_metric(x[2], mp.mksh0);
  D3 j2 = mks2_dtheta_dx2_metric(x[2], mp.mksh0);
  D3 xk[4] = {x[0], r, th, x[3]};
  D3 gks[4][4];
  gcov_ks(xk, mp, gks);
  D3 jf[4] = {dconst(1.0), j1, j2, dconst(1.0)};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) g[i][j] = dmul(dmul(gks[i][j], jf[i]), jf[j]);
}
KC_HD void gcov_dual(int coords, const MetricParams& mp, const double x[4], D3 g[4][4]) {
  D3 xd[4] = {dconst(x[0]), dvar(x[1], 0), dvar(x[2], 1), dvar(x[3], 2)};
  if (coords == MKS2) gcov_mks2(xd, mp, g);
  else if (coords == KS) gcov_ks(xd, mp, g);
  else if (coords == BL) gcov_bl(xd, mp, g);
  else {
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) g[i][j] = dconst(0.0);
    g[0][0] = dconst(-1.0);
    g[1][1] = dconst(1.0);
    g[2][2] = dconst(1.0);
    g[3][3] = dconst(1.0);
  }
}

// ---- 4x4 cofactor det/inverse (koral/math/linalg.zig) ------------------------
KC_HD D3 minor3(const D3 m[4][4], const int r[3], const int c[3]) {
  D3 t0 = dmul(m[r[0]][c[0]], dsub(dmul(m[r[1]][c[1]], m[r[2]][c[2]]), dmul(m[r[1]][c[2]], m[r[2]][c[1]])));
  D3 t1 = dmul(m[r[0]][c[1]], dsub(dmul(m[r[1]][c[0]], m[r[2]][c[2]]), dmul(m[r[1]][c[2]], m[r[2]][c[0]])));
  D3 t2 = dmul(m[r[0]][c[2]], dsub(dmul(m[r[1]][c[0]], m[r[2]][c[1]]), dmul(m[r[1]][c[1]], m[r[2]][c[0]])));
  return dadd(dsub(t0, t1), t2);
}
KC_HD void complement(int i, int c[3]) {
  int n = 0;
  for (int k = 0; k < 4; ++k)
    if (k != i) c[n++] = k;
}
KC_HD D3 det4(const D3 m[4][4]) {
  D3 d = dconst(0.0);
  double sign = 1.0;
  int c0[3];
  complement(0, c0);
  for (int j = 0; j < 4; ++j) {
    int cj[3];
    complement(j, cj);
    D3 mn = minor3(m, c0, cj);
    d = dadd(d, dscale(dmul(m[0][j], mn), sign));
    sign = -sign;
  }
  return d;
}
KC_HD void inv4(const D3 m[4][4], const D3& det, D3 out[4][4]) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      int cj[3], ci[3];
      complement(j, cj);
      complement(i, ci);
      D3 mn = minor3(m, cj, ci);
      double sign = ((i + j) % 2 == 0) ? 1.0 : -1.0;
      out[i][j] = ddiv(dscale(mn, sign), det);
    }
}

// ---- metric assembly (koral/metric/metric.zig) -------------------------------
struct CoordData {
  double gcov[4][4], gcon[4][4];
  double gdet;
  double dlgdet[3];
  double kris[4][4][4];
  double gttpert;
};
KC_HD double r_horizon_bl(double a) { return 1.0 + kmath::sqrt(1.0 - a * a); }
// metric.zig:26 (C r_ISCO_BL)
KC_HD double r_isco_bl(double ac) {
  const double c3 = 1.0 / 3.0;
  double z1 = 1.0 + kmath::pow(1.0 - ac * ac, c3) * (kmath::pow(1.0 + ac, c3) + kmath::pow(1.0 - ac, c3));
  double z2 = kmath::pow(3.0 * ac * ac + z1 * z1, 1.0 / 2.0);
  return 3.0 + z2 - kmath::pow((3.0 - z1) * (3.0 + z1 + 2.0 * z2), 1.0 / 2.0);
}
// metric.zig:146 (C calc_gttpert_arb)
KC_HD double gttpert_at(int coords, const MetricParams& mp, const double x[4]) {
  if (coords == MINK) return 0.0;
  double r, th;
  if (coords == MKS2) {
    r = kmath::exp(x[1]) + mp.mksr0;
    th = mks2_theta(dconst(x[2]), mp.mksh0).v;
  } else {
    r = x[1];
    th = x[2];
  }
  double c = kmath::cos(th);
  return 2.0 * r / (r * r + mp.a * mp.a * c * c);
}
KC_HD double dpart(const D3 g[4][4], int a, int b, int m) { return (m == 0) ? 0.0 : g[a][b].d[m - 1]; }
// metric.zig:75 (compute)
KC_HDN void metric_compute(int coords, const MetricParams& mp, const double x[4], CoordData& out) {
  D3 g[4][4], ginv[4][4];
  gcov_dual(coords, mp, x, g);
  D3 det = det4(g);
  inv4(g, det, ginv);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      out.gcov[i][j] = g[i][j].v;
      out.gcon[i][j] = ginv[i][j].v;
    }
  out.gdet = kmath::sqrt(-det.v);
  for (int i = 0; i < 3; ++i) out.dlgdet[i] = 0.5 * det.d[i] / det.v;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = j; k < 4; ++k) {
        double s = 0.0;
        for (int l = 0; l < 4; ++l) {
          double t = dpart(g, l, k, j) + dpart(g, l, j, k) - dpart(g, j, k, l);
          s += out.gcon[i][l] * t;
        }
        out.kris[i][j][k] = 0.5 * s;
        out.kris[i][k][j] = 0.5 * s;
      }
  out.gttpert = gttpert_at(coords, mp, x);
}
// metric.zig:113 (gdetAt)
KC_HD double gdet_at(int coords, const MetricParams& mp, const double x[4]) {
  D3 g[4][4];
  gcov_dual(coords, mp, x, g);
  return kmath::sqrt(-det4(g).v);
}

// ---- the uniform internal grid (koral/grid.zig) ------------------------------
struct Grid {
  int nx, ny, nz, ng, ngx, ngy, ngz;
  double minx, maxx, miny, maxy, minz, maxz, dx, dy, dz;
};
inline Grid grid_init(int nx, int ny, int nz, int ng, double minx, double maxx, double miny, double maxy, double minz,
                      double maxz) {
  Grid g;
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  g.ng = ng;
  g.ngx = nx > 1 ? ng : 0;
  g.ngy = ny > 1 ? ng : 0;
  g.ngz = nz > 1 ? ng : 0;
  g.minx = minx;
  g.maxx = maxx;
  g.miny = miny;
  g.maxy = maxy;
  g.minz = minz;
  g.maxz = maxz;
  g.dx = (maxx - minx) / (double)nx;
  g.dy = (maxy - miny) / (double)ny;
  g.dz = (maxz - minz) / (double)nz;
  return g;
}
KC_HD double grid_xl(const Grid& g, long i) { return g.minx + (double)i * g.dx; }
KC_HD double grid_yl(const Grid& g, long i) { return g.miny + (double)i * g.dy; }
KC_HD double grid_zl(const Grid& g, long i) { return g.minz + (double)i * g.dz; }
KC_HD double grid_xc(const Grid& g, long i) { return 0.5 * (grid_xl(g, i) + grid_xl(g, i + 1)); }
KC_HD double grid_yc(const Grid& g, long i) { return 0.5 * (grid_yl(g, i) + grid_yl(g, i + 1)); }
KC_HD double grid_zc(const Grid& g, long i) { return 0.5 * (grid_zl(g, i) + grid_zl(g, i + 1)); }
// C get_size_x (grid.zig:152)
KC_HD double cell_size(const Grid& g, long i, int dim) {
  if (dim == 0) return grid_xl(g, i + 1) - grid_xl(g, i);
  if (dim == 1) return grid_yl(g, i + 1) - grid_yl(g, i);
  return grid_zl(g, i + 1) - grid_zl(g, i);
}

// C calc_Krzysie_at_center with MODYFIKUJKRZYSIE (precompute.zig:30)
KC_HD void apply_kris_correction(int coords, const MetricParams& mp, const Grid& g, CoordData& d, long ix, long iy,
                                  long iz) {
  double xc[4] = {0.0, grid_xc(g, ix), grid_yc(g, iy), grid_zc(g, iz)};
  double gdet_c = d.gdet;
  double dxs[3] = {g.dx, g.dy, g.dz};
  for (int kappa = 1; kappa < 4; ++kappa) {
    double ck = 0.0, sk = 1.0e-300;
    for (int mu = 0; mu < 4; ++mu) {
      ck += d.kris[mu][kappa][mu];
      sk += kmath::fabs(d.kris[mu][kappa][mu]);
    }
    double xh[4] = {xc[0], xc[1], xc[2], xc[3]}, xlo[4] = {xc[0], xc[1], xc[2], xc[3]};
    if (kappa == 1) {
      xh[1] = grid_xl(g, ix + 1);
      xlo[1] = grid_xl(g, ix);
    } else if (kappa == 2) {
      xh[2] = grid_yl(g, iy + 1);
      xlo[2] = grid_yl(g, iy);
    } else {
      xh[3] = grid_zl(g, iz + 1);
      xlo[3] = grid_zl(g, iz);
    }
    double gdet_hi = gdet_at(coords, mp, xh);
    double gdet_lo = gdet_at(coords, mp, xlo);
    double dk = (gdet_hi - gdet_lo) / (dxs[kappa - 1] * gdet_c);
    for (int mu = 0; mu < 4; ++mu) {
      double wk = kmath::fabs(d.kris[mu][kappa][mu]) / sk;
      d.kris[mu][kappa][mu] += (dk - ck) * wk;
      d.kris[mu][mu][kappa] = d.kris[mu][kappa][mu];
    }
  }
}

// the 4x5 g / G blocks (precompute.zig:274 storeBlocks)
KC_HD void store_blocks(const CoordData& d, double gblk[20], double Gblk[20]) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      gblk[i * 5 + j] = d.gcov[i][j];
      Gblk[i * 5 + j] = d.gcon[i][j];
    }
  for (int j = 0; j < 3; ++j) gblk[j * 5 + 4] = d.dlgdet[j];
  gblk[3 * 5 + 4] = d.gdet;
  for (int i = 0; i < 3; ++i) Gblk[i * 5 + 4] = 0.0;
  Gblk[3 * 5 + 4] = d.gttpert;
}
// Geometry from cached blocks (precompute.zig:451 geometryFromBlocks)
KC_HD void geom_from_blocks(const double gblk[20], const double Gblk[20], double x1, double x2, double x3, Geom& g) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 5; ++j) {
      g.gg[i][j] = gblk[i * 5 + j];
      g.GG[i][j] = Gblk[i * 5 + j];
    }
  g.xx[0] = 0.0;
  g.xx[1] = x1;
  g.xx[2] = x2;
  g.xx[3] = x3;
  geom_finish(g);
}
// geometry at an arbitrary point (precompute.zig:90 geometryAt)
KC_HD void geometry_at(int coords, const MetricParams& mp, const double x[4], Geom& geo) {
  CoordData d;
  metric_compute(coords, mp, x, d);
  double gb[20], Gb[20];
  store_blocks(d, gb, Gb);
  geom_from_blocks(gb, Gb, x[1], x[2], x[3], geo);
}

// ---- coordinate transforms (koral/metric/coco.zig) ---------------------------
// The BL<->KS time shift only moves x^0, which no consumer reads (the metric is
// stationary and the BL geometry stores xxvec[0] = 0), so it is not evaluated.
KC_HD void mks2_to_ks(const double x[4], const MetricParams& mp, double o[4]) {
  double r = kmath::exp(x[1]) + mp.mksr0;
  double th = mks2_theta(dconst(x[2]), mp.mksh0).v;
  o[0] = x[0];
  o[1] = r;
  o[2] = th;
  o[3] = x[3];
}
KC_HD void eye4(double m[4][4]) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) m[i][j] = (i == j) ? 1.0 : 0.0;
}
KC_HD void matmul4(const double a[4][4], const double b[4][4], double c[4][4]) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double s = 0.0;
      for (int k = 0; k < 4; ++k) s += a[i][k] * b[k][j];
      c[i][j] = s;
    }
}
// coco.zig:94,104,113,123
KC_HD void dxdx_bl_to_ks(const double x[4], const MetricParams& mp, double m[4][4]) {
  double r = x[1];
  double delta = r * r - 2.0 * r + mp.a * mp.a;
  eye4(m);
  m[0][1] = 2.0 * r / delta;
  m[3][1] = mp.a / delta;
}
KC_HD void dxdx_ks_to_bl(const double x[4], const MetricParams& mp, double m[4][4]) {
  double r = x[1];
  double delta = r * r - 2.0 * r + mp.a * mp.a;
  eye4(m);
  m[0][1] = -2.0 * r / delta;
  m[3][1] = -mp.a / delta;
}
KC_HD void dxdx_mks2_to_ks(const double x[4], const MetricParams& mp, double m[4][4]) {
  eye4(m);
  m[1][1] = kmath::exp(x[1]);
  m[2][2] = mks2_dtheta_dx2_metric(dconst(x[2]), mp.mksh0).v;
}
KC_HD void dxdx_ks_to_mks2(const double x[4], const MetricParams& mp, double m[4][4]) {
  double h0 = mp.mksh0;
  eye4(m);
  m[1][1] = 1.0 / (x[1] - mp.mksr0);
  double v = (2.0 / KP_PI) * (x[2] - 0.5 * KP_PI) * kmath::tan(0.5 * KP_PI * h0);
  m[2][2] = 2.0 * kmath::tan(0.5 * KP_PI * h0) / (h0 * KP_PI * KP_PI * (1.0 + v * v));
}
// Jacobian dx_to/dx_from at x (coco.zig:146), the pairs this engine uses
KC_HD void dxdx(const double x[4], int from, int to, const MetricParams& mp, double m[4][4]) {
  if (from == to) {
    eye4(m);
    return;
  }
  double a[4][4], b[4][4], xk[4];
  if (from == MKS2 && to == BL) {
    mks2_to_ks(x, mp, xk);
    dxdx_ks_to_bl(xk, mp, a);
    dxdx_mks2_to_ks(x, mp, b);
    matmul4(a, b, m);
  } else if (from == BL && to == MKS2) {
    dxdx_ks_to_mks2(x, mp, a);  // blToKs moves x^0 only
    dxdx_bl_to_ks(x, mp, b);
    matmul4(a, b, m);
  } else if (from == MKS2 && to == KS) {
    dxdx_mks2_to_ks(x, mp, m);
  } else if (from == KS && to == MKS2) {
    dxdx_ks_to_mks2(x, mp, m);
  } else if (from == BL && to == KS) {
    dxdx_bl_to_ks(x, mp, m);
  } else {
    dxdx_ks_to_bl(x, mp, m);
  }
}
// MKS2 -> BL point transform (coco.zig:56, spatial part)
KC_HD void mks2_to_bl(const double x[4], const MetricParams& mp, double o[4]) { mks2_to_ks(x, mp, o); }

// The full point transform including the x^0 shift (coco.zig:21,56), for
// diagnostics and the coordinate goldens.
KC_HD double bl_ks_time_shift(double r, double a) {
  double delta = r * r - 2.0 * r + a * a;
  double sqrta = kmath::sqrt(1.0 - a * a);
  return 2.0 / sqrta * kmath::atanh(sqrta / (1.0 - r)) + kmath::log(delta);
}
KC_HD double mks2_x2_from_theta(double theta, double h0) {
  return (0.5 * h0 + (1.0 / KP_PI) * kmath::atan((1.0 / KP_PI) * (2.0 * theta - KP_PI) * kmath::tan(0.5 * KP_PI * h0))) / h0;
}
KC_HD void coco_full(const double x[4], int from, int to, const MetricParams& mp, double y[4]) {
  double k[4] = {x[0], x[1], x[2], x[3]};
  if (from == to) {
    for (int i = 0; i < 4; ++i) y[i] = x[i];
    return;
  }
  if (from == MKS2) mks2_to_ks(x, mp, k);
  else if (from == BL) k[0] = x[0] + bl_ks_time_shift(x[1], mp.a);
  if (to == KS) {
    for (int i = 0; i < 4; ++i) y[i] = k[i];
  } else if (to == BL) {
    y[0] = k[0] - bl_ks_time_shift(k[1], mp.a);
    y[1] = k[1];
    y[2] = k[2];
    y[3] = k[3];
  } else {  // MKS2
    y[0] = k[0];
    y[1] = kmath::log(k[1] - mp.mksr0);
    y[2] = mks2_x2_from_theta(k[2], mp.mksh0);
    y[3] = k[3];
  }
}

// BL geometry at a cell center (precompute.zig:122 geometryBLat)
KC_HD void geometry_bl_at(const Grid& gr, const MetricParams& mp, long ix, long iy, long iz, Geom& geo) {
  double xx[4] = {0.0, grid_xc(gr, ix), grid_yc(gr, iy), grid_zc(gr, iz)};
  double xbl[4];
  mks2_to_bl(xx, mp, xbl);
  geometry_at(BL, mp, xbl, geo);
}

// ---- whole-primitive coordinate transform (koral/frames.zig:225 transPmhdCocoJ)
KC_HD int trans_pmhd_coco_j(const double ppin[NV], const Geom& g1, const Geom& g2, const double jac[4][4], double pp2[NV]) {
  double t[NV];
  for (int i = 0; i < NV; ++i) t[i] = ppin[i];
  double ucon1[4], ucov1[4];
  ucon_ucov_from_prims(ppin[VX], ppin[VY], ppin[VZ], g1, ucon1, ucov1);
  double B[3] = {ppin[B1], ppin[B2], ppin[B3]};
  double bcon[4];
  bcon_from_4vel(B, ucon1, ucov1, bcon);
  transform_vec(bcon, jac, bcon);
  double ucon[4];
  transform_vec(ucon1, jac, ucon);
  int e = convert(ucon, VEL4, VELR, g2, TRUST_UT, ucon);
  if (e) return e;
  t[VX] = ucon[1];
  t[VY] = ucon[2];
  t[VZ] = ucon[3];
  double ucon2[4], ucov2[4], Bc[4];
  ucon_ucov_from_prims(t[VX], t[VY], t[VZ], g2, ucon2, ucov2);
  big_bcon_from_4vel(bcon, ucon2, Bc);
  t[B1] = Bc[1];
  t[B2] = Bc[2];
  t[B3] = Bc[3];
  for (int i = 0; i < NV; ++i) pp2[i] = t[i];
  return E_OK;
}
// frames.zig:267 (transPradCoco) with the point Jacobian supplied
KC_HD int trans_prad_coco_j(const double ppin[NV], const Geom& g1, const Geom& g2, const double jac[4][4], double pp2[NV]) {
  double t[NV];
  for (int i = 0; i < NV; ++i) t[i] = ppin[i];
  double vin[4] = {0.0, ppin[FX], ppin[FY], ppin[FZ]}, ucon[4];
  velr_to_vel4(vin, g1, ucon);
  transform_vec(ucon, jac, ucon);
  int e = convert(ucon, VEL4, VELR, g2, TRUST_UT, ucon);
  if (e) return e;
  t[FX] = ucon[1];
  t[FY] = ucon[2];
  t[FZ] = ucon[3];
  for (int i = 0; i < NV; ++i) pp2[i] = t[i];
  return E_OK;
}

}  // namespace kp
