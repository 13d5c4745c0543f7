// orc_sim.cpp — TEST INFRASTRUCTURE (the CPU oracle), not product code.
//
// A serial, array-of-structs restatement of the reference's evolution driver
// `Sim(cfg).step` (koral/sim.zig:1792) and every pass it calls: ghost fill and
// corners (koral/sim/bc.zig), the PUFFY boundary callback
// (koral/problems/puffy/puffy.zig:1080), polar-axis overwrite
// (koral/sim/polaraxis.zig), wavespeeds/CFL (sim.zig:747), the interpolation
// sweeps and face fluxes (sim.zig:1209-1503), flux-CT (koral/sim/ct.zig), the
// conserved update with the metric source (sim.zig:1140,1542), u2p + fixups
// (sim.zig:924-1133), the implicit operator (sim.zig:1715), stage arithmetic
// (sim.zig:1586-1709), radiative viscosity (koral/sim/rijvisc.zig) and the
// mimic dynamo (koral/sim/dynamo.zig). The per-point physics is the shared
// restatement in include/koral/. Tests compare the sm_100a engine with this
// and this with the reference's self-goldens. Only tests/ and bench.py's CPU
// baseline load it.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "../include/koral/kdump.h"
#include "../include/koral/kinit.h"
#include "../include/koral/kvisc.h"

using namespace kp;

namespace {

const int NFL = 6;  // entropy, entropy2, entropy3, hd_fixup, rad_fixup, radimp_fixup
enum { F_ENTROPY = 0, F_ENTROPY2 = 1, F_ENTROPY3 = 2, F_HD = 3, F_RAD = 4, F_RADIMP = 5 };
const int NSCAL = 20;
// Scal slots (koral/sim/storage.zig:30): per dim {ahd l, r, m, arad l, r, m}
inline int s_ahd_l(int d) { return 6 * d + 0; }
inline int s_ahd_r(int d) { return 6 * d + 1; }
inline int s_ahd_m(int d) { return 6 * d + 2; }
inline int s_arad_l(int d) { return 6 * d + 3; }
inline int s_arad_r(int d) { return 6 * d + 4; }
inline int s_arad_m(int d) { return 6 * d + 5; }
const int S_TSTEPDEN = 18, S_CELLDT = 19;

struct Face {
  long nxs = 0, nys = 0, nzs = 0, ngx = 0, ngy = 0, ngz = 0;
  std::vector<double> d;
  void init(const Grid& g, int dim) {
    nxs = g.nx + 2 * g.ngx + (dim == 0);
    nys = g.ny + 2 * g.ngy + (dim == 1);
    nzs = g.nz + 2 * g.ngz + (dim == 2);
    ngx = g.ngx;
    ngy = g.ngy;
    ngz = g.ngz;
    d.assign((size_t)nxs * nys * nzs * NV, 0.0);
  }
  double* at(long ix, long iy, long iz) {
    return &d[(size_t)((((iz + ngz) * nys + (iy + ngy)) * nxs + (ix + ngx)) * NV)];
  }
};

struct Err {
  int code = 0;
  void set(int e) {
    if (e && !code) code = e;
  }
};

struct OSim {
  Grid g;
  kc_options opt;
  SimParams sp;
  long sx, sy, sz, nc;
  std::vector<double> cg, cG, kris, jbl;
  std::vector<Geom> blg;
  std::vector<double> fgb[3], fGb[3];
  std::vector<double> p, u, ut0, ut1, ut2, dut1, dut2, drt1, drt2, uforget, u_bak, p_bak;
  Face pb_l[3], pb_r[3], fl_l[3], fl_r[3], flb[3];
  std::vector<double> scal;
  std::vector<int> flags;
  std::vector<double> emf[3];
  std::vector<double> vecpot, rijvisc, dyn_a, scaleth;
  double t = 0, time = 0, dt = 0, own_dt = 0, tstepdenmax = 0, tstepdenmin = 1.0e50;
  double min_dx = 0, min_dy = 0, min_dz = 0;
  long nstep = 0, n_radimp_failures = 0, n_radimp_fail_step = 0, n_radimp_iters = 0, n_radimp_solves = 0;
  long n_guard = 0;
  int nthreads = 1;

  long nxi() const { return g.nx; }
  long nyi() const { return g.ny; }
  long nzi() const { return g.nz; }
  long ndim(int d) const { return d == 0 ? g.nx : d == 1 ? g.ny : g.nz; }
  long ci(long ix, long iy, long iz) const { return (ix + g.ngx) + (iy + g.ngy) * sx + (iz + g.ngz) * sx * sy; }
  double* P(long ix, long iy, long iz) { return &p[ci(ix, iy, iz) * NV]; }
  double* U(long ix, long iy, long iz) { return &u[ci(ix, iy, iz) * NV]; }
  double* F(std::vector<double>& f, long ix, long iy, long iz) { return &f[ci(ix, iy, iz) * NV]; }
  int& flag(int f, long ix, long iy, long iz) { return flags[ci(ix, iy, iz) * NFL + f]; }
  double& sc(int s, long ix, long iy, long iz) { return scal[ci(ix, iy, iz) * NSCAL + s]; }
  double cgdet(long ix, long iy, long iz) const { return cg[ci(ix, iy, iz) * 20 + 19]; }
  const double* kr(long ix, long iy, long iz) const { return &kris[ci(ix, iy, iz) * 64]; }

  void geom(long ix, long iy, long iz, Geom& geo) const {
    long c = ci(ix, iy, iz);
    geom_from_blocks(&cg[c * 20], &cG[c * 20], grid_xc(g, ix), grid_yc(g, iy), grid_zc(g, iz), geo);
  }
  long face_index(int dim, long ix, long iy, long iz) const {
    long jx = ix + g.ngx, jy = iy + g.ngy, jz = iz + g.ngz;
    if (dim == 0) return jx + jy * (sx + 1) + jz * sy * (sx + 1);
    if (dim == 1) return jx + jy * sx + jz * (sy + 1) * sx;
    return jx + jy * sx + jz * sy * sx;
  }
  void geom_face(long ix, long iy, long iz, int dim, Geom& geo) const {
    long f = face_index(dim, ix, iy, iz);
    double x1 = dim == 0 ? grid_xl(g, ix) : grid_xc(g, ix);
    double x2 = dim == 1 ? grid_yl(g, iy) : grid_yc(g, iy);
    double x3 = dim == 2 ? grid_zl(g, iz) : grid_zc(g, iz);
    geom_from_blocks(&fgb[dim][f * 20], &fGb[dim][f * 20], x1, x2, x3, geo);
  }
  void jac_bl(long ix, long iy, long iz, double j[4][4]) const {
    const double* s = &jbl[ci(ix, iy, iz) * 16];
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) j[a][b] = s[a * 4 + b];
  }
  bool is_corner(long ix, long iy, long iz) const {
    int n = 0;
    if (ix < 0 || ix >= g.nx) ++n;
    if (iy < 0 || iy >= g.ny) ++n;
    if (iz < 0 || iz >= g.nz) ++n;
    return n >= 2;
  }
  bool polar_band() const { return sp.correct_polaraxis != 0; }
  bool polar_owns(long iy) const {
    return polar_band() && (iy < sp.nccorrectpolar || iy > g.ny - sp.nccorrectpolar - 1);
  }
};

// rows handed out one at a time from an atomic ticket (the dynamic tiles of
// koral/threading.zig:235), since implicit-solve cost varies ~17x across rows;
// every row writes only its own cells, so results do not depend on the order
template <class Fn>
void par_for(int nthreads, long lo, long hi, Fn fn) {
  if (nthreads <= 1 || hi - lo < 2) {
    for (long i = lo; i < hi; ++i) fn(i);
    return;
  }
  std::atomic<long> next(lo);
  std::vector<std::thread> th;
  for (int w = 0; w < nthreads; ++w) {
    th.emplace_back([&]() {
      for (long i = next.fetch_add(1); i < hi; i = next.fetch_add(1)) fn(i);
    });
  }
  for (auto& x : th) x.join();
}

// ---- metric cache (koral/metric/precompute.zig:175) -------------------------
void build_cache(OSim& s) {
  const Grid& g = s.g;
  const MetricParams mp = s.sp.mp;
  s.cg.assign(s.nc * 20, 0.0);
  s.cG.assign(s.nc * 20, 0.0);
  s.kris.assign(s.nc * 64, 0.0);
  s.jbl.assign(s.nc * 16, 0.0);
  s.blg.resize(s.nc);
  long zr = g.nz + 2 * g.ngz, yr = g.ny + 2 * g.ngy;
  par_for(s.nthreads, 0, zr * yr, [&](long k) {
    long iz = k / yr - g.ngz, iy = k % yr - g.ngy;
    for (long ix = -g.ngx; ix < g.nx + g.ngx; ++ix) {
      double x[4] = {0.0, grid_xc(g, ix), grid_yc(g, iy), grid_zc(g, iz)};
      CoordData d;
      metric_compute(MKS2, mp, x, d);
      apply_kris_correction(MKS2, mp, g, d, ix, iy, iz);
      long c = s.ci(ix, iy, iz);
      store_blocks(d, &s.cg[c * 20], &s.cG[c * 20]);
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
          for (int l = 0; l < 4; ++l) s.kris[c * 64 + i * 16 + j * 4 + l] = d.kris[i][j][l];
      double m[4][4];
      dxdx(x, MKS2, BL, mp, m);
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) s.jbl[c * 16 + i * 4 + j] = m[i][j];
      geometry_bl_at(g, mp, ix, iy, iz, s.blg[c]);
    }
  });
  for (int dim = 0; dim < 3; ++dim) {
    long nf = (s.sx + (dim == 0)) * (s.sy + (dim == 1)) * (s.sz + (dim == 2));
    s.fgb[dim].assign(nf * 20, 0.0);
    s.fGb[dim].assign(nf * 20, 0.0);
  }
  long zr1 = zr + 1, yr1 = yr + 1;
  par_for(s.nthreads, 0, zr1 * yr1, [&](long k) {
    long iz = k / yr1 - g.ngz, iy = k % yr1 - g.ngy;
    long nxh = g.nx + g.ngx, nyh = g.ny + g.ngy, nzh = g.nz + g.ngz;
    for (long ix = -g.ngx; ix <= nxh; ++ix) {
      CoordData d;
      if (iy < nyh && iz < nzh) {
        double x[4] = {0.0, grid_xl(g, ix), grid_yc(g, iy), grid_zc(g, iz)};
        metric_compute(MKS2, mp, x, d);
        long f = s.face_index(0, ix, iy, iz);
        store_blocks(d, &s.fgb[0][f * 20], &s.fGb[0][f * 20]);
      }
      if (ix < nxh && iz < nzh) {
        double x[4] = {0.0, grid_xc(g, ix), grid_yl(g, iy), grid_zc(g, iz)};
        metric_compute(MKS2, mp, x, d);
        long f = s.face_index(1, ix, iy, iz);
        store_blocks(d, &s.fgb[1][f * 20], &s.fGb[1][f * 20]);
      }
      if (ix < nxh && iy < nyh) {
        double x[4] = {0.0, grid_xc(g, ix), grid_yc(g, iy), grid_zl(g, iz)};
        metric_compute(MKS2, mp, x, d);
        long f = s.face_index(2, ix, iy, iz);
        store_blocks(d, &s.fgb[2][f * 20], &s.fGb[2][f * 20]);
      }
    }
  });
}

// ---- boundary conditions (koral/sim/bc.zig, puffy.zig:1080) -----------------
int puffy_bc(OSim& s, long ix, long iy, long iz, int face, double pp[NV]) {
  const long nx = s.g.nx, ny = s.g.ny;
  const MetricParams& mp = s.sp.mp;
  if (face == 1) {  // xhi: outflow with r-rescaling + no-inflow
    for (int i = 0; i < NV; ++i) pp[i] = s.P(nx - 1, iy, iz)[i];
    Geom geo;
    s.geom(ix, iy, iz, geo);
    const Geom& gbl = s.blg[s.ci(ix, iy, iz)];
    double jm2b[4][4], jb2m[4][4];
    s.jac_bl(ix, iy, iz, jm2b);
    int e = trans_pmhd_coco_j(pp, geo, gbl, jm2b, pp);
    if (e) return e;
    const Geom& gbd = s.blg[s.ci(nx - 1, iy, iz)];
    double rghost = gbl.xx[1], rbound = gbd.xx[1];
    double scale1 = rbound * rbound / rghost / rghost;
    double scale2 = rbound / rghost;
    pp[RHO] *= scale1;
    pp[UU] *= scale1;
    pp[B1] *= scale1;
    pp[B2] *= scale2;
    pp[B3] *= scale2;
    pp[VY] *= scale1;
    pp[VZ] *= scale1;
    pp[EE] *= scale1;
    pp[FY] *= scale1;
    pp[FZ] *= scale1;
    double xbl[4] = {0.0, gbl.xx[1], gbl.xx[2], gbl.xx[3]};
    dxdx(xbl, BL, MKS2, mp, jb2m);
    e = trans_pmhd_coco_j(pp, gbl, geo, jb2m, pp);
    if (e) return e;
    double ucon[4] = {0.0, pp[VX], pp[VY], pp[VZ]};
    velr_to_vel4(ucon, geo, ucon);
    transform_vec(ucon, jm2b, ucon);
    if (ucon[1] < 0.0) {
      ucon[1] = 0.0;
      transform_vec(ucon, jb2m, ucon);
      e = convert(ucon, VEL4, VELR, geo, RECOMPUTE_UT, ucon);
      if (e) return e;
      pp[VX] = ucon[1];
      pp[VY] = ucon[2];
      pp[VZ] = ucon[3];
    }
    double urf[4] = {0.0, pp[FX], pp[FY], pp[FZ]};
    velr_to_vel4(urf, geo, urf);
    transform_vec(urf, jm2b, urf);
    if (urf[1] < 0.0) {
      urf[1] = 0.0;
      transform_vec(urf, jb2m, urf);
      e = convert(urf, VEL4, VELR, geo, RECOMPUTE_UT, urf);
      if (e) return e;
      pp[FX] = urf[1];
      pp[FY] = urf[2];
      pp[FZ] = urf[3];
    }
    return E_OK;
  }
  if (face == 0) {  // xlo: copy of the first active column
    for (int i = 0; i < NV; ++i) pp[i] = s.P(0, iy, iz)[i];
    return E_OK;
  }
  long iiy = (face == 2) ? -iy - 1 : ny - (iy - ny) - 1;  // polar reflection
  for (int i = 0; i < NV; ++i) pp[i] = s.P(ix, iiy, iz)[i];
  pp[VY] = -pp[VY];
  pp[B2] = -pp[B2];
  pp[FY] = -pp[FY];
  return E_OK;
}

int set_bc_cell(OSim& s, long ix, long iy, long iz, int face) {
  int axis = face / 2;
  int kind = s.sp.bc[axis];
  double pp[NV];
  if (kind == KC_BC_PUFFY) {
    int e = puffy_bc(s, ix, iy, iz, face, pp);
    if (e) return e;
  } else {
    long iix = ix, iiy = iy, iiz = iz;
    long nx = s.g.nx, ny = s.g.ny, nz = s.g.nz;
    if (axis == 0) {
      if (kind == KC_BC_PERIODIC) {
        if (ix < 0) iix = ix + nx;
        if (ix > nx - 1) iix = ix - nx;
      } else {
        if (ix < 0) iix = 0;
        if (ix > nx - 1) iix = nx - 1;
      }
    } else if (axis == 1) {
      if (kind == KC_BC_PERIODIC) {
        if (iy < 0) iiy = iy + ny;
        if (iy > ny - 1) iiy = iy - ny;
        if (ny < s.g.ng) iiy = 0;
      } else {
        if (iy < 0) iiy = 0;
        if (iy > ny - 1) iiy = ny - 1;
      }
    } else {
      if (kind == KC_BC_PERIODIC) {
        if (iz < 0) iiz = iz + nz;
        if (iz > nz - 1) iiz = iz - nz;
        if (nz < s.g.ng) iiz = 0;
      } else {
        if (iz < 0) iiz = 0;
        if (iz > nz - 1) iiz = nz - 1;
      }
    }
    for (int i = 0; i < NV; ++i) pp[i] = s.P(iix, iiy, iiz)[i];
  }
  Geom geo;
  s.geom(ix, iy, iz, geo);
  double uu[NV];
  p2u(pp, uu, geo, s.sp.gam);
  for (int i = 0; i < NV; ++i) {
    s.P(ix, iy, iz)[i] = pp[i];
    s.U(ix, iy, iz)[i] = uu[i];
  }
  return E_OK;
}
void p2u_cell(OSim& s, long ix, long iy, long iz) {
  Geom geo;
  s.geom(ix, iy, iz, geo);
  p2u(s.P(ix, iy, iz), s.U(ix, iy, iz), geo, s.sp.gam);
}
void copy_p(OSim& s, const long d[3], const long src[3]) {
  double tmp[NV];
  for (int i = 0; i < NV; ++i) tmp[i] = s.P(src[0], src[1], src[2])[i];
  for (int i = 0; i < NV; ++i) s.P(d[0], d[1], d[2])[i] = tmp[i];
}
void avg_p(OSim& s, const long d[3], const long a[3], const long b[3]) {
  double pp[NV];
  for (int i = 0; i < NV; ++i) pp[i] = 0.5 * (s.P(a[0], a[1], a[2])[i] + s.P(b[0], b[1], b[2])[i]);
  for (int i = 0; i < NV; ++i) s.P(d[0], d[1], d[2])[i] = pp[i];
}

// bc.zig:256 fillCorners2d (no periodic x/y in PUFFY; the periodic sources kept)
void fill_corners_2d(OSim& s) {
  long nx = s.g.nx, ny = s.g.ny, ng = s.g.ng;
  bool px = s.sp.bc[0] == KC_BC_PERIODIC, py = s.sp.bc[1] == KC_BC_PERIODIC;
  auto cp = [&](long dx, long dy, long sx_, long sy_) {
    long d[3] = {dx, dy, 0}, src[3] = {sx_, sy_, 0};
    copy_p(s, d, src);
    p2u_cell(s, dx, dy, 0);
  };
  auto av = [&](long dx, long dy, const long s1[4]) {
    long d[3] = {dx, dy, 0}, a[3] = {s1[0], s1[1], 0}, b[3] = {s1[2], s1[3], 0};
    avg_p(s, d, a, b);
    p2u_cell(s, dx, dy, 0);
  };
  // bottom-left
  for (long i = 0; i < ng - 1; ++i) {
    cp(-ng + i, -1, -ng + i, 0);
    cp(-1, -ng + i, 0, -ng + i);
  }
  {
    long s1[4] = {-1, 0, 0, -1};
    if (py) { s1[0] = -1; s1[1] = ny - 1; s1[2] = -1; s1[3] = ny - 1; }
    if (px) { s1[0] = nx - 1; s1[1] = -1; s1[2] = nx - 1; s1[3] = -1; }
    av(-1, -1, s1);
    long s2[4] = {-2, -1, -1, -2};
    if (py) { s2[0] = -2; s2[1] = ny - 2; s2[2] = -2; s2[3] = ny - 2; }
    if (px) { s2[0] = nx - 2; s2[1] = -2; s2[2] = nx - 2; s2[3] = -2; }
    av(-2, -2, s2);
  }
  // top-left
  for (long i = 0; i < ng - 1; ++i) {
    cp(-ng + i, ny, -ng + i, ny - 1);
    cp(-1, ny + i + 1, 0, ny + i + 1);
  }
  {
    long s1[4] = {-1, ny - 1, 0, ny};
    if (py) { s1[0] = -1; s1[1] = 0; s1[2] = -1; s1[3] = 0; }
    if (px) { s1[0] = nx - 1; s1[1] = ny; s1[2] = nx - 1; s1[3] = ny; }
    av(-1, ny, s1);
    long s2[4] = {-2, ny, -1, ny + 1};
    if (py) { s2[0] = -2; s2[1] = 1; s2[2] = -2; s2[3] = 1; }
    if (px) { s2[0] = nx - 2; s2[1] = ny + 1; s2[2] = nx - 2; s2[3] = ny + 1; }
    av(-2, ny + 1, s2);
  }
  // bottom-right
  for (long i = 0; i < ng - 1; ++i) {
    cp(nx + i + 1, -1, nx + i + 1, 0);
    cp(nx, -ng + i, nx - 1, -ng + i);
  }
  {
    long s1[4] = {nx - 1, -1, nx, 0};
    if (py) { s1[0] = nx; s1[1] = ny - 1; s1[2] = nx; s1[3] = ny - 1; }
    if (px) { s1[0] = 0; s1[1] = -1; s1[2] = 0; s1[3] = -1; }
    av(nx, -1, s1);
    long s2[4] = {nx, -2, nx + 1, -1};
    if (py) { s2[0] = nx + 1; s2[1] = ny - 2; s2[2] = nx + 1; s2[3] = ny - 2; }
    if (px) { s2[0] = 1; s2[1] = -2; s2[2] = 1; s2[3] = -2; }
    av(nx + 1, -2, s2);
  }
  // top-right
  for (long i = 0; i < ng - 1; ++i) {
    cp(nx + i + 1, ny, nx + i + 1, ny - 1);
    cp(nx, ny + i + 1, nx - 1, ny + i + 1);
  }
  {
    long s1[4] = {nx - 1, ny, nx, ny - 1};
    if (py) { s1[0] = nx; s1[1] = 0; s1[2] = nx; s1[3] = 0; }
    if (px) { s1[0] = 0; s1[1] = ny; s1[2] = 0; s1[3] = ny; }
    av(nx, ny, s1);
    long s2[4] = {nx, ny + 1, nx + 1, ny};
    if (py) { s2[0] = nx + 1; s2[1] = 1; s2[2] = nx + 1; s2[3] = 1; }
    if (px) { s2[0] = 1; s2[1] = ny + 1; s2[2] = 1; s2[3] = ny + 1; }
    av(nx + 1, ny + 1, s2);
  }
}

// bc.zig:404 fillEdgeTube
void fill_edge_tube(OSim& s, int pa, bool a_hi, int pb, bool b_hi, int pc) {
  long ng = s.g.ng;
  long dims[3] = {s.g.nx, s.g.ny, s.g.nz};
  long na = dims[pa], nb = dims[pb], ncc = dims[pc];
  long a_edge = a_hi ? na - 1 : 0, a_g1 = a_hi ? na : -1, a_g2 = a_hi ? na + 1 : -2;
  long b_edge = b_hi ? nb - 1 : 0, b_g1 = b_hi ? nb : -1, b_g2 = b_hi ? nb + 1 : -2;
  auto cell = [&](long av, long bv, long cv, long o[3]) {
    o[pa] = av;
    o[pb] = bv;
    o[pc] = cv;
  };
  for (long c = -ng; c < ncc + ng; ++c) {
    for (long i = 0; i < ng - 1; ++i) {
      long a_out = a_hi ? na + i + 1 : -ng + i;
      long b_out = b_hi ? nb + i + 1 : -ng + i;
      long db[3], sb[3], da[3], sa[3];
      cell(a_out, b_g1, c, db);
      cell(a_out, b_edge, c, sb);
      copy_p(s, db, sb);
      p2u_cell(s, db[0], db[1], db[2]);
      cell(a_g1, b_out, c, da);
      cell(a_edge, b_out, c, sa);
      copy_p(s, da, sa);
      p2u_cell(s, da[0], da[1], da[2]);
    }
    long d1[3], x1[3], y1[3];
    cell(a_g1, b_g1, c, d1);
    cell(a_g1, b_edge, c, x1);
    cell(a_edge, b_g1, c, y1);
    avg_p(s, d1, x1, y1);
    p2u_cell(s, d1[0], d1[1], d1[2]);
    long d2[3], x2[3], y2[3];
    cell(a_g2, b_g2, c, d2);
    cell(a_g2, b_g1, c, x2);
    cell(a_g1, b_g2, c, y2);
    avg_p(s, d2, x2, y2);
    p2u_cell(s, d2[0], d2[1], d2[2]);
  }
}
// bc.zig:457 fillCornerCube
void fill_corner_cube(OSim& s, bool xh, bool yh, bool zh) {
  long ng = s.g.ng, nx = s.g.nx, ny = s.g.ny, nz = s.g.nz;
  long src[3] = {xh ? nx - 1 : 0, yh ? ny - 1 : 0, zh ? nz - 1 : 0};
  for (long ix = xh ? nx : -ng; ix < (xh ? nx + ng : 0); ++ix)
    for (long iy = yh ? ny : -ng; iy < (yh ? ny + ng : 0); ++iy)
      for (long iz = zh ? nz : -ng; iz < (zh ? nz + ng : 0); ++iz) {
        long d[3] = {ix, iy, iz};
        copy_p(s, d, src);
        p2u_cell(s, ix, iy, iz);
      }
}
void fill_corners_3d(OSim& s) {
  fill_edge_tube(s, 0, false, 1, false, 2);
  fill_edge_tube(s, 0, false, 1, true, 2);
  fill_edge_tube(s, 0, true, 1, false, 2);
  fill_edge_tube(s, 0, true, 1, true, 2);
  fill_edge_tube(s, 0, false, 2, false, 1);
  fill_edge_tube(s, 0, false, 2, true, 1);
  fill_edge_tube(s, 0, true, 2, false, 1);
  fill_edge_tube(s, 0, true, 2, true, 1);
  fill_edge_tube(s, 1, false, 2, false, 0);
  fill_edge_tube(s, 1, false, 2, true, 0);
  fill_edge_tube(s, 1, true, 2, false, 0);
  fill_edge_tube(s, 1, true, 2, true, 0);
  fill_corner_cube(s, false, false, false);
  fill_corner_cube(s, true, false, false);
  fill_corner_cube(s, false, true, false);
  fill_corner_cube(s, true, true, false);
  fill_corner_cube(s, false, false, true);
  fill_corner_cube(s, true, false, true);
  fill_corner_cube(s, false, true, true);
  fill_corner_cube(s, true, true, true);
}

// C set_bc (bc.zig:40)
int set_bc(OSim& s) {
  const Grid& g = s.g;
  Err er;
  if (g.ngx > 0)
    for (long iz = 0; iz < g.nz; ++iz)
      for (long iy = 0; iy < g.ny; ++iy)
        for (long i = 1; i <= g.ngx; ++i) {
          er.set(set_bc_cell(s, -i, iy, iz, 0));
          er.set(set_bc_cell(s, g.nx - 1 + i, iy, iz, 1));
        }
  if (g.ngy > 0)
    for (long iz = 0; iz < g.nz; ++iz)
      for (long ix = 0; ix < g.nx; ++ix)
        for (long i = 1; i <= g.ngy; ++i) {
          er.set(set_bc_cell(s, ix, -i, iz, 2));
          er.set(set_bc_cell(s, ix, g.ny - 1 + i, iz, 3));
        }
  if (g.ngz > 0)
    for (long iy = 0; iy < g.ny; ++iy)
      for (long ix = 0; ix < g.nx; ++ix)
        for (long i = 1; i <= g.ngz; ++i) {
          er.set(set_bc_cell(s, ix, iy, -i, 4));
          er.set(set_bc_cell(s, ix, iy, g.nz - 1 + i, 5));
        }
  if (er.code) return er.code;
  if (g.ny > 1 && g.nz == 1) fill_corners_2d(s);
  else if (g.nz > 1 && g.ny > 1) fill_corners_3d(s);
  return E_OK;
}

// ---- polar axis (koral/sim/polaraxis.zig:84) ---------------------------------
void do_correct(OSim& s) {
  if (!s.polar_band()) return;
  long nc = s.sp.nccorrectpolar, ny = s.g.ny;
  for (long iz = 0; iz < s.g.nz; ++iz)
    for (long ix = 0; ix < s.g.nx; ++ix)
      for (long ic = 0; ic < nc; ++ic)
        for (int side = 0; side < 2; ++side) {
          long iy = side == 0 ? ic : ny - 1 - ic;
          long iysrc = (iy < nc) ? nc : ny - 1 - nc;
          double thaxis = grid_yl(s.g, (iy < nc) ? 0 : ny);
          double fac = kmath::fabs((grid_yc(s.g, iy) - thaxis) / (grid_yc(s.g, iysrc) - thaxis));
          double pp[NV], pps[NV];
          for (int i = 0; i < NV; ++i) {
            pp[i] = s.P(ix, iy, iz)[i];
            pps[i] = s.P(ix, iysrc, iz)[i];
          }
          pp[RHO] = pps[RHO];
          pp[UU] = pps[UU];
          pp[ENTR] = pps[ENTR];
          pp[VX] = pps[VX];
          pp[VZ] = pps[VZ];
          pp[VY] = fac * pps[VY];
          pp[EE] = pps[EE];
          pp[FX] = pps[FX];
          pp[FZ] = pps[FZ];
          pp[FY] = fac * pps[FY];
          Geom geo;
          s.geom(ix, iy, iz, geo);
          double uu[NV];
          p2u(pp, uu, geo, s.sp.gam);
          for (int i = 0; i < NV; ++i) {
            s.P(ix, iy, iz)[i] = pp[i];
            s.U(ix, iy, iz)[i] = uu[i];
          }
        }
}

// ---- u2p + fixups (sim.zig:924-1133) ------------------------------------------
void cell_fixup_hd(OSim& s) {
  if (!s.sp.do_fixups) return;
  const Grid& g = s.g;
  bool any = false;
  for (long iz = 0; iz < g.nz && !any; ++iz)
    for (long iy = 0; iy < g.ny && !any; ++iy)
      for (long ix = 0; ix < g.nx; ++ix)
        if (s.flag(F_HD, ix, iy, iz) != 0) {
          any = true;
          break;
        }
  if (!any) return;
  s.u_bak = s.u;
  s.p_bak = s.p;
  long nx = g.nx, ny = g.ny, nz = g.nz;
  for (long iz = 0; iz < nz; ++iz)
    for (long iy = 0; iy < ny; ++iy) {
      if (s.polar_owns(iy)) continue;
      for (long ix = 0; ix < nx; ++ix) {
        if (s.flag(F_HD, ix, iy, iz) == 0) continue;
        long nb[6][3] = {{ix - 1, iy, iz}, {ix + 1, iy, iz}, {ix, iy - 1, iz},
                         {ix, iy + 1, iz}, {ix, iy, iz - 1}, {ix, iy, iz + 1}};
        const double* ppn[6];
        int in_n = 0;
        for (int k = 0; k < 6; ++k) {
          if (nb[k][0] < 0 || nb[k][0] >= nx || nb[k][1] < 0 || nb[k][1] >= ny || nb[k][2] < 0 || nb[k][2] >= nz) continue;
          if (s.flag(F_HD, nb[k][0], nb[k][1], nb[k][2]) != 0) continue;
          ppn[in_n++] = s.P(nb[k][0], nb[k][1], nb[k][2]);
        }
        bool enough = (nz == 1 && ny == 1 && in_n >= 1) || (nz == 1 && in_n >= 2) || (ny == 1 && in_n >= 2) || in_n >= 3;
        if (!enough) continue;
        double pp[NV];
        for (int iv = 0; iv < NV; ++iv) pp[iv] = s.P(ix, iy, iz)[iv];
        for (int iv = 0; iv < NV; ++iv) {
          if (iv != RHO && iv < B1) {
            double sum = 0.0;
            for (int k = 0; k < in_n; ++k) sum += ppn[k][iv];
            pp[iv] = sum / (double)in_n;
          }
        }
        Geom geo;
        s.geom(ix, iy, iz, geo);
        double uu[NV];
        p2u(pp, uu, geo, s.sp.gam);
        for (int iv = 0; iv < NV; ++iv) {
          s.F(s.u_bak, ix, iy, iz)[iv] = uu[iv];
          s.F(s.p_bak, ix, iy, iz)[iv] = pp[iv];
        }
      }
    }
  s.u = s.u_bak;
  s.p = s.p_bak;
}

int calc_u2p(OSim& s) {
  const Grid& g = s.g;
  std::vector<long> guards(g.ny, 0);
  par_for(s.nthreads, 0, g.ny, [&](long iy) {
    for (long iz = 0; iz < g.nz; ++iz) {
      bool polar = s.polar_owns(iy);
      for (long ix = 0; ix < g.nx; ++ix) {
        double uu[NV], pp[NV];
        for (int i = 0; i < NV; ++i) {
          uu[i] = s.U(ix, iy, iz)[i];
          pp[i] = s.P(ix, iy, iz)[i];
        }
        s.flag(F_ENTROPY, ix, iy, iz) = 0;
        s.flag(F_ENTROPY2, ix, iy, iz) = 0;
        Geom geo;
        s.geom(ix, iy, iz, geo);
        if (polar) {
          double gdetu_inv = 1.0 / geo.gdet;
          pp[B1] = uu[B1] * gdetu_inv;
          pp[B2] = uu[B2] * gdetu_inv;
          pp[B3] = uu[B3] * gdetu_inv;
          for (int i = 0; i < NV; ++i) s.P(ix, iy, iz)[i] = pp[i];
          s.flag(F_HD, ix, iy, iz) = 0;
          s.flag(F_RAD, ix, iy, iz) = 0;
          continue;
        }
        U2pMhdRes res = u2p_mhd(uu, pp, geo, s.sp.gam, s.sp.fl);
        if (res.entropy_used) s.flag(F_ENTROPY, ix, iy, iz) = 1;
        U2pRadRes rr = u2p_rad(uu, pp, geo, s.sp.rp);
        int gc = 0;
        check_floors_mhd(pp, geo, s.sp.gam, s.sp.fl, gc);
        guards[iy] += gc;
        check_floors_rad(pp, geo, s.sp.rp);
        for (int i = 0; i < NV; ++i) s.P(ix, iy, iz)[i] = pp[i];
        s.flag(F_HD, ix, iy, iz) = res.fixup ? 1 : 0;
        s.flag(F_RAD, ix, iy, iz) = rr.corrected ? -1 : 0;
      }
    }
  });
  for (long v : guards) s.n_guard += v;
  cell_fixup_hd(s);
  return set_bc(s);
}

// ---- wavespeeds & CFL (sim.zig:747) -------------------------------------------
int calc_wavespeeds(OSim& s) {
  const Grid& g = s.g;
  bool act[3] = {g.nx > 1, g.ny > 1, g.nz > 1};
  long lx = act[0] ? 1 : 0, ly = act[1] ? 1 : 0, lz = act[2] ? 1 : 0;
  std::vector<double> tmax(g.ny + 2, -INFINITY), tmin(g.ny + 2, INFINITY);
  par_for(s.nthreads, -ly, g.ny + ly, [&](long iy) {
    for (long iz = -lz; iz < g.nz + lz; ++iz)
      for (long ix = -lx; ix < g.nx + lx; ++ix) {
        const double* pp = s.P(ix, iy, iz);
        Geom geo;
        s.geom(ix, iy, iz, geo);
        double aaa[6];
        gas_wavespeeds_lr(pp, geo, s.sp.gam, act, aaa);
        double tautot[3] = {0.0, 0.0, 0.0};
        double chi = calc_chi_slim(pp, geo, s.sp.gam, s.sp.op);
        long idx3[3] = {ix, iy, iz};
        for (int d = 0; d < 3; ++d) {
          double sg = kmath::sqrt(geo.gg[d + 1][d + 1]);
          double dxp = kmath::fmax(cell_size(g, idx3[d], d) * sg, cell_size(g, idx3[d] + 1, d) * sg);
          tautot[d] = chi * dxp;
        }
        if (s.sp.dampradwavespeednearaxis > 0) {
          long ncx = s.sp.dampradwavespeednearaxis;
          if (iy < ncx || iy >= g.ny - ncx) tautot[0] = tautot[1] = tautot[2] = 0.0;
        }
        double aval[12], rad0[6], radl[6];
        rad_wavespeeds(pp, geo, tautot, act, aval);
        for (int i = 0; i < 6; ++i) {
          rad0[i] = aval[i];
          radl[i] = aval[6 + i];
        }
        for (int d = 0; d < 3; ++d) {
          if (radl[2 * d] > 0.0) radl[2 * d] = 0.0;
          if (radl[2 * d + 1] < 0.0) radl[2 * d + 1] = 0.0;
          if (rad0[2 * d] > 0.0) rad0[2 * d] = 0.0;
          if (rad0[2 * d + 1] < 0.0) rad0[2 * d + 1] = 0.0;
        }
        for (int d = 0; d < 3; ++d) {
          s.sc(s_ahd_l(d), ix, iy, iz) = aaa[2 * d];
          s.sc(s_ahd_r(d), ix, iy, iz) = aaa[2 * d + 1];
        }
        double ax = kmath::fmax(kmath::fabs(aaa[0]), kmath::fabs(aaa[1]));
        double ay = kmath::fmax(kmath::fabs(aaa[2]), kmath::fabs(aaa[3]));
        double az = kmath::fmax(kmath::fabs(aaa[4]), kmath::fabs(aaa[5]));
        s.sc(s_ahd_m(0), ix, iy, iz) = ax;
        s.sc(s_ahd_m(1), ix, iy, iz) = ay;
        s.sc(s_ahd_m(2), ix, iy, iz) = az;
        for (int d = 0; d < 3; ++d) {
          s.sc(s_arad_l(d), ix, iy, iz) = radl[2 * d];
          s.sc(s_arad_r(d), ix, iy, iz) = radl[2 * d + 1];
          s.sc(s_arad_m(d), ix, iy, iz) = kmath::fmax(kmath::fabs(radl[2 * d]), kmath::fabs(radl[2 * d + 1]));
        }
        double wsx = kmath::fmax(ax, kmath::fmax(kmath::fabs(rad0[0]), kmath::fabs(rad0[1])));
        double wsy = kmath::fmax(ay, kmath::fmax(kmath::fabs(rad0[2]), kmath::fabs(rad0[3])));
        double wsz = kmath::fmax(az, kmath::fmax(kmath::fabs(rad0[4]), kmath::fabs(rad0[5])));
        bool in_domain = ix >= 0 && ix < g.nx && iy >= 0 && iy < g.ny && iz >= 0 && iz < g.nz;
        if (!in_domain) continue;
        double dx = cell_size(g, ix, 0), dy = cell_size(g, iy, 1), dz = cell_size(g, iz, 2);
        double tsd;
        if (g.nz > 1 && g.ny > 1) tsd = wsx / dx + wsy / dy + wsz / dz;
        else if (g.nz == 1 && g.ny > 1) tsd = wsx / dx + wsy / dy;
        else if (g.ny == 1 && g.nz > 1) tsd = wsx / dx + wsz / dz;
        else tsd = wsx / dx;
        tsd /= s.sp.tsteplim;
        s.sc(S_TSTEPDEN, ix, iy, iz) = tsd;
        if (tsd > tmax[iy + 1]) tmax[iy + 1] = tsd;
        if (tsd < tmin[iy + 1]) tmin[iy + 1] = tsd;
      }
  });
  double mx = -INFINITY, mn = INFINITY;
  for (size_t i = 0; i < tmax.size(); ++i) {
    if (tmax[i] > mx) mx = tmax[i];
    if (tmin[i] < mn) mn = tmin[i];
  }
  if (mx > s.tstepdenmax) s.tstepdenmax = mx;
  if (mn < s.tstepdenmin) s.tstepdenmin = mn;
  return E_OK;
}

// ---- interpolation sweep (sim.zig:1209) -------------------------------------
void face_avg_rijvisc(OSim& s, int dim, const long c[3], double out[4][4]) {
  const double* a = &s.rijvisc[s.ci(c[0], c[1], c[2]) * 16];
  long m[3] = {c[0], c[1], c[2]};
  m[dim] -= 1;
  const double* b = &s.rijvisc[s.ci(m[0], m[1], m[2]) * 16];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) out[i][j] = 0.5 * (a[i * 4 + j] + b[i * 4 + j]);
}

int sweep_face(OSim& s, int dim, long i, const long cell[3], const double dx5[5], long& guards) {
  long n = s.ndim(dim);
  bool dol = i >= 0, dor = i < n;
  double st[5][NV];
  long c[3] = {cell[0], cell[1], cell[2]};
  for (int k = 0; k < 5; ++k) {
    c[dim] = i - 2 + k;
    for (int iv = 0; iv < NV; ++iv) st[k][iv] = s.P(c[0], c[1], c[2])[iv];
  }
  double pl[NV], pr[NV];
  for (int iv = 0; iv < NV; ++iv) {
    double uv[5] = {st[0][iv], st[1][iv], st[2][iv], st[3][iv], st[4][iv]};
    Faces f = reconstruct(RECON_PPM, uv, dx5, s.sp.minmod_theta);
    pl[iv] = f.left;
    pr[iv] = f.right;
  }
  double ffl[NV], ffr[NV];
  bool yact = s.g.ny > 1, zact = s.g.nz > 1;
  if (dol) {
    Geom geo;
    s.geom_face(cell[0], cell[1], cell[2], dim, geo);
    int gc = 0;
    check_floors_mhd(pl, geo, s.sp.gam, s.sp.fl, gc);
    guards += gc;
    int e = f_flux_prime(pl, dim, geo, s.sp.gam, ffl);
    if (e) return e;
    if (s.sp.radviscosity) {
      double rv[4][4], uu[NV];
      face_avg_rijvisc(s, dim, cell, rv);
      p2u(pl, uu, geo, s.sp.gam);
      add_visc_flux(ffl, uu, rv, geo, dim, yact, zact, s.sp.maxradviscvel);
    }
  }
  long cp[3] = {cell[0], cell[1], cell[2]};
  cp[dim] = i + 1;
  if (dor) {
    Geom geo;
    s.geom_face(cp[0], cp[1], cp[2], dim, geo);
    int gc = 0;
    check_floors_mhd(pr, geo, s.sp.gam, s.sp.fl, gc);
    guards += gc;
    int e = f_flux_prime(pr, dim, geo, s.sp.gam, ffr);
    if (e) return e;
    if (s.sp.radviscosity) {
      double rv[4][4], uu[NV];
      face_avg_rijvisc(s, dim, cp, rv);
      p2u(pr, uu, geo, s.sp.gam);
      add_visc_flux(ffr, uu, rv, geo, dim, yact, zact, s.sp.maxradviscvel);
    }
  }
  double* d = s.pb_r[dim].at(cell[0], cell[1], cell[2]);
  for (int iv = 0; iv < NV; ++iv) d[iv] = pl[iv];
  if (dol) {
    d = s.fl_r[dim].at(cell[0], cell[1], cell[2]);
    for (int iv = 0; iv < NV; ++iv) d[iv] = ffl[iv];
  }
  d = s.pb_l[dim].at(cp[0], cp[1], cp[2]);
  for (int iv = 0; iv < NV; ++iv) d[iv] = pr[iv];
  if (dor) {
    d = s.fl_l[dim].at(cp[0], cp[1], cp[2]);
    for (int iv = 0; iv < NV; ++iv) d[iv] = ffr[iv];
  }
  return E_OK;
}

void cross_dims(int dim, int& c0, int& c1) {
  if (dim == 0) { c0 = 1; c1 = 2; }
  else if (dim == 1) { c0 = 0; c1 = 2; }
  else { c0 = 0; c1 = 1; }
}
long cross_lo(const OSim& s, int d) { return s.ndim(d) > 1 ? -1 : 0; }
long cross_hi(const OSim& s, int d) { return s.ndim(d) > 1 ? s.ndim(d) + 1 : s.ndim(d); }

int sweep(OSim& s, int dim) {
  long n = s.ndim(dim);
  if (n <= 1) return E_OK;
  int c0d, c1d;
  cross_dims(dim, c0d, c1d);
  long lo = cross_lo(s, c0d), hi = cross_hi(s, c0d);
  std::vector<long> guards(hi - lo, 0);
  std::vector<int> errs(hi - lo, 0);
  par_for(s.nthreads, lo, hi, [&](long c0) {
    for (long c1 = cross_lo(s, c1d); c1 < cross_hi(s, c1d); ++c1)
      for (long i = -1; i < n + 1; ++i) {
        double dx5[5];
        for (int k = 0; k < 5; ++k) dx5[k] = cell_size(s.g, i - 2 + k, dim);
        long cell[3];
        cell[dim] = i;
        cell[c0d] = c0;
        cell[c1d] = c1;
        int e = sweep_face(s, dim, i, cell, dx5, guards[c0 - lo]);
        if (e && !errs[c0 - lo]) errs[c0 - lo] = e;
      }
  });
  for (long v : guards) s.n_guard += v;
  for (int e : errs)
    if (e) return e;
  return E_OK;
}

void fluxes_at_faces(OSim& s) {
  for (int d = 0; d < 3; ++d) std::fill(s.flb[d].d.begin(), s.flb[d].d.end(), 0.0);
  for (int dim = 0; dim < 3; ++dim) {
    long n = s.ndim(dim);
    if (n <= 1) continue;
    int c0d, c1d;
    cross_dims(dim, c0d, c1d);
    par_for(s.nthreads, cross_lo(s, c0d), cross_hi(s, c0d), [&](long c0) {
      for (long c1 = cross_lo(s, c1d); c1 < cross_hi(s, c1d); ++c1)
        for (long i = 0; i <= n; ++i) {
          long cf[3], cm[3];
          cf[dim] = i;
          cf[c0d] = c0;
          cf[c1d] = c1;
          cm[0] = cf[0];
          cm[1] = cf[1];
          cm[2] = cf[2];
          cm[dim] = i - 1;
          double ap1 = s.sc(s_ahd_m(dim), cf[0], cf[1], cf[2]);
          double am1 = s.sc(s_ahd_m(dim), cm[0], cm[1], cm[2]);
          double rp1 = s.sc(s_arad_m(dim), cf[0], cf[1], cf[2]);
          double rm1 = s.sc(s_arad_m(dim), cm[0], cm[1], cm[2]);
          const double* pLl = s.pb_l[dim].at(cf[0], cf[1], cf[2]);
          const double* pRl = s.pb_r[dim].at(cf[0], cf[1], cf[2]);
          Geom geo;
          s.geom_face(cf[0], cf[1], cf[2], dim, geo);
          double uL[NV], uR[NV];
          p2u(pLl, uL, geo, s.sp.gam);
          p2u(pRl, uR, geo, s.sp.gam);
          double ag = kmath::fmax(ap1, am1);
          double agr = kmath::fmax(rp1, rm1);
          const double* fll = s.fl_l[dim].at(cf[0], cf[1], cf[2]);
          const double* flr = s.fl_r[dim].at(cf[0], cf[1], cf[2]);
          double* out = s.flb[dim].at(cf[0], cf[1], cf[2]);
          for (int iv = 0; iv < NV; ++iv) out[iv] = laxf(fll[iv], flr[iv], uL[iv], uR[iv], iv >= EE ? agr : ag);
        }
    });
  }
}

// ---- flux-CT (koral/sim/ct.zig:38) ------------------------------------------
long pin(long n, long i) { return n == 1 ? 0 : i; }
void flux_ct(OSim& s) {
  long nx = s.g.nx, ny = s.g.ny, nz = s.g.nz;
  double coef1 = (ny > 1 && nz > 1) ? 0.25 : 0.5;
  double coef2 = (nx > 1 && nz > 1) ? 0.25 : 0.5;
  double coef3 = (nx > 1 && ny > 1) ? 0.25 : 0.5;
  auto eidx = [&](long ix, long iy, long iz) { return (size_t)((iz * (ny + 1) + iy) * (nx + 1) + ix); };
  for (int c = 0; c < 3; ++c) s.emf[c].assign((nx + 1) * (ny + 1) * (nz + 1), 0.0);
  for (long iz = 0; iz <= nz; ++iz)
    for (long iy = 0; iy <= ny; ++iy)
      for (long ix = 0; ix <= nx; ++ix) {
        if (ny > 1 || nz > 1) {
          double sm = 0.0;
          if (ny > 1)
            sm += s.flb[1].at(pin(nx, ix), pin(ny, iy), pin(nz, iz))[B3] +
                  s.flb[1].at(pin(nx, ix), pin(ny, iy), pin(nz, iz - 1))[B3];
          if (nz > 1)
            sm -= s.flb[2].at(pin(nx, ix), pin(ny, iy), pin(nz, iz))[B2] +
                  s.flb[2].at(pin(nx, ix), pin(ny, iy - 1), pin(nz, iz))[B2];
          s.emf[0][eidx(ix, iy, iz)] = coef1 * sm;
        }
        if (nx > 1 || nz > 1) {
          double sm = 0.0;
          if (nz > 1)
            sm += s.flb[2].at(pin(nx, ix), pin(ny, iy), pin(nz, iz))[B1] +
                  s.flb[2].at(pin(nx, ix - 1), pin(ny, iy), pin(nz, iz))[B1];
          if (nx > 1)
            sm -= s.flb[0].at(ix, pin(ny, iy), pin(nz, iz))[B3] + s.flb[0].at(ix, pin(ny, iy), pin(nz, iz - 1))[B3];
          s.emf[1][eidx(ix, iy, iz)] = coef2 * sm;
        }
        if (nx > 1 || ny > 1) {
          double sm = 0.0;
          if (nx > 1)
            sm += s.flb[0].at(ix, pin(ny, iy), pin(nz, iz))[B2] + s.flb[0].at(ix, pin(ny, iy - 1), pin(nz, iz))[B2];
          if (ny > 1)
            sm -= s.flb[1].at(pin(nx, ix), pin(ny, iy), pin(nz, iz))[B1] +
                  s.flb[1].at(pin(nx, ix - 1), pin(ny, iy), pin(nz, iz))[B1];
          s.emf[2][eidx(ix, iy, iz)] = coef3 * sm;
        }
      }
  auto E = [&](int comp, long ix, long iy, long iz) { return s.emf[comp - 1][eidx(ix, iy, iz)]; };
  for (long iz = 0; iz <= nz; ++iz)
    for (long iy = 0; iy <= ny; ++iy)
      for (long ix = 0; ix <= nx; ++ix) {
        if (nx > 1 && iy < ny && iz < nz) {
          double* f = s.flb[0].at(ix, iy, iz);
          f[B1] = 0.0;
          f[B2] = 0.5 * (E(3, ix, iy, iz) + E(3, ix, iy + 1, iz));
          f[B3] = -0.5 * (E(2, ix, iy, iz) + E(2, ix, iy, iz + 1));
        }
        if (ny > 1 && ix < nx && iz < nz) {
          double* f = s.flb[1].at(ix, iy, iz);
          f[B1] = -0.5 * (E(3, ix, iy, iz) + E(3, ix + 1, iy, iz));
          f[B2] = 0.0;
          f[B3] = 0.5 * (E(1, ix, iy, iz) + E(1, ix, iy, iz + 1));
        }
        if (nz > 1 && ix < nx && iy < ny) {
          double* f = s.flb[2].at(ix, iy, iz);
          f[B1] = 0.5 * (E(2, ix, iy, iz) + E(2, ix + 1, iy, iz));
          f[B2] = -0.5 * (E(1, ix, iy, iz) + E(1, ix, iy + 1, iz));
          f[B3] = 0.0;
        }
      }
}

// ---- conserved update + metric source (sim.zig:1140,1542) --------------------
void metric_source(OSim& s, long ix, long iy, long iz, double ss[NV]) {
  Geom geo;
  s.geom(ix, iy, iz, geo);
  const double* pp = s.P(ix, iy, iz);
  double gdetu = geo.gdet;
  for (int i = 0; i < NV; ++i) ss[i] = 0.0;
  double tij[4][4], t[4][4], rup[4][4], rij[4][4];
  calc_tij(pp, geo, s.sp.gam, tij);
  lower_second(tij, geo, t);
  const double* k = s.kr(ix, iy, iz);
  calc_rij(pp, geo, rup);
  lower_second(rup, geo, rij);
  const int rows[4] = {UU, VX, VY, VZ}, rrows[4] = {EE, FX, FY, FZ};
  for (int a = 0; a < 4; ++a)
    for (int l = 0; l < 4; ++l)
      for (int nu = 0; nu < 4; ++nu) {
        ss[rows[nu]] += gdetu * t[a][l] * k[l * 16 + nu * 4 + a];
        ss[rrows[nu]] += gdetu * rij[a][l] * k[l * 16 + nu * 4 + a];
      }
}
void update_rows(OSim& s, double dtin) {
  const Grid& g = s.g;
  par_for(s.nthreads, 0, g.ny, [&](long iy) {
    for (long iz = 0; iz < g.nz; ++iz)
      for (long ix = 0; ix < g.nx; ++ix) {
        double ms[NV];
        metric_source(s, ix, iy, iz, ms);
        double dx = cell_size(g, ix, 0), dy = cell_size(g, iy, 1), dz = cell_size(g, iz, 2);
        double dt = dtin;
        const double* flxl = s.flb[0].at(ix, iy, iz);
        const double* flxr = s.flb[0].at(ix + 1, iy, iz);
        const double* flyl = s.flb[1].at(ix, iy, iz);
        const double* flyr = s.flb[1].at(ix, iy + 1, iz);
        const double* flzl = s.flb[2].at(ix, iy, iz);
        const double* flzr = s.flb[2].at(ix, iy, iz + 1);
        double* uu = s.U(ix, iy, iz);
        for (int iv = 0; iv < NV; ++iv) {
          double du = -(flxr[iv] - flxl[iv]) * dt / dx - (flyr[iv] - flyl[iv]) * dt / dy - (flzr[iv] - flzl[iv]) * dt / dz;
          uu[iv] = uu[iv] + du + ms[iv] * dt;
        }
      }
  });
}

int op_explicit(OSim& s, double dtin) {
  int e = calc_wavespeeds(s);
  if (e) return e;
  for (int d = 0; d < 3; ++d) {
    e = sweep(s, d);
    if (e) return e;
  }
  fluxes_at_faces(s);
  flux_ct(s);
  update_rows(s, dtin);
  return calc_u2p(s);
}

// ---- implicit operator (sim.zig:1715) ---------------------------------------
void op_implicit(OSim& s, double dtin) {
  const Grid& g = s.g;
  std::vector<long> nf(g.ny, 0), ni(g.ny, 0), ns(g.ny, 0);
  par_for(s.nthreads, 0, g.ny, [&](long iy) {
    if (s.polar_owns(iy)) return;
    for (long iz = 0; iz < g.nz; ++iz)
      for (long ix = 0; ix < g.nx; ++ix) {
        double uu[NV], pp[NV];
        for (int i = 0; i < NV; ++i) {
          uu[i] = s.U(ix, iy, iz)[i];
          pp[i] = s.P(ix, iy, iz)[i];
        }
        Geom geo;
        s.geom(ix, iy, iz, geo);
        ImplicitResult r = solve_implicit_lab(uu, pp, geo, dtin, s.sp.gam, s.sp.rp, s.sp.op, s.sp.ip);
        if (r.ok) {
          for (int i = 0; i < NV; ++i) {
            s.U(ix, iy, iz)[i] = uu[i];
            s.P(ix, iy, iz)[i] = pp[i];
          }
          s.flag(F_RADIMP, ix, iy, iz) = 0;
          ni[iy] += r.iters;
          ns[iy] += 1;
        } else {
          s.flag(F_RADIMP, ix, iy, iz) = -1;
          nf[iy] += 1;
        }
      }
  });
  for (long iy = 0; iy < g.ny; ++iy) {
    s.n_radimp_failures += nf[iy];
    s.n_radimp_iters += ni[iy];
    s.n_radimp_solves += ns[iy];
  }
}

// ---- stage arithmetic (sim.zig:1586-1709) -------------------------------------
void stage_deriv(OSim& s, std::vector<double>& dst, const std::vector<double>& a, const std::vector<double>& b, double delta) {
  double f1 = 1.0 / delta, f2 = -1.0 / delta;
  const Grid& g = s.g;
  for (long iz = 0; iz < g.nz; ++iz)
    for (long iy = 0; iy < g.ny; ++iy)
      for (long ix = 0; ix < g.nx; ++ix) {
        long c = s.ci(ix, iy, iz) * NV;
        for (int iv = 0; iv < NV; ++iv) dst[c + iv] = f1 * a[c + iv] + f2 * b[c + iv];
      }
}
void stage_combine(OSim& s, std::vector<double>& dst, const std::vector<double>& a, double f1, const std::vector<double>& b,
                   double f2, const std::vector<double>& cc) {
  const Grid& g = s.g;
  for (long iz = 0; iz < g.nz; ++iz)
    for (long iy = 0; iy < g.ny; ++iy)
      for (long ix = 0; ix < g.nx; ++ix) {
        long c = s.ci(ix, iy, iz) * NV;
        for (int iv = 0; iv < NV; ++iv) dst[c + iv] = a[c + iv] + f1 * b[c + iv] + f2 * cc[c + iv];
      }
}
void update_entropy(OSim& s) {
  const Grid& g = s.g;
  for (long iz = 0; iz < g.nz; ++iz)
    for (long iy = 0; iy < g.ny; ++iy)
      for (long ix = 0; ix < g.nx; ++ix) {
        double* pp = s.P(ix, iy, iz);
        pp[ENTR] = s_from_u(pp[RHO], pp[UU], s.sp.gam);
        Geom geo;
        s.geom(ix, iy, iz, geo);
        p2u_mhd(pp, s.U(ix, iy, iz), geo, s.sp.gam);
      }
}

// ---- radiative viscosity (koral/sim/rijvisc.zig) ------------------------------
int calc_shear_lab(OSim& s, long ix, long iy, long iz, double sh[4][4]) {
  const double* pp0 = s.P(ix, iy, iz);
  Geom geo;
  s.geom(ix, iy, iz, geo);
  double du[4][4] = {}, du2[4][4] = {};
  double ucon[4], ucov[4];
  ucon_ucov_from_prims(pp0[FX], pp0[FY], pp0[FZ], geo, ucon, ucov);
  long nd[3] = {s.g.nx, s.g.ny, s.g.nz};
  long nx = nd[0], ny = nd[1], nz = nd[2];
  for (int idim = 1; idim < 4; ++idim) {
    int dim = idim - 1;
    if (nd[dim] <= 1) continue;
    long cm[3] = {ix, iy, iz}, cp[3] = {ix, iy, iz};
    cm[dim] -= 1;
    cp[dim] += 1;
    const double* pm = s.P(cm[0], cm[1], cm[2]);
    const double* pq = s.P(cp[0], cp[1], cp[2]);
    Geom gm, gp;
    s.geom(cm[0], cm[1], cm[2], gm);
    s.geom(cp[0], cp[1], cp[2], gp);
    double umc[4], umv[4], upc[4], upv[4];
    ucon_ucov_from_prims(pm[FX], pm[FY], pm[FZ], gm, umc, umv);
    ucon_ucov_from_prims(pq[FX], pq[FY], pq[FZ], gp, upc, upv);
    double xm = gm.xx[idim], xc = geo.xx[idim], xp = gp.xx[idim];
    for (int i = 0; i < 4; ++i) {
      double dc = (upv[i] - umv[i]) / (xp - xm);
      double dr = (upv[i] - ucov[i]) / (xp - xc);
      double dl = (ucov[i] - umv[i]) / (xc - xm);
      double dc2 = (upc[i] - umc[i]) / (xp - xm);
      double dr2 = (upc[i] - ucon[i]) / (xp - xc);
      double dl2 = (ucon[i] - umc[i]) / (xc - xm);
      if ((ix < 0 && iy == 0 && iz == 0 && idim != 1) || (iy < 0 && ix == 0 && iz == 0 && idim != 2) ||
          (iz < 0 && ix == 0 && iy == 0 && idim != 3)) {
        du[i][idim] = dr;
        du2[i][idim] = dr2;
      } else if ((ix < 0 && iy == ny - 1 && iz == nz - 1 && idim != 1) ||
                 (iy < 0 && ix == nx - 1 && iz == nz - 1 && idim != 2) ||
                 (iz < 0 && ix == nx - 1 && iy == ny - 1 && idim != 3)) {
        du[i][idim] = dl;
        du2[i][idim] = dl2;
      } else if ((ix >= nx && iy == 0 && iz == 0 && idim != 1) || (iy >= ny && ix == 0 && iz == 0 && idim != 2) ||
                 (iz >= nz && ix == 0 && iy == 0 && idim != 3)) {
        du[i][idim] = dr;
        du2[i][idim] = dr2;
      } else if ((ix >= nx && iy == ny - 1 && iz == nz - 1 && idim != 1) ||
                 (iy >= ny && ix == nx - 1 && iz == nz - 1 && idim != 2) ||
                 (iz >= nz && ix == nx - 1 && iy == ny - 1 && idim != 3)) {
        du[i][idim] = dl;
        du2[i][idim] = dl2;
      } else {
        du[i][idim] = dc;
        du2[i][idim] = dc2;
      }
    }
  }
  shear_from_gradients(du, du2, ucon, ucov, geo, s.kr(ix, iy, iz), sh);
  return E_OK;
}
void calc_rijvisc_total(OSim& s, double global_dt) {
  std::fill(s.rijvisc.begin(), s.rijvisc.end(), 0.0);
  const Grid& g = s.g;
  long ylim = g.ny > 1 ? 1 : 0, xlim = g.nx > 1 ? 1 : 0, zlim = g.nz > 1 ? 1 : 0;
  double rhor = r_horizon_bl(s.sp.mp.a);
  par_for(s.nthreads, -ylim, g.ny + ylim, [&](long iy) {
    for (long iz = -zlim; iz < g.nz + zlim; ++iz)
      for (long ix = -xlim; ix < g.nx + xlim; ++ix) {
        if (s.is_corner(ix, iy, iz)) continue;
        const double* pp = s.P(ix, iy, iz);
        Geom geo;
        s.geom(ix, iy, iz, geo);
        double sl[4][4], shear[4][4];
        calc_shear_lab(s, ix, iy, iz, sl);
        raise_both(sl, geo, shear);
        double chi = calc_chi_slim(pp, geo, s.sp.gam, s.sp.op);
        double dx[3] = {cell_size(g, ix, 0) * kmath::sqrt(geo.gg[1][1]), cell_size(g, iy, 1) * kmath::sqrt(geo.gg[2][2]),
                        cell_size(g, iz, 2) * kmath::sqrt(geo.gg[3][3])};
        double mindx;
        if (g.ny == 1 && g.nz == 1) mindx = dx[0];
        else if (g.nz == 1) mindx = kmath::fmin(dx[0], dx[1]);
        else if (g.ny == 1) mindx = kmath::fmin(dx[0], dx[2]);
        else mindx = kmath::fmin(dx[0], kmath::fmin(dx[1], dx[2]));
        double nu = visc_coeff(chi, mindx, s.blg[s.ci(ix, iy, iz)].xx[1], rhor, s.sp.alpharadvisc, global_dt);
        double rv[4][4];
        rij_visc(nu, pp[EE], shear, geo, rv);
        double* out = &s.rijvisc[s.ci(ix, iy, iz) * 16];
        for (int i = 0; i < 4; ++i)
          for (int j = 0; j < 4; ++j) out[i * 4 + j] = rv[i][j];
      }
  });
}

// ---- mimic dynamo (koral/sim/dynamo.zig) --------------------------------------
void calc_scale_height(OSim& s) {
  const Grid& g = s.g;
  for (long ix = 0; ix < g.nx; ++ix) {
    double sigma = 0.0, sth = 0.0;
    for (long iy = 0; iy < g.ny; ++iy)
      for (long iz = 0; iz < g.nz; ++iz) {
        double gd = s.cgdet(ix, iy, iz);
        double th = s.blg[s.ci(ix, iy, iz)].xx[2];
        double rho = s.P(ix, iy, iz)[RHO];
        double dth = KP_PI / 2.0 - th;
        sigma += rho * gd;
        sth += rho * gd * dth * dth;
      }
    s.scaleth[ix] = (ix > 0) ? kmath::sqrt(sth / sigma) : sth;
  }
}
// ct.zig:224 cornerAverageA + :282 calcBfromACore (curl into vecpot slots 3..5)
void curl_from_a(OSim& s, const std::vector<double>& src, int srcnv, int base) {
  const Grid& g = s.g;
  long nx = g.nx, ny = g.ny, nz = g.nz;
  auto S = [&](int c, long ix, long iy, long iz) { return src[s.ci(ix, iy, iz) * srcnv + base + c]; };
  auto V = [&](int c, long ix, long iy, long iz) -> double& { return s.vecpot[s.ci(ix, iy, iz) * 6 + c]; };
  for (long iz = 0; iz <= nz; ++iz)
    for (long iy = 0; iy <= ny; ++iy)
      for (long ix = 0; ix <= nx; ++ix) {
        if (nz == 1 && iz > 0) continue;
        if (ny == 1 && iy > 0) continue;
        for (int c = 0; c < 3; ++c) {
          double a;
          if (ny == 1 && nz == 1) a = 1.0 / 2.0 * (S(c, ix, iy, iz) + S(c, ix - 1, iy, iz));
          else if (ny > 1 && nz == 1)
            a = 1.0 / 4.0 * (S(c, ix, iy, iz) + S(c, ix, iy - 1, iz) + S(c, ix - 1, iy, iz) + S(c, ix - 1, iy - 1, iz));
          else if (nz > 1 && ny == 1)
            a = 1.0 / 4.0 * (S(c, ix, iy, iz) + S(c, ix, iy, iz - 1) + S(c, ix - 1, iy, iz) + S(c, ix - 1, iy, iz - 1));
          else
            a = 1.0 / 8.0 *
                (S(c, ix, iy, iz) + S(c, ix, iy - 1, iz) + S(c, ix - 1, iy, iz) + S(c, ix - 1, iy - 1, iz) +
                 S(c, ix, iy, iz - 1) + S(c, ix, iy - 1, iz - 1) + S(c, ix - 1, iy, iz - 1) + S(c, ix - 1, iy - 1, iz - 1));
          V(c, ix, iy, iz) = a;
        }
      }
  for (long iz = 0; iz < nz; ++iz)
    for (long iy = 0; iy < ny; ++iy)
      for (long ix = 0; ix < nx; ++ix) {
        double dA[4][4] = {};
        if (nz == 1) {
          for (int c = 0; c < 3; ++c) {
            dA[c + 1][2] = -(V(c, ix, iy, iz) - V(c, ix, iy + 1, iz) + V(c, ix + 1, iy, iz) - V(c, ix + 1, iy + 1, iz)) /
                           (2.0 * cell_size(g, iy, 1));
            dA[c + 1][1] = -(V(c, ix, iy, iz) + V(c, ix, iy + 1, iz) - V(c, ix + 1, iy, iz) - V(c, ix + 1, iy + 1, iz)) /
                           (2.0 * cell_size(g, ix, 0));
            dA[c + 1][3] = 0.0;
          }
        } else {
          for (int c = 0; c < 3; ++c) {
            dA[c + 1][1] = (V(c, ix + 1, iy, iz) - V(c, ix, iy, iz) + V(c, ix + 1, iy + 1, iz) - V(c, ix, iy + 1, iz) +
                            V(c, ix + 1, iy, iz + 1) - V(c, ix, iy, iz + 1) + V(c, ix + 1, iy + 1, iz + 1) -
                            V(c, ix, iy + 1, iz + 1)) /
                           (4.0 * cell_size(g, ix, 0));
            dA[c + 1][2] = (V(c, ix, iy + 1, iz) - V(c, ix, iy, iz) + V(c, ix + 1, iy + 1, iz) - V(c, ix + 1, iy, iz) +
                            V(c, ix, iy + 1, iz + 1) - V(c, ix, iy, iz + 1) + V(c, ix + 1, iy + 1, iz + 1) -
                            V(c, ix + 1, iy, iz + 1)) /
                           (4.0 * cell_size(g, iy, 1));
            dA[c + 1][3] = (V(c, ix, iy, iz + 1) - V(c, ix, iy, iz) + V(c, ix + 1, iy, iz + 1) - V(c, ix + 1, iy, iz) +
                            V(c, ix, iy + 1, iz + 1) - V(c, ix, iy + 1, iz) + V(c, ix + 1, iy + 1, iz + 1) -
                            V(c, ix + 1, iy + 1, iz)) /
                           (4.0 * cell_size(g, iz, 2));
          }
        }
        double gdet = s.cgdet(ix, iy, iz);
        V(3, ix, iy, iz) = (dA[2][3] - dA[3][2]) / gdet;
        V(4, ix, iy, iz) = (dA[3][1] - dA[1][3]) / gdet;
        V(5, ix, iy, iz) = (dA[1][2] - dA[2][1]) / gdet;
      }
}
int mimic_dynamo(OSim& s, double dt) {
  const Grid& g = s.g;
  std::fill(s.dyn_a.begin(), s.dyn_a.end(), 0.0);
  long ylim = g.ny > 1 ? 1 : 0, xlim = g.nx > 1 ? 1 : 0, zlim = g.nz > 1 ? 1 : 0;
  double rhor = r_horizon_bl(s.sp.mp.a), risco = r_isco_bl(s.sp.mp.a);
  std::vector<int> errs(g.ny + 2, 0);
  par_for(s.nthreads, -ylim, g.ny + ylim, [&](long iy) {
    for (long iz = -zlim; iz < g.nz + zlim; ++iz)
      for (long ix = -xlim; ix < g.nx + xlim; ++ix) {
        Geom geo;
        s.geom(ix, iy, iz, geo);
        const Geom& gbl = s.blg[s.ci(ix, iy, iz)];
        double jac[4][4];
        s.jac_bl(ix, iy, iz, jac);
        double* pp = s.P(ix, iy, iz);
        double angle, bsq;
        int e = field_angle(geo, gbl, jac, pp, angle, bsq);
        if (e) {
          errs[iy + 1] = e;
          continue;
        }
        double r = gbl.xx[1], th = gbl.xx[2];
        if (r < 1.0001 * rhor) continue;
        double prermhd = (s.sp.gam - 1.0) * pp[UU];
        double ehat = -calc_ff_rtt(pp, geo, nullptr);
        prermhd += ehat / 3.0;
        long gix = std::min(std::max(ix, 0L), (long)g.nx - 1);
        DynamoOut o = dynamo_delta_a(s.sp.dp, s.sp.mp.a, dt, rhor, risco, r, th, pp[B3], bsq, angle, prermhd, geo.gg[3][3],
                                     s.scaleth[gix]);
        s.dyn_a[s.ci(ix, iy, iz) * 3 + 2] = o.aphi;
        if (s.sp.dp.dampbeta) pp[B3] = o.bphi;
      }
  });
  for (int e : errs)
    if (e) return e;
  curl_from_a(s, s.dyn_a, 3, 0);
  for (long iz = 0; iz < g.nz; ++iz)
    for (long iy = 0; iy < g.ny; ++iy)
      for (long ix = 0; ix < g.nx; ++ix) {
        double* pp = s.P(ix, iy, iz);
        const double* v = &s.vecpot[s.ci(ix, iy, iz) * 6];
        pp[B1] += v[3];
        pp[B2] += v[4];
        pp[B3] += v[5];
        Geom geo;
        s.geom(ix, iy, iz, geo);
        double uu[NV];
        p2u(pp, uu, geo, s.sp.gam);
        double* ud = s.U(ix, iy, iz);
        ud[B1] = uu[B1];
        ud[B2] = uu[B2];
        ud[B3] = uu[B3];
      }
  return E_OK;
}
int apply_dynamo(OSim& s, double dt) {
  calc_scale_height(s);
  int e = set_bc(s);
  if (e) return e;
  e = mimic_dynamo(s, dt);
  if (e) return e;
  return calc_u2p(s);
}

// ---- initTimestepGuess + step (sim.zig:693, :1792) ----------------------------
void init_timestep_guess(OSim& s) {
  const double ws = 10000.0;
  double tsd;
  if (s.g.nz > 1) tsd = ws / s.min_dx + ws / s.min_dy + ws / s.min_dz;
  else if (s.g.ny > 1) tsd = ws / s.min_dx + ws / s.min_dy;
  else tsd = ws / s.min_dx;
  tsd /= s.sp.tsteplim;
  s.tstepdenmax = tsd;
  s.tstepdenmin = tsd;
  for (long iz = 0; iz < s.g.nz; ++iz)
    for (long iy = 0; iy < s.g.ny; ++iy)
      for (long ix = 0; ix < s.g.nx; ++ix) {
        s.sc(S_TSTEPDEN, ix, iy, iz) = tsd;
        s.sc(S_CELLDT, ix, iy, iz) = 1.0 / tsd;
      }
}

int step(OSim& s, double forced_dt) {
  double t = s.t;
  s.time = t;
  s.own_dt = 1.0 / s.tstepdenmax;
  double dt = isnan(forced_dt) ? s.own_dt : forced_dt;
  s.dt = dt;
  long fail0 = s.n_radimp_failures;
  s.tstepdenmax = -1.0;
  s.tstepdenmin = 1.0e50;
  if (s.sp.radviscosity) calc_rijvisc_total(s, dt);
  const double gam_imex = KP_GAM_IMEX;
  for (long iz = 0; iz < s.g.nz; ++iz)
    for (long iy = 0; iy < s.g.ny; ++iy)
      for (long ix = 0; ix < s.g.nx; ++ix) s.sc(S_CELLDT, ix, iy, iz) = 1.0 / s.sc(S_TSTEPDEN, ix, iy, iz);
  int e;
  // 1st implicit
  s.ut0 = s.u;
  op_implicit(s, dt * gam_imex);
  stage_deriv(s, s.drt1, s.u, s.ut0, dt * gam_imex);
  // 1st explicit
  s.ut1 = s.u;
  if ((e = calc_u2p(s))) return e;
  do_correct(s);
  if ((e = set_bc(s))) return e;
  if ((e = op_explicit(s, dt))) return e;
  if (s.sp.dynamo && (e = apply_dynamo(s, dt))) return e;
  for (long iz = 0; iz < s.g.nz; ++iz)
    for (long iy = 0; iy < s.g.ny; ++iy)
      for (long ix = 0; ix < s.g.nx; ++ix) s.flag(F_ENTROPY3, ix, iy, iz) = s.flag(F_ENTROPY, ix, iy, iz);
  stage_deriv(s, s.dut1, s.u, s.ut1, dt);
  stage_combine(s, s.u, s.ut0, dt, s.dut1, dt * KP_ONE_M2GAM, s.drt1);
  // 2nd implicit
  s.uforget = s.u;
  if ((e = calc_u2p(s))) return e;
  do_correct(s);
  op_implicit(s, gam_imex * dt);
  stage_deriv(s, s.drt2, s.u, s.uforget, dt * gam_imex);
  // 2nd explicit
  s.ut2 = s.u;
  if ((e = calc_u2p(s))) return e;
  do_correct(s);
  if ((e = set_bc(s))) return e;
  if ((e = op_explicit(s, dt))) return e;
  if (s.sp.dynamo && (e = apply_dynamo(s, dt))) return e;
  stage_deriv(s, s.dut2, s.u, s.ut2, dt);
  stage_combine(s, s.u, s.ut0, dt / 2.0, s.dut1, dt / 2.0, s.dut2);
  stage_combine(s, s.u, s.u, dt / 2.0, s.drt1, dt / 2.0, s.drt2);
  if ((e = calc_u2p(s))) return e;
  do_correct(s);
  if ((e = set_bc(s))) return e;
  s.t = t + dt;
  update_entropy(s);
  s.n_radimp_fail_step = s.n_radimp_failures - fail0;
  s.nstep += 1;
  return E_OK;
}

// ---- PUFFY initial state (puffy.zig:873 initAllWith) -------------------------
// prepinit + p2u over the domain (puffy.zig:839), set_bc, calc_BfromA with
// overwrite (ct.zig:184: every cell, ghosts get the zero scratch B), set_bc,
// postinit (puffy.zig:892: global beta max over the domain, B scaled by
// sqrt(maxbeta/maxb), ghosts keep their unscaled B). Returns the error code;
// `fac` receives the beta normalization factor.
// stage 0: prepinit + p2u over the domain, then set_bc (A_phi in the B slots)
int init_stage0(OSim& s, double perturb, double perturb_rho, uint64_t seed) {
  const Grid& g = s.g;
  kcinit::PuffyPhysics ph;
  ph.mass = s.opt.mass;
  const double a = s.sp.mp.a;
  kcinit::TorusConsts tc = kcinit::torus_consts(a, ph);
  std::vector<int> errs(g.ny, 0);
  par_for(s.nthreads, 0, g.ny, [&](long iy) {
    for (long ix = 0; ix < g.nx; ++ix) {
      const Geom& gb0 = s.blg[s.ci(ix, iy, 0)];
      kcinit::DsVels dv = kcinit::init_dsandvels(gb0.xx[1], gb0.xx[2], a, tc, ph);
      for (long iz = 0; iz < g.nz; ++iz) {
        Geom geo;
        s.geom(ix, iy, iz, geo);
        const Geom& gbl = s.blg[s.ci(ix, iy, iz)];
        double jac[4][4];
        double xbl[4] = {0.0, gbl.xx[1], gbl.xx[2], gbl.xx[3]};
        dxdx(xbl, BL, MKS2, s.sp.mp, jac);
        double pp[NV];
        int e = kcinit::prep_init_cell(geo, gbl, jac, dv, s.sp, ph, perturb, perturb_rho, seed, pp);
        if (e) {
          errs[iy] = e;
          continue;
        }
        pp[ENTR] = s_from_u(pp[RHO], pp[UU], s.sp.gam);
        double* P = s.P(ix, iy, iz);
        for (int i = 0; i < NV; ++i) P[i] = pp[i];
        p2u(P, s.U(ix, iy, iz), geo, s.sp.gam);
      }
    }
  });
  for (int e : errs)
    if (e) return e;
  return set_bc(s);
}
// stage 1: calc_BfromA with overwrite (ghosts take the zero scratch), set_bc
int init_stage1(OSim& s) {
  const Grid& g = s.g;
  std::fill(s.vecpot.begin(), s.vecpot.end(), 0.0);
  curl_from_a(s, s.p, NV, B1);
  for (long iz = -g.ngz; iz < g.nz + g.ngz; ++iz)
    for (long iy = -g.ngy; iy < g.ny + g.ngy; ++iy)
      for (long ix = -g.ngx; ix < g.nx + g.ngx; ++ix) {
        double* pp = s.P(ix, iy, iz);
        const double* v = &s.vecpot[s.ci(ix, iy, iz) * 6];
        pp[B1] = v[3];
        pp[B2] = v[4];
        pp[B3] = v[5];
        Geom geo;
        s.geom(ix, iy, iz, geo);
        p2u(pp, s.U(ix, iy, iz), geo, s.sp.gam);
      }
  return set_bc(s);
}
// stage 2: postinit beta normalization of the domain B (ghosts keep theirs)
void init_stage2(OSim& s, double& fac) {
  const Grid& g = s.g;
  kcinit::PuffyPhysics ph;
  double maxb = 0.0;
  for (long iz = 0; iz < g.nz; ++iz)
    for (long iy = 0; iy < g.ny; ++iy)
      for (long ix = 0; ix < g.nx; ++ix) {
        const double* pp = s.P(ix, iy, iz);
        Geom geo;
        s.geom(ix, iy, iz, geo);
        double ucon[4], ucov[4], bcon[4], bcov[4], bsq;
        ucon_ucov_from_prims(pp[VX], pp[VY], pp[VZ], geo, ucon, ucov);
        double B[3] = {pp[B1], pp[B2], pp[B3]};
        bcon_bcov_bsq(B, ucon, ucov, geo, bcon, bcov, bsq);
        double pmag = bsq / 2.0;
        double ptot = (s.sp.gam - 1.0) * pp[UU];
        ptot += -calc_ff_rtt(pp, geo, nullptr) / 3.0;
        if (pmag / ptot > maxb) maxb = pmag / ptot;
      }
  fac = kmath::sqrt(ph.maxbeta / maxb);
  for (long iz = 0; iz < g.nz; ++iz)
    for (long iy = 0; iy < g.ny; ++iy)
      for (long ix = 0; ix < g.nx; ++ix) {
        double* pp = s.P(ix, iy, iz);
        pp[B1] *= fac;
        pp[B2] *= fac;
        pp[B3] *= fac;
        Geom geo;
        s.geom(ix, iy, iz, geo);
        p2u(pp, s.U(ix, iy, iz), geo, s.sp.gam);
      }
}

// ---- diagnostics (koral/io/scalars.zig, koral/io/dump.zig:358-410) -----------
// r_BL of a radial index (scalars.zig:47 radiusBL)
double radius_bl(const OSim& s, long ix) {
  double xx[4] = {0.0, grid_xc(s.g, ix), grid_yc(s.g, 0), grid_zc(s.g, 0)}, o[4];
  mks2_to_bl(xx, s.sp.mp, o);
  return o[1];
}
// scalars.zig:58 radialShellIndex
long radial_shell_index(const OSim& s, double radius) {
  for (long ix = 0; ix < s.g.nx; ++ix)
    if (radius_bl(s, ix) > radius) return ix;
  return s.g.nx - 1;
}
// BL theta / phi widths of a cell (scalars.zig:190,199)
double bl_theta_width(const OSim& s, long ix, long iy, long iz) {
  double a[4] = {0.0, grid_xc(s.g, ix), grid_yl(s.g, iy), grid_zc(s.g, iz)}, oa[4];
  double b[4] = {0.0, grid_xc(s.g, ix), grid_yl(s.g, iy + 1), grid_zc(s.g, iz)}, ob[4];
  mks2_to_bl(a, s.sp.mp, oa);
  mks2_to_bl(b, s.sp.mp, ob);
  return kmath::fabs(ob[2] - oa[2]);
}
double bl_phi_width(const OSim& s, long ix, long iy, long iz) {
  double a[4] = {0.0, grid_xc(s.g, ix), grid_yc(s.g, iy), grid_zl(s.g, iz)}, oa[4];
  double b[4] = {0.0, grid_xc(s.g, ix), grid_yc(s.g, iy), grid_zl(s.g, iz + 1)}, ob[4];
  mks2_to_bl(a, s.sp.mp, oa);
  mks2_to_bl(b, s.sp.mp, ob);
  return kmath::fabs(ob[3] - oa[3]);
}
// dump.zig:383 scalarRow with scalars.zig:225 globalScalars (serial order)
int scalar_row(OSim& s, double dt, double r_lum, double r_scale, kc_scalar_row& row) {
  const Grid& g = s.g;
  const double pi = KP_PI;
  const bool twod = g.nz == 1;
  long ix_h = radial_shell_index(s, r_horizon_bl(s.sp.mp.a));
  long ix_l = radial_shell_index(s, r_lum);
  // collectDiag (dump.zig:358)
  long n_nan = 0, n_hd = 0;
  for (long iz = 0; iz < g.nz; ++iz)
    for (long iy = 0; iy < g.ny; ++iy)
      for (long ix = 0; ix < g.nx; ++ix) {
        const double* pp = s.P(ix, iy, iz);
        for (int iv = 0; iv < NV; ++iv)
          if (!kmath::isfinite(pp[iv])) {
            n_nan += 1;
            break;
          }
        if (s.flag(F_HD, ix, iy, iz) != 0) n_hd += 1;
      }
  // totalMass (scalars.zig:78)
  double phifac = g.nz > 1 ? 2.0 * pi / (g.maxz - g.minz) : 1.0;
  double mass = 0.0;
  for (long iz = 0; iz < g.nz; ++iz)
    for (long iy = 0; iy < g.ny; ++iy)
      for (long ix = 0; ix < g.nx; ++ix) {
        double dx = cell_size(g, ix, 0), dy = cell_size(g, iy, 1), dz = cell_size(g, iz, 2) * phifac;
        mass += s.P(ix, iy, iz)[RHO] * dx * dy * dz * s.cgdet(ix, iy, iz);
      }
  // mdot (scalars.zig:106)
  double mdot = 0.0;
  for (long iz = 0; iz < g.nz; ++iz)
    for (long iy = 0; iy < g.ny; ++iy) {
      const double* pp = s.P(ix_h, iy, iz);
      Geom geo;
      s.geom(ix_h, iy, iz, geo);
      double vcon[4] = {0.0, pp[VX], pp[VY], pp[VZ]}, ucon[4];
      int e = convert(vcon, VELR, VEL4, geo, RECOMPUTE_UT, ucon);
      if (e) return e;
      double rhouconr = pp[RHO] * ucon[1];
      double dy = cell_size(g, iy, 1);
      double dz = twod ? 2.0 * pi : cell_size(g, iz, 2) * (2.0 * pi / (g.maxz - g.minz));
      mdot += geo.gdet * rhouconr * dy * dz;
    }
  // lum, type 1 (scalars.zig:136)
  double radlum = 0.0, totallum = 0.0;
  for (long iz = 0; iz < g.nz; ++iz)
    for (long iy = 0; iy < g.ny; ++iy) {
      double pp[NV];
      for (int i = 0; i < NV; ++i) pp[i] = s.P(ix_l, iy, iz)[i];
      Geom geo;
      s.geom(ix_l, iy, iz, geo);
      const Geom& gbl = s.blg[s.ci(ix_l, iy, iz)];
      double jac[4][4];
      s.jac_bl(ix_l, iy, iz, jac);
      int e = trans_pmhd_coco_j(pp, geo, gbl, jac, pp);
      if (!e) e = trans_prad_coco_j(pp, geo, gbl, jac, pp);
      if (e) return e;
      double dth = bl_theta_width(s, ix_l, iy, iz);
      double dph = twod ? 2.0 * pi : bl_phi_width(s, ix_l, iy, iz) * (2.0 * pi / (g.maxz - g.minz));
      double vcon[4] = {0.0, pp[VX], pp[VY], pp[VZ]}, ucon[4];
      if ((e = convert(vcon, VELR, VEL4, gbl, RECOMPUTE_UT, ucon))) return e;
      double rhour = pp[RHO] * ucon[1];
      double tup[4][4], tij[4][4], rup[4][4], rij[4][4];
      calc_tij(pp, gbl, s.sp.gam, tup);
      lower_second(tup, gbl, tij);
      double trt = tij[1][0];
      calc_rij(pp, gbl, rup);
      lower_second(rup, gbl, rij);
      double rrt = -rij[1][0];
      if (rrt < 0.0) rrt = 0.0;
      radlum += gbl.gdet * rrt * dth * dph;
      totallum += gbl.gdet * (rhour + trt + rrt) * dth * dph;
    }
  // scale height (dynamo.zig:239 parts, :267 finalize)
  long ix_s = radial_shell_index(s, r_scale);
  double sig = 0.0, sth = 0.0;
  for (long iy = 0; iy < g.ny; ++iy)
    for (long iz = 0; iz < g.nz; ++iz) {
      double gd = s.cgdet(ix_s, iy, iz);
      double th = s.blg[s.ci(ix_s, iy, iz)].xx[2];
      double rho = s.P(ix_s, iy, iz)[RHO];
      double dth = pi / 2.0 - th;
      sig += rho * gd;
      sth += rho * gd * dth * dth;
    }
  // maxPmagPtot (scalars.zig:276)
  double maxb = 0.0;
  for (long iz = 0; iz < g.nz; ++iz)
    for (long iy = 0; iy < g.ny; ++iy)
      for (long ix = 0; ix < g.nx; ++ix) {
        const double* pp = s.P(ix, iy, iz);
        Geom geo;
        s.geom(ix, iy, iz, geo);
        double ucon[4], ucov[4], bcon[4], bcov[4], bsq;
        ucon_ucov_from_prims(pp[VX], pp[VY], pp[VZ], geo, ucon, ucov);
        double B[3] = {pp[B1], pp[B2], pp[B3]};
        bcon_bcov_bsq(B, ucon, ucov, geo, bcon, bcov, bsq);
        double pmag = bsq / 2.0;
        double ptot = (s.sp.gam - 1.0) * pp[UU];
        ptot += (-calc_ff_rtt(pp, geo, nullptr)) / 3.0;
        if (pmag / ptot > maxb) maxb = pmag / ptot;
      }
  row.t = s.t;
  row.dt = dt;
  row.nstep = s.nstep;
  row.mass = mass;
  row.mdot = -mdot;
  row.radlum = radlum;
  row.totallum = totallum;
  row.scaleheight = ix_s > 0 ? kmath::sqrt(sth / sig) : sth;
  row.max_pmag_ptot = maxb;
  row.n_hd_fixup = n_hd;
  row.n_radimp_fail = s.n_radimp_failures;
  row.n_nan = n_nan;
  row.n_floorguard = s.n_guard;
  return E_OK;
}

int init_puffy(OSim& s, double perturb, double perturb_rho, uint64_t seed, double& fac) {
  int e = init_stage0(s, perturb, perturb_rho, seed);
  if (!e) e = init_stage1(s);
  if (!e) init_stage2(s, fac);
  return e;
}

// A bare simulation of an nx x ny x nz grid with ng ghosts (extents
// [minx, maxx] x ...): sizes and the zeroed arrays the per-function passes
// below touch, with sqrt(-g) = 1 (the Minkowski grids of the reference's
// flux_ct and calc_BfromA goldens).
void bare_sim(OSim& s, int nx, int ny, int nz, int ng, const double ext[6]) {
  s.g = grid_init(nx, ny, nz, ng, ext[0], ext[1], ext[2], ext[3], ext[4], ext[5]);
  s.sx = nx + 2 * s.g.ngx;
  s.sy = ny + 2 * s.g.ngy;
  s.sz = nz + 2 * s.g.ngz;
  s.nc = s.sx * s.sy * s.sz;
  s.p.assign(s.nc * NV, 0.0);
  s.vecpot.assign(s.nc * 6, 0.0);
  s.cg.assign(s.nc * 20, 0.0);
  for (long c = 0; c < s.nc; ++c) s.cg[c * 20 + 19] = 1.0;
  for (int d = 0; d < 3; ++d) s.flb[d].init(s.g, d);
}

}  // namespace

// ---- ctypes surface ----------------------------------------------------------
extern "C" {

void orc_options_puffy(kc_options* o) { options_puffy(o); }
void orc_grid_puffy(int nx, int ny, int nz, kc_grid* g) { grid_puffy(nx, ny, nz, g); }

void* orc_sim_create(const kc_grid* kg, const kc_options* opt, int nthreads) {
  if (validate_config(*kg, *opt)) return nullptr;
  OSim* s = new OSim();
  s->g = grid_init(kg->nx, kg->ny, kg->nz, kg->ng, kg->minx, kg->maxx, kg->miny, kg->maxy, kg->minz, kg->maxz);
  s->opt = *opt;
  params_from_options(*opt, s->sp);
  s->nthreads = nthreads > 0 ? nthreads : 1;
  const Grid& g = s->g;
  s->sx = g.nx + 2 * g.ngx;
  s->sy = g.ny + 2 * g.ngy;
  s->sz = g.nz + 2 * g.ngz;
  s->nc = s->sx * s->sy * s->sz;
  build_cache(*s);
  size_t nf = s->nc * NV;
  for (auto* f : {&s->p, &s->u, &s->ut0, &s->ut1, &s->ut2, &s->dut1, &s->dut2, &s->drt1, &s->drt2, &s->uforget, &s->u_bak,
                  &s->p_bak})
    f->assign(nf, 0.0);
  for (int d = 0; d < 3; ++d) {
    s->pb_l[d].init(g, d);
    s->pb_r[d].init(g, d);
    s->fl_l[d].init(g, d);
    s->fl_r[d].init(g, d);
    s->flb[d].init(g, d);
  }
  s->scal.assign(s->nc * NSCAL, 0.0);
  s->flags.assign(s->nc * NFL, 0);
  for (int c = 0; c < 3; ++c) s->emf[c].assign((g.nx + 1) * (g.ny + 1) * (g.nz + 1), 0.0);
  s->vecpot.assign(s->nc * 6, 0.0);
  s->rijvisc.assign(s->nc * 16, 0.0);
  s->dyn_a.assign(s->nc * 3, 0.0);
  s->scaleth.assign(g.nx, 0.0);
  // set_grid min-size scan with C's mdx quirk (sim.zig:443)
  double mdx = -1, mdy = -1, mdz = -1;
  for (long ix = 0; ix < g.nx; ++ix)
    for (long iy = 0; iy < g.ny; ++iy)
      for (long iz = 0; iz < g.nz; ++iz) {
        double dx = cell_size(g, ix, 0), dy = cell_size(g, iy, 1), dz = cell_size(g, iz, 2);
        if (dx < mdx || mdx < 0) mdx = dx;
        if (dy < mdx || mdy < 0) mdy = dy;
        if (dz < mdx || mdz < 0) mdz = dz;
      }
  s->min_dx = mdx;
  s->min_dy = mdy;
  s->min_dz = mdz;
  return s;
}
void orc_sim_destroy(void* h) { delete (OSim*)h; }
long orc_sim_ncell(void* h) { return ((OSim*)h)->nc; }
void orc_sim_set_threads(void* h, int n) { ((OSim*)h)->nthreads = n > 0 ? n : 1; }
void orc_sim_set_prims(void* h, const double* p) {
  OSim* s = (OSim*)h;
  memcpy(s->p.data(), p, s->p.size() * 8);
}
void orc_sim_set_cons(void* h, const double* u) {
  OSim* s = (OSim*)h;
  memcpy(s->u.data(), u, s->u.size() * 8);
}
void orc_sim_set_flags(void* h, const int* f) {
  OSim* s = (OSim*)h;
  memcpy(s->flags.data(), f, s->flags.size() * 4);
}
void orc_sim_get_prims(void* h, double* p) {
  OSim* s = (OSim*)h;
  memcpy(p, s->p.data(), s->p.size() * 8);
}
void orc_sim_get_cons(void* h, double* u) {
  OSim* s = (OSim*)h;
  memcpy(u, s->u.data(), s->u.size() * 8);
}
void orc_sim_get_flags(void* h, int* f) {
  OSim* s = (OSim*)h;
  memcpy(f, s->flags.data(), s->flags.size() * 4);
}
void orc_sim_set_counters(void* h, const kc_counters* c) {
  OSim* s = (OSim*)h;
  s->t = c->t;
  s->dt = c->dt;
  s->own_dt = c->own_dt;
  s->tstepdenmax = c->tstepdenmax;
  s->tstepdenmin = c->tstepdenmin;
  s->nstep = c->nstep;
  s->n_radimp_failures = c->n_radimp_failures;
  s->n_radimp_fail_step = c->n_radimp_fail_step;
  s->n_radimp_iters = c->n_radimp_iters;
  s->n_radimp_solves = c->n_radimp_solves;
  s->n_guard = c->n_guard_recoveries;
}
void orc_sim_get_counters(void* h, kc_counters* c) {
  OSim* s = (OSim*)h;
  c->t = s->t;
  c->dt = s->dt;
  c->own_dt = s->own_dt;
  c->tstepdenmax = s->tstepdenmax;
  c->tstepdenmin = s->tstepdenmin;
  c->nstep = s->nstep;
  c->n_radimp_failures = s->n_radimp_failures;
  c->n_radimp_fail_step = s->n_radimp_fail_step;
  c->n_radimp_iters = s->n_radimp_iters;
  c->n_radimp_solves = s->n_radimp_solves;
  c->n_guard_recoveries = s->n_guard;
}
void orc_sim_init_timestep_guess(void* h) { init_timestep_guess(*(OSim*)h); }
int orc_sim_set_bc(void* h) { return set_bc(*(OSim*)h); }
int orc_sim_calc_u2p(void* h) { return calc_u2p(*(OSim*)h); }
int orc_sim_step(void* h, double forced_dt) { return step(*(OSim*)h, forced_dt); }
int orc_sim_init_puffy(void* h, double perturb, double perturb_rho, unsigned long long seed, double* fac) {
  return init_puffy(*(OSim*)h, perturb, perturb_rho, seed, *fac);
}
int orc_sim_scalar_row(void* h, double dt, double r_lum, double r_scale, kc_scalar_row* row) {
  return scalar_row(*(OSim*)h, dt, r_lum, r_scale, *row);
}
// one stage of the init sequence on the current state (0: prepinit + set_bc,
// 1: B from A + set_bc, 2: beta normalization), for the C init goldens
int orc_sim_init_stage(void* h, int stage, double perturb, double perturb_rho, unsigned long long seed, double* fac) {
  OSim& s = *(OSim*)h;
  if (stage == 0) return init_stage0(s, perturb, perturb_rho, seed);
  if (stage == 1) return init_stage1(s);
  if (stage == 2) {
    init_stage2(s, *fac);
    return 0;
  }
  return -1;
}
// single passes, for localizing engine-vs-oracle differences
int orc_sim_phase(void* h, int phase, double dt) {
  OSim& s = *(OSim*)h;
  switch (phase) {
    case 0: return calc_wavespeeds(s);
    case 1: {
      for (int d = 0; d < 3; ++d) {
        int e = sweep(s, d);
        if (e) return e;
      }
      fluxes_at_faces(s);
      return 0;
    }
    case 2: flux_ct(s); return 0;
    case 3: update_rows(s, dt); return 0;
    case 4: return calc_u2p(s);
    case 5: op_implicit(s, dt); return 0;
    case 6: calc_rijvisc_total(s, dt); return 0;
    case 7: return apply_dynamo(s, dt);
    case 8: do_correct(s); return 0;
    case 9: return op_explicit(s, dt);
    default: return -1;
  }
}
// KDMP v2 (dump.zig:100 serializePrimDump, :143 loadPrimDump): serial loops
// over the domain, iz slowest, iv fastest; the load stores p verbatim and u =
// p2u(p) per cell (sim.zig:672 initCell). The caller adopts t / nstep.
long orc_sim_kdmp_size(void* h) {
  OSim& s = *(OSim*)h;
  return KC_KDMP_HEADER_SIZE + kdump::body_bytes(s.g.nx, s.g.ny, s.g.nz, NV);
}
int orc_sim_kdmp_write(void* h, unsigned out_idx, unsigned char* out, long cap) {
  OSim& s = *(OSim*)h;
  if (cap < orc_sim_kdmp_size(h)) return KC_ERR_INVALID_CONFIG;
  kc_dump_header hd = {(uint32_t)s.g.nx, (uint32_t)s.g.ny, (uint32_t)s.g.nz, (uint32_t)NV, s.t, (uint64_t)s.nstep,
                       out_idx};
  long w = kdump::write_header(hd, out);
  for (long iz = 0; iz < s.g.nz; ++iz)
    for (long iy = 0; iy < s.g.ny; ++iy)
      for (long ix = 0; ix < s.g.nx; ++ix)
        for (int iv = 0; iv < NV; ++iv) {
          memcpy(out + w, &s.P(ix, iy, iz)[iv], 8);
          w += 8;
        }
  return KC_OK;
}
int orc_sim_kdmp_load(void* h, const unsigned char* b, long len, kc_dump_header* out) {
  OSim& s = *(OSim*)h;
  kc_dump_header hd;
  int st = kdump::parse_header(b, len, hd);
  if (st) return st;
  if (hd.nx != (uint32_t)s.g.nx || hd.ny != (uint32_t)s.g.ny || hd.nz != (uint32_t)s.g.nz || hd.nv != (uint32_t)NV)
    return KC_ERR_KDMP_DIM_MISMATCH;
  if (len < orc_sim_kdmp_size(h)) return KC_ERR_KDMP_TRUNCATED;
  long r = KC_KDMP_HEADER_SIZE;
  for (long iz = 0; iz < s.g.nz; ++iz)
    for (long iy = 0; iy < s.g.ny; ++iy)
      for (long ix = 0; ix < s.g.nx; ++ix) {
        double pp[NV];
        for (int iv = 0; iv < NV; ++iv) {
          memcpy(&pp[iv], b + r, 8);
          r += 8;
        }
        for (int iv = 0; iv < NV; ++iv) s.P(ix, iy, iz)[iv] = pp[iv];
        p2u_cell(s, ix, iy, iz);
      }
  if (out) *out = hd;
  return KC_OK;
}
// read-only views of internal arrays for parity tests
int orc_sim_get_array(void* h, int which, double* out) {
  OSim& s = *(OSim*)h;
  const std::vector<double>* v = nullptr;
  switch (which) {
    case 0: v = &s.scal; break;
    case 1: v = &s.rijvisc; break;
    case 2: v = &s.flb[0].d; break;
    case 3: v = &s.flb[1].d; break;
    case 4: v = &s.flb[2].d; break;
    case 5: v = &s.scaleth; break;
    case 6: v = &s.cg; break;
    case 7: v = &s.kris; break;
    default: return -1;
  }
  memcpy(out, v->data(), v->size() * 8);
  return (int)v->size();
}

// ct.fluxCt (koral/sim/ct.zig:38) on given face fluxes: fb[dim] holds the
// B1, B2, B3 rows of the dim-direction face fluxes in the FaceStore layout
// (koral/sim/storage.zig:62: one extra slice in its own dimension, ghosts
// included, the three components fastest); rebuilt in place. NULL for an
// inactive direction. The grid extents do not enter.
int orc_flux_ct(int nx, int ny, int nz, int ng, double* fbx, double* fby, double* fbz) {
  OSim s;
  const double ext[6] = {0.0, 1.0, 0.0, 1.0, 0.0, 1.0};
  bare_sim(s, nx, ny, nz, ng, ext);
  double* fb[3] = {fbx, fby, fbz};
  for (int d = 0; d < 3; ++d) {
    if (!fb[d]) continue;
    size_t nfc = s.flb[d].d.size() / NV;
    for (size_t f = 0; f < nfc; ++f)
      for (int k = 0; k < 3; ++k) s.flb[d].d[f * NV + B1 + k] = fb[d][f * 3 + k];
  }
  flux_ct(s);
  for (int d = 0; d < 3; ++d) {
    if (!fb[d]) continue;
    size_t nfc = s.flb[d].d.size() / NV;
    for (size_t f = 0; f < nfc; ++f)
      for (int k = 0; k < 3; ++k) fb[d][f * 3 + k] = s.flb[d].d[f * NV + B1 + k];
  }
  return 0;
}
// calc_BfromA (koral/sim/ct.zig:184, overwrite) on a sqrt(-g) = 1 grid: A_i
// of every cell, ghosts included (cell-major, 3 fastest, the Field order of
// koral/field.zig), to B^i of the domain cells in the same layout (ghost
// entries are zeroed, as the overwrite leaves them before set_bc).
int orc_b_from_a(int nx, int ny, int nz, int ng, const double* ext, const double* a, double* b) {
  OSim s;
  bare_sim(s, nx, ny, nz, ng, ext);
  for (long c = 0; c < s.nc; ++c)
    for (int k = 0; k < 3; ++k) s.p[c * NV + B1 + k] = a[c * 3 + k];
  curl_from_a(s, s.p, NV, B1);
  for (long c = 0; c < s.nc; ++c)
    for (int k = 0; k < 3; ++k) b[c * 3 + k] = s.vecpot[c * 6 + 3 + k];
  return 0;
}
}
