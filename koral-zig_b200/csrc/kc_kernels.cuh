// kc_kernels.cuh — the sm_100a kernels of one RK2IMEX step. Each kernel is
// one pass of the reference's Sim.step (koral/sim.zig:1792) over a grid of
// cells, faces or corners, calling the shared per-point restatement; the
// arithmetic of every point is the reference's, so the plain FP64 build
// (--fmad=false) reproduces the CPU oracle bit for bit.
#pragma once
#include "kc_dev.cuh"
#include "kc_implicit_sm.cuh"
#include "kc_mixed.cuh"
#include "kc_mlp.cuh"

// Resident blocks of 128 per SM that the register budgets of the u2p, radiative
// viscosity, dynamo and boundary kernels must allow (1: uncapped). Measured on
// the wedge: 3 (168 registers) makes the dynamo 4% faster and the boundary kernel
// 3% slower; the viscosity kernel is indifferent. The u2p kernel with its
// inversion inlined: 4 (128 registers, 16 warps per SM) 4% faster than 3.
#ifndef KC_U2P_MIN_BLOCKS
#define KC_U2P_MIN_BLOCKS 4
#endif
#ifndef KC_RIJVISC_MIN_BLOCKS
#define KC_RIJVISC_MIN_BLOCKS 1
#endif
#ifndef KC_DYNAMO_MIN_BLOCKS
#define KC_DYNAMO_MIN_BLOCKS 3
#endif
#ifndef KC_BC_MIN_BLOCKS
#define KC_BC_MIN_BLOCKS 1
#endif

namespace kc {

__device__ __forceinline__ void set_err(DevScalars* sc, int code, long long cell) {
  if (atomicCAS(&sc->err, 0, code) == 0) sc->err_cell = cell;
}
__device__ __forceinline__ unsigned long long dbits(double x) { return (unsigned long long)__double_as_longlong(x); }

// ---- generic cell ranges -----------------------------------------------------
// A launch covers ix in [x0, x0+nx), iy in [y0, y0+ny), iz in [z0, z0+nz); the
// thread's x coordinate walks ix so neighbouring lanes touch neighbouring cells.
struct Range {
  long x0, y0, z0, nx, ny, nz;
};
// The domain cell of this thread with phi (z) fastest: the cells of a warp then
// share (r, theta), and on an axisymmetric torus they take nearly the same path
// through a per-cell solver (the implicit solve, the u2p inversion).
__device__ __forceinline__ bool domain_cell_phi_fastest(const DGrid& gr, long& ix, long& iy, long& iz) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)gr.nx * gr.ny * gr.nz) return false;
  iz = t % gr.nz;
  long q = t / gr.nz;
  ix = q % gr.nx;
  iy = q / gr.nx;
  return true;
}
__device__ __forceinline__ bool range_cell(const Range& r, long& ix, long& iy, long& iz) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long n = r.nx * r.ny * r.nz;
  if (t >= n) return false;
  ix = r.x0 + t % r.nx;
  long q = t / r.nx;
  iy = r.y0 + q % r.ny;
  iz = r.z0 + q / r.ny;
  return true;
}

// ---- AoS <-> SoA transposes at the host boundary ---------------------------------
__global__ void k_aos_to_soa(const double* __restrict__ aos, double* __restrict__ soa, long nc, int nv) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nc * nv) return;
  long c = t / nv;
  int v = (int)(t % nv);
  soa[(long)v * nc + c] = aos[t];
}
__global__ void k_soa_to_aos(const double* __restrict__ soa, double* __restrict__ aos, long nc, int nv) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nc * nv) return;
  long c = t / nv;
  int v = (int)(t % nv);
  aos[t] = soa[(long)v * nc + c];
}
// ---- the metric cache, built on the device (koral/metric/precompute.zig:175) ----
// The same per-point code as the host build of the oracle (dual-number metric,
// MODYFIKUJKRZYSIE correction, BL geometry and Jacobians), one thread per cell
// (ghosts included) or per face. Symmetry of the packed layouts is checked
// bitwise and reported through *asym.
struct CacheOut {
  double *cgc, *cGc, *kr, *jbl, *blg, *jb2m;
  double *fgc[3], *fGc[3];
  long nf[3], ngh;
  int* asym;
};
__global__ void __launch_bounds__(128) k_cache_centers(Grid g, MetricParams mp, long sx, long sy, long sz, CacheOut o) {
  long nc = sx * sy * sz;
  long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  long ix = c % sx - g.ngx, iy = (c / sx) % sy - g.ngy, iz = c / (sx * sy) - g.ngz;
  double x[4] = {0.0, grid_xc(g, ix), grid_yc(g, iy), grid_zc(g, iz)};
  CoordData d;
  metric_compute(MKS2, mp, x, d);
  apply_kris_correction(MKS2, mp, g, d, ix, iy, iz);
  int asym = 0;
  for (int i = 0; i < 4; ++i)
    for (int j = i; j < 4; ++j) {
      o.cgc[(long)sym10(i, j) * nc + c] = d.gcov[i][j];
      if (dbits(d.gcov[i][j]) != dbits(d.gcov[j][i])) asym = 1;
    }
  o.cgc[10L * nc + c] = d.gdet;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) o.cGc[(long)(i * 4 + j) * nc + c] = d.gcon[i][j];
  o.cGc[16L * nc + c] = d.gttpert;
  for (int l = 0; l < 4; ++l)
    for (int m = 0; m < 4; ++m)
      for (int n = m; n < 4; ++n) {
        o.kr[(long)(l * 10 + sym10(m, n)) * nc + c] = d.kris[l][m][n];
        if (dbits(d.kris[l][m][n]) != dbits(d.kris[l][n][m])) asym = 1;
      }
  double m4[4][4];
  dxdx(x, MKS2, BL, mp, m4);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) o.jbl[(long)(i * 4 + j) * nc + c] = m4[i][j];
  Geom gb;
  geometry_bl_at(g, mp, ix, iy, iz, gb);
  for (int i = 0; i < 4; ++i)
    for (int j = i; j < 4; ++j) {
      o.blg[(long)sym10(i, j) * nc + c] = gb.gg[i][j];
      if (dbits(gb.gg[i][j]) != dbits(gb.gg[j][i])) asym = 1;
    }
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) o.blg[(long)(10 + i * 4 + j) * nc + c] = gb.GG[i][j];
  o.blg[26L * nc + c] = gb.xx[1];
  o.blg[27L * nc + c] = gb.xx[2];
  if (ix >= g.nx) {
    long gi = (ix - g.nx) + (long)g.ngx * ((iy + g.ngy) + sy * (iz + g.ngz));
    double xbl[4] = {0.0, gb.xx[1], gb.xx[2], gb.xx[3]};
    dxdx(xbl, BL, MKS2, mp, m4);
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) o.jb2m[(long)(i * 4 + j) * o.ngh + gi] = m4[i][j];
  }
  if (asym) atomicOr(o.asym, 1);
}
__device__ __forceinline__ void cache_put_face(const CacheOut& o, int dim, long f, const CoordData& d) {
  long nf = o.nf[dim];
  for (int i = 0; i < 4; ++i)
    for (int j = i; j < 4; ++j) o.fgc[dim][(long)sym10(i, j) * nf + f] = d.gcov[i][j];
  o.fgc[dim][10L * nf + f] = d.gdet;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) o.fGc[dim][(long)(i * 4 + j) * nf + f] = d.gcon[i][j];
  o.fGc[dim][16L * nf + f] = d.gttpert;
}
// faces of direction `dim` at lower corners (ix, iy, iz) over (sx+1)(sy+1)(sz+1)
__global__ void __launch_bounds__(128) k_cache_faces(Grid g, MetricParams mp, long sx, long sy, long sz, int dim,
                                                     CacheOut o) {
  long n = (sx + 1) * (sy + 1) * (sz + 1);
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  long jx = t % (sx + 1), jy = (t / (sx + 1)) % (sy + 1), jz = t / ((sx + 1) * (sy + 1));
  long ix = jx - g.ngx, iy = jy - g.ngy, iz = jz - g.ngz;
  long nxh = g.nx + g.ngx, nyh = g.ny + g.ngy, nzh = g.nz + g.ngz;
  CoordData d;
  if (dim == 0 && iy < nyh && iz < nzh) {
    double x[4] = {0.0, grid_xl(g, ix), grid_yc(g, iy), grid_zc(g, iz)};
    metric_compute(MKS2, mp, x, d);
    cache_put_face(o, 0, jx + jy * (sx + 1) + jz * sy * (sx + 1), d);
  }
  if (dim == 1 && ix < nxh && iz < nzh) {
    double x[4] = {0.0, grid_xc(g, ix), grid_yl(g, iy), grid_zc(g, iz)};
    metric_compute(MKS2, mp, x, d);
    cache_put_face(o, 1, jx + jy * sx + jz * (sy + 1) * sx, d);
  }
  if (dim == 2 && ix < nxh && iy < nyh) {
    double x[4] = {0.0, grid_xc(g, ix), grid_yc(g, iy), grid_zl(g, iz)};
    metric_compute(MKS2, mp, x, d);
    cache_put_face(o, 2, jx + jy * sx + jz * sy * sx, d);
  }
}

// KDMP body (dump.zig:122 serializePrimBody): the domain primitives in
// [iz][iy][ix][iv] order, one thread per output double (coalesced writes)
__global__ void k_domain_to_kdmp(DevState s, double* __restrict__ body) {
  long nx = s.gr.nx, ny = s.gr.ny, nd = nx * ny * s.gr.nz;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nd * NV) return;
  long d = t / NV;
  int v = (int)(t % NV);
  long c = cidx(s.gr, d % nx, (d / nx) % ny, d / (nx * ny));
  body[t] = s.p[(long)v * s.gr.nc + c];
}
// KDMP load (dump.zig:160 loadPrimBody + sim.zig:672 initCell): p stored as
// read, u = p2u(p) with the cell's geometry, one thread per domain cell
__global__ void __launch_bounds__(128) k_kdmp_to_domain(DevState s, const double* __restrict__ body, double gam) {
  long nx = s.gr.nx, ny = s.gr.ny, nd = nx * ny * s.gr.nz;
  long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= nd) return;
  long ix = d % nx, iy = (d / nx) % ny, iz = d / (nx * ny);
  long c = cidx(s.gr, ix, iy, iz);
  double pp[NV], uu[NV];
  for (int v = 0; v < NV; ++v) pp[v] = body[d * NV + v];
  Geom g;
  geom_cell(s, ix, iy, iz, g);
  p2u(pp, uu, g, gam);
  store_cell(s.p, s.gr.nc, c, pp);
  store_cell(s.u, s.gr.nc, c, uu);
}
__global__ void k_flags_to_soa(const int* __restrict__ aos, int* __restrict__ soa, long nc) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nc * 6) return;
  soa[(t % 6) * nc + t / 6] = aos[t];
}
__global__ void k_flags_to_aos(const int* __restrict__ soa, int* __restrict__ aos, long nc) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nc * 6) return;
  aos[t] = soa[(t % 6) * nc + t / 6];
}

// ---- stage arithmetic (koral/sim.zig:1586-1709) ------------------------------
// dst = (1/delta) a + (-1/delta) b over the domain
__global__ void k_stage_deriv(DevState s, double* dst, const double* a, const double* b, int delta_slot) {
  const double delta = s.coef[delta_slot];
  Range r = {0, 0, 0, s.gr.nx, s.gr.ny, s.gr.nz};
  long ix, iy, iz;
  if (!range_cell(r, ix, iy, iz)) return;
  long c = cidx(s.gr, ix, iy, iz);
  double f1 = 1.0 / delta, f2 = -1.0 / delta;
  long nc = s.gr.nc;
#pragma unroll
  for (int iv = 0; iv < NV; ++iv) dst[iv * nc + c] = f1 * a[iv * nc + c] + f2 * b[iv * nc + c];
}
// dst = a + f1 b + f2 cc over the domain
__global__ void k_stage_combine(DevState s, double* dst, const double* a, int f1_slot, const double* b, int f2_slot,
                                const double* cc) {
  const double f1 = s.coef[f1_slot], f2 = s.coef[f2_slot];
  Range r = {0, 0, 0, s.gr.nx, s.gr.ny, s.gr.nz};
  long ix, iy, iz;
  if (!range_cell(r, ix, iy, iz)) return;
  long c = cidx(s.gr, ix, iy, iz);
  long nc = s.gr.nc;
#pragma unroll
  for (int iv = 0; iv < NV; ++iv) dst[iv * nc + c] = a[iv * nc + c] + f1 * b[iv * nc + c] + f2 * cc[iv * nc + c];
}
// flags entropy3 = entropy (C copy_entropycount)
__global__ void k_copy_entropy_count(DevState s) {
  Range r = {0, 0, 0, s.gr.nx, s.gr.ny, s.gr.nz};
  long ix, iy, iz;
  if (!range_cell(r, ix, iy, iz)) return;
  long c = cidx(s.gr, ix, iy, iz);
  s.flags[2 * s.gr.nc + c] = s.flags[0 * s.gr.nc + c];
}
// C update_entropy (koral/sim.zig:1683)
__global__ void __launch_bounds__(128) k_update_entropy(DevState s, double gam) {
  Range r = {0, 0, 0, s.gr.nx, s.gr.ny, s.gr.nz};
  long ix, iy, iz;
  if (!range_cell(r, ix, iy, iz)) return;
  long c = cidx(s.gr, ix, iy, iz), nc = s.gr.nc;
  double pp[NV], uu[NV];
  load_cell(s.p, nc, c, pp);
  load_cell(s.u, nc, c, uu);
  pp[ENTR] = s_from_u(pp[RHO], pp[UU], gam);
  s.p[ENTR * nc + c] = pp[ENTR];
  Geom g;
  geom_cell(s, ix, iy, iz, g);
  p2u_mhd(pp, uu, g, gam);
#pragma unroll
  for (int iv = 0; iv < 9; ++iv) s.u[iv * nc + c] = uu[iv];
}

// ---- u2p (koral/sim.zig:924-1000) --------------------------------------------
__global__ void __launch_bounds__(128, KC_U2P_MIN_BLOCKS) k_u2p(DevState s, DevScalars* sc, double gam, const __grid_constant__ FloorParams fl,
                                             const __grid_constant__ RadParams rp,
                                             int polar_nc, int phi_fastest) {
  Range r = {0, 0, 0, s.gr.nx, s.gr.ny, s.gr.nz};
  long ix, iy, iz;
  if (phi_fastest) {
    if (!domain_cell_phi_fastest(s.gr, ix, iy, iz)) return;
  } else if (!range_cell(r, ix, iy, iz)) {
    return;
  }
  long c = cidx(s.gr, ix, iy, iz), nc = s.gr.nc;
  double uu[NV], pp[NV];
  load_cell(s.u, nc, c, uu);
  load_cell(s.p, nc, c, pp);
  s.flags[0 * nc + c] = 0;
  s.flags[1 * nc + c] = 0;
  Geom g;
  geom_cell<true>(s, ix, iy, iz, g);  // read once: evict-first in L2
  bool polar = polar_nc > 0 && (iy < polar_nc || iy > s.gr.ny - polar_nc - 1);
  if (polar) {
    double gdetu_inv = 1.0 / g.gdet;
    s.p[B1 * nc + c] = uu[B1] * gdetu_inv;
    s.p[B2 * nc + c] = uu[B2] * gdetu_inv;
    s.p[B3 * nc + c] = uu[B3] * gdetu_inv;
    s.flags[3 * nc + c] = 0;
    s.flags[4 * nc + c] = 0;
    return;
  }
  // the inversion, the M1 closure and the floors inlined: measured faster than
  // their out-of-line forms, whose array arguments went through the call frame
  U2pMhdRes res = u2p_mhd_t<true>(uu, pp, g, gam, fl);
  if (res.entropy_used) s.flags[0 * nc + c] = 1;
  U2pRadRes rr = u2p_rad_inl(uu, pp, g, rp);
  int gc = 0;
  check_floors_mhd_inl(pp, g, gam, fl, gc);
  if (gc) atomicAdd(&sc->n_guard, (unsigned long long)gc);
  check_floors_rad(pp, g, rp);
  store_cell<true>(s.p, nc, c, pp);
  s.flags[3 * nc + c] = res.fixup ? 1 : 0;
  s.flags[4 * nc + c] = rr.corrected ? -1 : 0;
  if (res.fixup) atomicOr(&sc->any_hd, 1);
}

// cell_fixup(FIXUP_U2PMHD), pass 1: flagged cells average their non-flagged
// in-domain neighbours into the staging buffers (koral/sim.zig:1067)
__global__ void __launch_bounds__(128) k_fixup_hd(DevState s, DevScalars* sc, double gam, int polar_nc) {
  if (!sc->any_hd) return;
  Range r = {0, 0, 0, s.gr.nx, s.gr.ny, s.gr.nz};
  long ix, iy, iz;
  if (!range_cell(r, ix, iy, iz)) return;
  long nc = s.gr.nc, c = cidx(s.gr, ix, iy, iz);
  if (polar_nc > 0 && (iy < polar_nc || iy > s.gr.ny - polar_nc - 1)) return;
  const int* fhd = s.flags + 3 * nc;
  if (fhd[c] == 0) return;
  long nx = s.gr.nx, ny = s.gr.ny, nz = s.gr.nz;
  long nb[6][3] = {{ix - 1, iy, iz}, {ix + 1, iy, iz}, {ix, iy - 1, iz}, {ix, iy + 1, iz}, {ix, iy, iz - 1}, {ix, iy, iz + 1}};
  long ncells[6];
  int in_n = 0;
  for (int k = 0; k < 6; ++k) {
    if (nb[k][0] < 0 || nb[k][0] >= nx || nb[k][1] < 0 || nb[k][1] >= ny || nb[k][2] < 0 || nb[k][2] >= nz) continue;
    long cn = cidx(s.gr, nb[k][0], nb[k][1], nb[k][2]);
    if (fhd[cn] != 0) continue;
    ncells[in_n++] = cn;
  }
  bool enough = (nz == 1 && ny == 1 && in_n >= 1) || (nz == 1 && in_n >= 2) || (ny == 1 && in_n >= 2) || in_n >= 3;
  if (!enough) return;
  double pp[NV];
  load_cell(s.p, nc, c, pp);
  for (int iv = 0; iv < NV; ++iv) {
    if (iv != RHO && iv < B1) {
      double sum = 0.0;
      for (int k = 0; k < in_n; ++k) sum += s.p[iv * nc + ncells[k]];
      pp[iv] = sum / (double)in_n;
    }
  }
  Geom g;
  geom_cell(s, ix, iy, iz, g);
  double uu[NV];
  p2u(pp, uu, g, gam);
  store_cell(s.fix_p, nc, c, pp);
  store_cell(s.fix_u, nc, c, uu);
  // mark the cell as staged; the bit keeps the flag nonzero for the
  // neighbour tests of concurrent threads and is cleared in pass 2
  s.flags[3 * nc + c] = fhd[c] | 0x40000000;
}
// pass 2: copy the staged cells back
__global__ void k_fixup_apply(DevState s, DevScalars* sc) {
  if (!sc->any_hd) return;
  Range r = {0, 0, 0, s.gr.nx, s.gr.ny, s.gr.nz};
  long ix, iy, iz;
  if (!range_cell(r, ix, iy, iz)) return;
  long nc = s.gr.nc, c = cidx(s.gr, ix, iy, iz);
  int f = s.flags[3 * nc + c];
  if (!(f & 0x40000000)) return;
  s.flags[3 * nc + c] = f & ~0x40000000;
#pragma unroll
  for (int iv = 0; iv < NV; ++iv) {
    s.p[iv * nc + c] = s.fix_p[iv * nc + c];
    s.u[iv * nc + c] = s.fix_u[iv * nc + c];
  }
}

// ---- boundary conditions (koral/sim/bc.zig, puffy.zig:1080) ------------------
__device__ int puffy_bc_cell(const DevState& s, long ix, long iy, long iz, int face, double pp[NV]) {
  const long nx = s.gr.nx, ny = s.gr.ny, nc = s.gr.nc;
  if (face == 1) {
    load_cell(s.p, nc, cidx(s.gr, nx - 1, iy, iz), pp);
    Geom geo, gbl;
    geom_cell(s, ix, iy, iz, geo);
    long c = cidx(s.gr, ix, iy, iz);
    geom_bl(s, c, gbl);
    double jm2b[4][4], jb2m[4][4];
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) jm2b[a][b] = s.jbl[(long)(a * 4 + b) * nc + c];
    long gi = (ix - nx) + (long)s.gr.ngx * ((iy + s.gr.ngy) + s.gr.sy * (iz + s.gr.ngz));
    long ngh = (long)s.gr.ngx * s.gr.sy * s.gr.sz;
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) jb2m[a][b] = s.jb2m[(long)(a * 4 + b) * ngh + gi];
    int e = trans_pmhd_coco_j(pp, geo, gbl, jm2b, pp);
    if (e) return e;
    double rghost = gbl.xx[1];
    double rbound = s.blg[26L * nc + cidx(s.gr, nx - 1, iy, iz)];
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
  if (face == 0) {
    load_cell(s.p, nc, cidx(s.gr, 0, iy, iz), pp);
    return E_OK;
  }
  long iiy = (face == 2) ? -iy - 1 : ny - (iy - ny) - 1;
  load_cell(s.p, nc, cidx(s.gr, ix, iiy, iz), pp);
  pp[VY] = -pp[VY];
  pp[B2] = -pp[B2];
  pp[FY] = -pp[FY];
  return E_OK;
}

__device__ void bc_cell(const DevState& s, DevScalars* sc, long ix, long iy, long iz, int face, const int bc[3],
                        double gam) {
  int axis = face / 2;
  int kind = bc[axis];
  long nc = s.gr.nc;
  double pp[NV];
  if (kind == KC_BC_PUFFY) {
    int e = puffy_bc_cell(s, ix, iy, iz, face, pp);
    if (e) {
      set_err(sc, e, cidx(s.gr, ix, iy, iz));
      return;
    }
  } else {
    long iix = ix, iiy = iy, iiz = iz, nx = s.gr.nx, ny = s.gr.ny, nz = s.gr.nz;
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
        if (ny < s.gr.ng) iiy = 0;
      } else {
        if (iy < 0) iiy = 0;
        if (iy > ny - 1) iiy = ny - 1;
      }
    } else {
      if (kind == KC_BC_PERIODIC) {
        if (iz < 0) iiz = iz + nz;
        if (iz > nz - 1) iiz = iz - nz;
        if (nz < s.gr.ng) iiz = 0;
      } else {
        if (iz < 0) iiz = 0;
        if (iz > nz - 1) iiz = nz - 1;
      }
    }
    load_cell(s.p, nc, cidx(s.gr, iix, iiy, iiz), pp);
  }
  Geom g;
  geom_cell(s, ix, iy, iz, g);
  double uu[NV];
  p2u(pp, uu, g, gam);
  long c = cidx(s.gr, ix, iy, iz);
  store_cell(s.p, nc, c, pp);
  store_cell(s.u, nc, c, uu);
}

struct BcArgs {
  int bc[3];
  double gam;
};
// ghost faces of one axis; thread t -> (ghost layer i, two transverse indices)
__global__ void __launch_bounds__(128, KC_BC_MIN_BLOCKS) k_bc_faces(DevState s, DevScalars* sc, BcArgs a, int axis) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long nx = s.gr.nx, ny = s.gr.ny, nz = s.gr.nz;
  if (axis == 0) {
    long ng = s.gr.ngx;
    long n = 2 * ng * ny * nz;
    if (t >= n) return;
    long side = t % 2, q = t / 2;
    long i = 1 + q % ng;
    q /= ng;
    long iy = q % ny, iz = q / ny;
    if (side == 0) bc_cell(s, sc, -i, iy, iz, 0, a.bc, a.gam);
    else bc_cell(s, sc, nx - 1 + i, iy, iz, 1, a.bc, a.gam);
  } else if (axis == 1) {
    long ng = s.gr.ngy;
    long n = 2 * ng * nx * nz;
    if (t >= n) return;
    long ix = t % nx, q = t / nx;
    long side = q % 2;
    q /= 2;
    long i = 1 + q % ng, iz = q / ng;
    if (side == 0) bc_cell(s, sc, ix, -i, iz, 2, a.bc, a.gam);
    else bc_cell(s, sc, ix, ny - 1 + i, iz, 3, a.bc, a.gam);
  } else {
    long ng = s.gr.ngz;
    long n = 2 * ng * nx * ny;
    if (t >= n) return;
    long ix = t % nx, q = t / nx;
    long iy = q % ny;
    q /= ny;
    long side = q % 2, i = 1 + q / 2;
    if (side == 0) bc_cell(s, sc, ix, iy, -i, 4, a.bc, a.gam);
    else bc_cell(s, sc, ix, iy, nz - 1 + i, 5, a.bc, a.gam);
  }
}

__device__ void p2u_cell(const DevState& s, long ix, long iy, long iz, double gam) {
  long nc = s.gr.nc, c = cidx(s.gr, ix, iy, iz);
  double pp[NV], uu[NV];
  load_cell(s.p, nc, c, pp);
  Geom g;
  geom_cell(s, ix, iy, iz, g);
  p2u(pp, uu, g, gam);
  store_cell(s.u, nc, c, uu);
}
__device__ void copy_p_cell(const DevState& s, long dx, long dy, long dz, long sx_, long sy_, long sz_) {
  long nc = s.gr.nc, d = cidx(s.gr, dx, dy, dz), c = cidx(s.gr, sx_, sy_, sz_);
#pragma unroll
  for (int iv = 0; iv < NV; ++iv) s.p[iv * nc + d] = s.p[iv * nc + c];
}
__device__ void avg_p_cell(const DevState& s, const long d[3], const long a[3], const long b[3]) {
  long nc = s.gr.nc, cd = cidx(s.gr, d[0], d[1], d[2]), ca = cidx(s.gr, a[0], a[1], a[2]),
       cb = cidx(s.gr, b[0], b[1], b[2]);
  double v[NV];
  for (int iv = 0; iv < NV; ++iv) v[iv] = 0.5 * (s.p[iv * nc + ca] + s.p[iv * nc + cb]);
  store_cell(s.p, nc, cd, v);
}

// 2D corner surfaces + diagonals (bc.zig:256): one thread per corner, the
// strip -> diagonal order inside a corner kept serial
__global__ void k_corners_2d(DevState s, BcArgs a) {
  int corner = threadIdx.x;
  if (corner >= 4) return;
  long nx = s.gr.nx, ny = s.gr.ny, ng = s.gr.ng;
  bool px = a.bc[0] == KC_BC_PERIODIC, py = a.bc[1] == KC_BC_PERIODIC;
  bool xh = corner & 1, yh = corner & 2;
  for (long i = 0; i < ng - 1; ++i) {
    long ax = xh ? nx + i + 1 : -ng + i, ay = yh ? ny : -1, asy = yh ? ny - 1 : 0;
    copy_p_cell(s, ax, ay, 0, ax, asy, 0);
    p2u_cell(s, ax, ay, 0, a.gam);
    long bx = xh ? nx : -1, bsx = xh ? nx - 1 : 0, by = yh ? ny + i + 1 : -ng + i;
    copy_p_cell(s, bx, by, 0, bsx, by, 0);
    p2u_cell(s, bx, by, 0, a.gam);
  }
  long s1[4], s2[4], d1[3], d2[3];
  if (!xh && !yh) {
    long t1[4] = {-1, 0, 0, -1}, t2[4] = {-2, -1, -1, -2};
    if (py) { t1[0] = -1; t1[1] = ny - 1; t1[2] = -1; t1[3] = ny - 1; t2[0] = -2; t2[1] = ny - 2; t2[2] = -2; t2[3] = ny - 2; }
    if (px) { t1[0] = nx - 1; t1[1] = -1; t1[2] = nx - 1; t1[3] = -1; t2[0] = nx - 2; t2[1] = -2; t2[2] = nx - 2; t2[3] = -2; }
    for (int k = 0; k < 4; ++k) { s1[k] = t1[k]; s2[k] = t2[k]; }
    d1[0] = -1; d1[1] = -1; d2[0] = -2; d2[1] = -2;
  } else if (!xh && yh) {
    long t1[4] = {-1, ny - 1, 0, ny}, t2[4] = {-2, ny, -1, ny + 1};
    if (py) { t1[0] = -1; t1[1] = 0; t1[2] = -1; t1[3] = 0; t2[0] = -2; t2[1] = 1; t2[2] = -2; t2[3] = 1; }
    if (px) { t1[0] = nx - 1; t1[1] = ny; t1[2] = nx - 1; t1[3] = ny; t2[0] = nx - 2; t2[1] = ny + 1; t2[2] = nx - 2; t2[3] = ny + 1; }
    for (int k = 0; k < 4; ++k) { s1[k] = t1[k]; s2[k] = t2[k]; }
    d1[0] = -1; d1[1] = ny; d2[0] = -2; d2[1] = ny + 1;
  } else if (xh && !yh) {
    long t1[4] = {nx - 1, -1, nx, 0}, t2[4] = {nx, -2, nx + 1, -1};
    if (py) { t1[0] = nx; t1[1] = ny - 1; t1[2] = nx; t1[3] = ny - 1; t2[0] = nx + 1; t2[1] = ny - 2; t2[2] = nx + 1; t2[3] = ny - 2; }
    if (px) { t1[0] = 0; t1[1] = -1; t1[2] = 0; t1[3] = -1; t2[0] = 1; t2[1] = -2; t2[2] = 1; t2[3] = -2; }
    for (int k = 0; k < 4; ++k) { s1[k] = t1[k]; s2[k] = t2[k]; }
    d1[0] = nx; d1[1] = -1; d2[0] = nx + 1; d2[1] = -2;
  } else {
    long t1[4] = {nx - 1, ny, nx, ny - 1}, t2[4] = {nx, ny + 1, nx + 1, ny};
    if (py) { t1[0] = nx; t1[1] = 0; t1[2] = nx; t1[3] = 0; t2[0] = nx + 1; t2[1] = 1; t2[2] = nx + 1; t2[3] = 1; }
    if (px) { t1[0] = 0; t1[1] = ny; t1[2] = 0; t1[3] = ny; t2[0] = 1; t2[1] = ny + 1; t2[2] = 1; t2[3] = ny + 1; }
    for (int k = 0; k < 4; ++k) { s1[k] = t1[k]; s2[k] = t2[k]; }
    d1[0] = nx; d1[1] = ny; d2[0] = nx + 1; d2[1] = ny + 1;
  }
  d1[2] = 0;
  d2[2] = 0;
  long a1[3] = {s1[0], s1[1], 0}, b1[3] = {s1[2], s1[3], 0};
  avg_p_cell(s, d1, a1, b1);
  p2u_cell(s, d1[0], d1[1], 0, a.gam);
  long a2[3] = {s2[0], s2[1], 0}, b2[3] = {s2[2], s2[3], 0};
  avg_p_cell(s, d2, a2, b2);
  p2u_cell(s, d2[0], d2[1], 0, a.gam);
}

// one group of four 3D edge tubes (bc.zig:404): thread -> (tube, slice)
// The four edge tubes of the (pa, pb) plane along pc (bc.zig:420), in two
// phases. Phase 0: per (tube, cc), the 2 (ng-1) copies from the face ghosts and
// the (g1, g1) average, all independent (each writes its own cell and reads
// face ghosts only), one thread each. Phase 1: the (g2, g2) average, which
// reads two cells phase 0 wrote. Same values as one thread doing them in order.
__device__ __forceinline__ void tube_cell(int pa, int pb, int pc, long av, long bv, long cv, long o[3]) {
  o[pa] = av;
  o[pb] = bv;
  o[pc] = cv;
}
__global__ void k_edge_tubes(DevState s, double gam, int pa, int pb, int pc, int phase) {
  long dims[3] = {s.gr.nx, s.gr.ny, s.gr.nz};
  long ng = s.gr.ng;
  long nslice = dims[pc] + 2 * ng;
  long ntask = phase == 0 ? 2 * (ng - 1) + 1 : 1;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 4 * nslice * ntask) return;
  long task = t % ntask, q = t / ntask;
  int tube = (int)(q / nslice);
  long cc = -ng + q % nslice;
  bool a_hi = tube & 2, b_hi = tube & 1;
  long na = dims[pa], nb = dims[pb];
  long a_edge = a_hi ? na - 1 : 0, a_g1 = a_hi ? na : -1, a_g2 = a_hi ? na + 1 : -2;
  long b_edge = b_hi ? nb - 1 : 0, b_g1 = b_hi ? nb : -1, b_g2 = b_hi ? nb + 1 : -2;
  long d[3], x[3], y[3];
  if (phase == 1) {
    tube_cell(pa, pb, pc, a_g2, b_g2, cc, d);
    tube_cell(pa, pb, pc, a_g2, b_g1, cc, x);
    tube_cell(pa, pb, pc, a_g1, b_g2, cc, y);
    avg_p_cell(s, d, x, y);
  } else if (task == 2 * (ng - 1)) {
    tube_cell(pa, pb, pc, a_g1, b_g1, cc, d);
    tube_cell(pa, pb, pc, a_g1, b_edge, cc, x);
    tube_cell(pa, pb, pc, a_edge, b_g1, cc, y);
    avg_p_cell(s, d, x, y);
  } else {
    long i = task >> 1;
    long a_out = a_hi ? na + i + 1 : -ng + i;
    long b_out = b_hi ? nb + i + 1 : -ng + i;
    if ((task & 1) == 0) {
      tube_cell(pa, pb, pc, a_out, b_g1, cc, d);
      tube_cell(pa, pb, pc, a_out, b_edge, cc, x);
    } else {
      tube_cell(pa, pb, pc, a_g1, b_out, cc, d);
      tube_cell(pa, pb, pc, a_edge, b_out, cc, x);
    }
    copy_p_cell(s, d[0], d[1], d[2], x[0], x[1], x[2]);
  }
  p2u_cell(s, d[0], d[1], d[2], gam);
}
// the 8 corner cubes (bc.zig:457)
// Every cube cell copies its cube's domain corner cell, which no cube writes,
// so the 8 x ng^3 cells are independent: one thread each.
__global__ void k_corner_cubes(DevState s, double gam) {
  long ng = s.gr.ng;
  long per = ng * ng * ng;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 8 * per) return;
  int cube = (int)(t / per);
  t %= per;
  long nx = s.gr.nx, ny = s.gr.ny, nz = s.gr.nz;
  bool xh = cube & 1, yh = cube & 2, zh = cube & 4;
  long ix = (xh ? nx : -ng) + t % ng, iy = (yh ? ny : -ng) + (t / ng) % ng, iz = (zh ? nz : -ng) + t / (ng * ng);
  copy_p_cell(s, ix, iy, iz, xh ? nx - 1 : 0, yh ? ny - 1 : 0, zh ? nz - 1 : 0);
  p2u_cell(s, ix, iy, iz, gam);
}

// ---- polar axis overwrite (koral/sim/polaraxis.zig:124) -----------------------
__global__ void __launch_bounds__(128) k_polar_correct(DevState s, double gam, int ncp) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long nx = s.gr.nx, ny = s.gr.ny, nz = s.gr.nz, nc = s.gr.nc;
  if (t >= nx * nz * 2 * ncp) return;
  long ix = t % nx, q = t / nx;
  long k = q % (2 * ncp), iz = q / (2 * ncp);
  long ic = k / 2;
  long iy = (k % 2 == 0) ? ic : ny - 1 - ic;
  long iysrc = (iy < ncp) ? ncp : ny - 1 - ncp;
  double thaxis = grid_yl(s.gr.g, (iy < ncp) ? 0 : ny);
  double fac = kmath::fabs((grid_yc(s.gr.g, iy) - thaxis) / (grid_yc(s.gr.g, iysrc) - thaxis));
  long c = cidx(s.gr, ix, iy, iz), cs = cidx(s.gr, ix, iysrc, iz);
  double pp[NV], pps[NV];
  load_cell(s.p, nc, c, pp);
  load_cell(s.p, nc, cs, pps);
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
  Geom g;
  geom_cell(s, ix, iy, iz, g);
  double uu[NV];
  p2u(pp, uu, g, gam);
  store_cell(s.p, nc, c, pp);
  store_cell(s.u, nc, c, uu);
}

// ---- wavespeeds + CFL reduction (koral/sim.zig:747-886) ----------------------
struct WsArgs {
  double gam, tsteplim;
  OpacParams op;
  int damp_nc;
};
// 4 resident blocks (128 registers): measured 6% faster than 158 registers
__global__ void __launch_bounds__(128, 4) k_wavespeeds(DevState s, DevScalars* sc, const __grid_constant__ WsArgs a) {
  const Grid& g = s.gr.g;
  bool act[3] = {s.gr.nx > 1, s.gr.ny > 1, s.gr.nz > 1};
  long lx = act[0], ly = act[1], lz = act[2];
  Range r = {-lx, -ly, -lz, s.gr.nx + 2 * lx, s.gr.ny + 2 * ly, s.gr.nz + 2 * lz};
  long ix, iy, iz;
  double tsd = -1.0;
  if (range_cell(r, ix, iy, iz)) {
    long nc = s.gr.nc, c = cidx(s.gr, ix, iy, iz);
    double pp[NV];
    load_cell(s.p, nc, c, pp);
    Geom geo;
    geom_cell(s, ix, iy, iz, geo);
    double aaa[6];
    gas_wavespeeds_lr(pp, geo, a.gam, act, aaa);
    double tautot[3];
    double chi = calc_chi_slim(pp, geo, a.gam, a.op);
    long idx3[3] = {ix, iy, iz};
    for (int d = 0; d < 3; ++d) {
      double sg = kmath::sqrt(geo.gg[d + 1][d + 1]);
      double dxp = kmath::fmax(cell_size(g, idx3[d], d) * sg, cell_size(g, idx3[d] + 1, d) * sg);
      tautot[d] = chi * dxp;
    }
    if (a.damp_nc > 0 && (iy < a.damp_nc || iy >= s.gr.ny - a.damp_nc)) tautot[0] = tautot[1] = tautot[2] = 0.0;
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
    double ax = kmath::fmax(kmath::fabs(aaa[0]), kmath::fabs(aaa[1]));
    double ay = kmath::fmax(kmath::fabs(aaa[2]), kmath::fabs(aaa[3]));
    double az = kmath::fmax(kmath::fabs(aaa[4]), kmath::fabs(aaa[5]));
    s.amax[0 * nc + c] = ax;
    s.amax[1 * nc + c] = ay;
    s.amax[2 * nc + c] = az;
    for (int d = 0; d < 3; ++d)
      s.amax[(3 + d) * nc + c] = kmath::fmax(kmath::fabs(radl[2 * d]), kmath::fabs(radl[2 * d + 1]));
    double wsx = kmath::fmax(ax, kmath::fmax(kmath::fabs(rad0[0]), kmath::fabs(rad0[1])));
    double wsy = kmath::fmax(ay, kmath::fmax(kmath::fabs(rad0[2]), kmath::fabs(rad0[3])));
    double wsz = kmath::fmax(az, kmath::fmax(kmath::fabs(rad0[4]), kmath::fabs(rad0[5])));
    bool in_domain = ix >= 0 && ix < s.gr.nx && iy >= 0 && iy < s.gr.ny && iz >= 0 && iz < s.gr.nz;
    if (in_domain) {
      double dx = cell_size(g, ix, 0), dy = cell_size(g, iy, 1), dz = cell_size(g, iz, 2);
      if (s.gr.nz > 1 && s.gr.ny > 1) tsd = wsx / dx + wsy / dy + wsz / dz;
      else if (s.gr.nz == 1 && s.gr.ny > 1) tsd = wsx / dx + wsy / dy;
      else if (s.gr.ny == 1 && s.gr.nz > 1) tsd = wsx / dx + wsz / dz;
      else tsd = wsx / dx;
      tsd /= a.tsteplim;
      if (!(tsd == tsd)) tsd = -1.0;  // a NaN never wins the reference's max/min
    }
  }
  // block max/min of the positive CFL denominators, then one atomic per block
  double vmax = tsd > 0.0 ? tsd : 0.0;
  double vmin = tsd > 0.0 ? tsd : 1.0e300;
  for (int o = 16; o > 0; o >>= 1) {
    vmax = fmax(vmax, __shfl_down_sync(0xffffffff, vmax, o));
    vmin = fmin(vmin, __shfl_down_sync(0xffffffff, vmin, o));
  }
  __shared__ double smax[32], smin[32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    smax[warp] = vmax;
    smin[warp] = vmin;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0, n = 1.0e300;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      m = fmax(m, smax[w]);
      n = fmin(n, smin[w]);
    }
    if (m > 0.0) atomicMax(&sc->tsd_max_bits, dbits(m));
    if (n < 1.0e300) atomicMin(&sc->tsd_min_bits, dbits(n));
  }
}

// ---- face fluxes: reconstruct + floors + flux + LAXF (sim.zig:1209-1503) -----
struct FluxArgs {
  double gam, theta, maxvel;
  FloorParams fl;
  int radvisc;
  int fp32;  // the mixed instance's FP32 pieces (KC_FP32_PPM | KC_FP32_LAXF | KC_FP32_FLUX)
};
__device__ __forceinline__ void face_rijvisc(const DevState& s, long c, long cm, double rv[4][4]) {
  long nc = s.gr.nc;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) rv[i][j] = 0.5 * (s.rijvisc[(long)(i * 4 + j) * nc + c] + s.rijvisc[(long)(i * 4 + j) * nc + cm]);
}
// one face state: floors, one-sided flux, viscous addition, conserveds; the
// floors and the flux inlined (their out-of-line forms passed the state and the
// face metric through the call frame: 1.17 KB per thread, 27% slower)
__device__ int face_state(const DevState& s, DevScalars* sc, const FluxArgs& a, int dim, double pp[NV], const Geom& g,
                          long c, long cm, double ff[NV], double uu[NV]) {
  int gc = 0;
  check_floors_mhd_inl(pp, g, a.gam, a.fl, gc);
  if (gc) atomicAdd(&sc->n_guard, (unsigned long long)gc);
  int e = f_flux_prime_inl(pp, dim, g, a.gam, ff);
  if (e) return e;
  if (a.fp32 & KC_FP32_FLUX)
    for (int iv = 0; iv < NV; ++iv) ff[iv] = (double)(float)ff[iv];
  p2u(pp, uu, g, a.gam);
  if (a.radvisc) {
    double rv[4][4];
    face_rijvisc(s, c, cm, rv);
    add_visc_flux(ff, uu, rv, g, dim, s.gr.ny > 1, s.gr.nz > 1, a.maxvel);
  }
  return E_OK;
}
#ifndef KC_FLUX_MIN_BLOCKS
// resident blocks of 128 per SM the face kernel's register budget must allow:
// with the floors and the flux inlined, 4 (128 registers, 16 warps per SM)
// measured 10% faster than 3 (168) and 2 (206, no spills) 29% slower
#define KC_FLUX_MIN_BLOCKS 4
#endif
// MIXED: the instance of the mixed form, whose FP32 pieces (reconstruction,
// LAXF dissipation, rounded fluxes; kc_mixed.cuh) FluxArgs::fp32 selects
// DIM: the face direction, a template argument so that every index along it
// is a compile-time one (one instance per direction)
template <bool MIXED, int DIM>
__global__ void __launch_bounds__(128, KC_FLUX_MIN_BLOCKS) k_face_flux(DevState s, DevScalars* sc, const __grid_constant__ FluxArgs a) {
  constexpr int dim = DIM;
  long n = dim == 0 ? s.gr.nx : dim == 1 ? s.gr.ny : s.gr.nz;
  int c0d = dim == 0 ? 1 : 0, c1d = dim == 2 ? 1 : 2;
  long dims[3] = {s.gr.nx, s.gr.ny, s.gr.nz};
  long lo0 = dims[c0d] > 1 ? -1 : 0, n0 = dims[c0d] > 1 ? dims[c0d] + 2 : dims[c0d];
  long lo1 = dims[c1d] > 1 ? -1 : 0, n1 = dims[c1d] > 1 ? dims[c1d] + 2 : dims[c1d];
  // thread x walks the x index: for dim 0 that is the face index
  long nf0 = dim == 0 ? n + 1 : n0;
  long nfo = dim == 0 ? n0 : n + 1;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nf0 * nfo * n1) return;
  long a0 = t % nf0, q = t / nf0;
  long a1 = q % nfo, a2 = q / nfo;
  long f, cx0, cx1;
  if (dim == 0) {
    f = a0;
    cx0 = lo0 + a1;
  } else {
    cx0 = lo0 + a0;
    f = a1;
  }
  cx1 = lo1 + a2;
  long cf[3];
  cf[dim] = f;
  cf[c0d] = cx0;
  cf[c1d] = cx1;
  const Grid& g = s.gr.g;
  long nc = s.gr.nc;
  // stencil cells f-3 .. f+2 along dim
  long cst[6];
  for (int k = 0; k < 6; ++k) {
    long cc[3] = {cf[0], cf[1], cf[2]};
    cc[dim] = f - 3 + k;
    cst[k] = cidx(s.gr, cc[0], cc[1], cc[2]);
  }
  double dxs[6];
  for (int k = 0; k < 6; ++k) dxs[k] = cell_size(g, f - 3 + k, dim);
  double pL[NV], pR[NV];
  PpmCoef kl, kr;  // the width factors of the two stencils, shared by the 13 variables
  if (!MIXED || !(a.fp32 & KC_FP32_PPM)) {
    kl = ppm_coef(dxs);
    kr = ppm_coef(dxs + 1);
  }
  for (int iv = 0; iv < NV; ++iv) {
    double v[6];
    for (int k = 0; k < 6; ++k) v[k] = s.p[iv * nc + cst[k]];
    if (MIXED && (a.fp32 & KC_FP32_PPM)) {
      pL[iv] = recon_ppm_mixed(v, dxs).right;
      pR[iv] = recon_ppm_mixed(v + 1, dxs + 1).left;
    } else {
      pL[iv] = ppm_apply(v, kl).right;      // cell f-1: right face value
      pR[iv] = ppm_apply(v + 1, kr).left;   // cell f: left face value
    }
  }
  Geom geo;
  geom_face(s, cf[0], cf[1], cf[2], dim, geo);
  long c = cst[3], cm = cst[2];
  double ffl[NV], ffr[NV], uL[NV], uR[NV];
  int e = face_state(s, sc, a, dim, pL, geo, c, cm, ffl, uL);
  if (!e) e = face_state(s, sc, a, dim, pR, geo, c, cm, ffr, uR);
  if (e) {
    set_err(sc, e, c);
    return;
  }
  double ag = kmath::fmax(s.amax[(long)dim * nc + c], s.amax[(long)dim * nc + cm]);
  double agr = kmath::fmax(s.amax[(long)(3 + dim) * nc + c], s.amax[(long)(3 + dim) * nc + cm]);
  long fi = face_index(s.gr, dim, cf[0], cf[1], cf[2]);
  double* out = s.flb[dim];
  long nfd = s.nf[dim];
#pragma unroll
  for (int iv = 0; iv < NV; ++iv)
    out[iv * nfd + fi] = (MIXED && (a.fp32 & KC_FP32_LAXF)) ? laxf_f(ffl[iv], ffr[iv], uL[iv], uR[iv], iv >= EE ? agr : ag)
                                                         : laxf(ffl[iv], ffr[iv], uL[iv], uR[iv], iv >= EE ? agr : ag);
}

// ---- face fluxes through shared-memory tiles (sweeps along y and z) ---------------
// The same face fluxes as k_face_flux<false, DIM>, bit for bit, with the PPM
// stencils staged in shared memory. A block takes FT_COLS transverse columns
// (x fastest, then the other transverse index, linearised so that no lane
// idles at the end of an x row) and FT_FACES consecutive faces along the sweep.
// It loads the FT_FACES + 5 cells of each column that the faces' stencils
// cover, 13 variables, with coalesced loads; reconstructs each of the
// FT_FACES + 1 cells the faces need once (one PPM gives a cell's left and right
// face values, against two PPMs per face when each face reconstructs both of
// its neighbours); and then each thread forms one face's two states, one-sided
// fluxes and LAXF flux from the staged values.
constexpr int FT_COLS = 32, FT_FACES = 4, FT_ROWS = FT_FACES + 5, FT_REC = FT_FACES + 1, FT_LW = FT_COLS + 1;
// STAGE = false keeps the stencil reads in L1 and stages only the reconstructed
// face values (27 KB of shared memory per block instead of 59 KB, more L1 for
// the kernel's metric loads and call frames).
struct FaceTileOut {
  double fr[FT_FACES][NV][FT_LW];   // right value of cell f-1: the left state of face f
  double fl[FT_FACES][NV][FT_LW];   // left value of cell f: the right state of face f
  PpmCoef coef[FT_REC];             // width factors of cells f0-1 .. f0+FT_FACES-1
};
struct FaceTile {
  FaceTileOut o;
  double p[NV][FT_ROWS][FT_LW];     // stencil rows f0-3 .. f0+FT_FACES+1
};
template <int DIM, bool STAGE>
__global__ void __launch_bounds__(128, KC_FLUX_MIN_BLOCKS) k_face_flux_tiled(DevState s, DevScalars* sc,
                                                                               const __grid_constant__ FluxArgs a) {
  static_assert(DIM == 1 || DIM == 2, "tiles are along y or z");
  extern __shared__ __align__(16) unsigned char ft_smem[];
  FaceTile& T = *reinterpret_cast<FaceTile*>(ft_smem);  // only T.o exists when !STAGE
  constexpr int dim = DIM, c0d = 0, c1d = DIM == 1 ? 2 : 1;
  const long n = dim == 1 ? s.gr.ny : s.gr.nz;
  const long dims[3] = {s.gr.nx, s.gr.ny, s.gr.nz};
  const long lo0 = dims[c0d] > 1 ? -1 : 0, n0 = dims[c0d] > 1 ? dims[c0d] + 2 : dims[c0d];
  const long lo1 = dims[c1d] > 1 ? -1 : 0, n1 = dims[c1d] > 1 ? dims[c1d] + 2 : dims[c1d];
  const long ncols = n0 * n1, col0 = (long)blockIdx.x * FT_COLS, f0 = (long)blockIdx.y * FT_FACES;
  const long ng = dim == 1 ? s.gr.ngy : s.gr.ngz;
  const int tid = threadIdx.x;
  const Grid& g = s.gr.g;
  const long nc = s.gr.nc;
  // global index of the stencil cell of column col at sweep index sw (-1: outside the stored grid)
  auto stencil_cell = [&](long col, long sw) -> long {
    if (col >= ncols || sw < -ng || sw >= n + ng) return -1;
    long cc[3];
    cc[c0d] = lo0 + col % n0;
    cc[c1d] = lo1 + col / n0;
    cc[dim] = sw;
    return cidx(s.gr, cc[0], cc[1], cc[2]);
  };
  // 1. stage the stencil rows of the block's columns (rows outside the stored grid stay unread)
  for (int k = tid; STAGE && k < NV * FT_ROWS * FT_COLS; k += blockDim.x) {
    const int l = k % FT_COLS, q = k / FT_COLS, r = q % FT_ROWS, iv = q / FT_ROWS;
    const long cj = stencil_cell(col0 + l, f0 - 3 + r);
    T.p[iv][r][l] = cj >= 0 ? s.p[(long)iv * nc + cj] : 0.0;
  }
  if (tid < FT_REC) {
    double dxs[5];
    for (int k = 0; k < 5; ++k) dxs[k] = cell_size(g, f0 - 3 + tid + k, dim);
    T.o.coef[tid] = ppm_coef(dxs);
  }
  __syncthreads();
  // 2. one PPM per (cell, variable, column)
  for (int k = tid; k < NV * FT_REC * FT_COLS; k += blockDim.x) {
    const int l = k % FT_COLS, q = k / FT_COLS, rc = q % FT_REC, iv = q / FT_REC;
    double u[5];
    if (STAGE) {
      for (int j = 0; j < 5; ++j) u[j] = T.p[iv][rc + j][l];
    } else {
      for (int j = 0; j < 5; ++j) {
        const long cj = stencil_cell(col0 + l, f0 - 3 + rc + j);
        u[j] = cj >= 0 ? s.p[(long)iv * nc + cj] : 0.0;
      }
    }
    const Faces fc = ppm_apply(u, T.o.coef[rc]);
    if (rc < FT_FACES) T.o.fr[rc][iv][l] = fc.right;
    if (rc > 0) T.o.fl[rc - 1][iv][l] = fc.left;
  }
  __syncthreads();
  // 3. one face per thread
  const int w = tid >> 5, lane = tid & 31;
  const long f = f0 + w, col = col0 + lane;
  if (f > n || col >= ncols) return;
  long cf[3];
  cf[dim] = f;
  cf[c0d] = lo0 + col % n0;
  cf[c1d] = lo1 + col / n0;
  double pL[NV], pR[NV];
  for (int iv = 0; iv < NV; ++iv) {
    pL[iv] = T.o.fr[w][iv][lane];
    pR[iv] = T.o.fl[w][iv][lane];
  }
  long cc[3] = {cf[0], cf[1], cf[2]};
  cc[dim] = f;
  const long c = cidx(s.gr, cc[0], cc[1], cc[2]);
  cc[dim] = f - 1;
  const long cm = cidx(s.gr, cc[0], cc[1], cc[2]);
  Geom geo;
  geom_face(s, cf[0], cf[1], cf[2], dim, geo);
  double ffl[NV], ffr[NV], uL[NV], uR[NV];
  int e = face_state(s, sc, a, dim, pL, geo, c, cm, ffl, uL);
  if (!e) e = face_state(s, sc, a, dim, pR, geo, c, cm, ffr, uR);
  if (e) {
    set_err(sc, e, c);
    return;
  }
  const double ag = kmath::fmax(s.amax[(long)dim * nc + c], s.amax[(long)dim * nc + cm]);
  const double agr = kmath::fmax(s.amax[(long)(3 + dim) * nc + c], s.amax[(long)(3 + dim) * nc + cm]);
  const long fi = face_index(s.gr, dim, cf[0], cf[1], cf[2]);
  double* out = s.flb[dim];
  const long nfd = s.nf[dim];
#pragma unroll
  for (int iv = 0; iv < NV; ++iv) out[iv * nfd + fi] = laxf(ffl[iv], ffr[iv], uL[iv], uR[iv], iv >= EE ? agr : ag);
}

// ---- flux-CT (koral/sim/ct.zig:38) --------------------------------------------
__device__ __forceinline__ long pin(long n, long i) { return n == 1 ? 0 : i; }
__device__ __forceinline__ double flbv(const DevState& s, int dim, int iv, long ix, long iy, long iz) {
  return s.flb[dim][(long)iv * s.nf[dim] + face_index(s.gr, dim, ix, iy, iz)];
}
// R: the arithmetic type of the corner averages (float in the mixed form)
template <class R>
__global__ void k_ct_emf(DevState s) {
  long nx = s.gr.nx, ny = s.gr.ny, nz = s.gr.nz;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (nx + 1) * (ny + 1) * (nz + 1)) return;
  long ix = t % (nx + 1), q = t / (nx + 1), iy = q % (ny + 1), iz = q / (ny + 1);
  R coef1 = (ny > 1 && nz > 1) ? R(0.25) : R(0.5);
  R coef2 = (nx > 1 && nz > 1) ? R(0.25) : R(0.5);
  R coef3 = (nx > 1 && ny > 1) ? R(0.25) : R(0.5);
  auto F = [&](int dim, int iv, long jx, long jy, long jz) { return (R)flbv(s, dim, iv, jx, jy, jz); };
  if (ny > 1 || nz > 1) {
    R sm = R(0);
    if (ny > 1) sm += F(1, B3, pin(nx, ix), pin(ny, iy), pin(nz, iz)) + F(1, B3, pin(nx, ix), pin(ny, iy), pin(nz, iz - 1));
    if (nz > 1) sm -= F(2, B2, pin(nx, ix), pin(ny, iy), pin(nz, iz)) + F(2, B2, pin(nx, ix), pin(ny, iy - 1), pin(nz, iz));
    s.emf[0][t] = (double)(coef1 * sm);
  } else {
    s.emf[0][t] = 0.0;
  }
  if (nx > 1 || nz > 1) {
    R sm = R(0);
    if (nz > 1) sm += F(2, B1, pin(nx, ix), pin(ny, iy), pin(nz, iz)) + F(2, B1, pin(nx, ix - 1), pin(ny, iy), pin(nz, iz));
    if (nx > 1) sm -= F(0, B3, ix, pin(ny, iy), pin(nz, iz)) + F(0, B3, ix, pin(ny, iy), pin(nz, iz - 1));
    s.emf[1][t] = (double)(coef2 * sm);
  } else {
    s.emf[1][t] = 0.0;
  }
  if (nx > 1 || ny > 1) {
    R sm = R(0);
    if (nx > 1) sm += F(0, B2, ix, pin(ny, iy), pin(nz, iz)) + F(0, B2, ix, pin(ny, iy - 1), pin(nz, iz));
    if (ny > 1) sm -= F(1, B1, pin(nx, ix), pin(ny, iy), pin(nz, iz)) + F(1, B1, pin(nx, ix - 1), pin(ny, iy), pin(nz, iz));
    s.emf[2][t] = (double)(coef3 * sm);
  } else {
    s.emf[2][t] = 0.0;
  }
}
template <class R>
__global__ void k_ct_rebuild(DevState s) {
  long nx = s.gr.nx, ny = s.gr.ny, nz = s.gr.nz;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (nx + 1) * (ny + 1) * (nz + 1)) return;
  long ix = t % (nx + 1), q = t / (nx + 1), iy = q % (ny + 1), iz = q / (ny + 1);
  auto E = [&](int comp, long jx, long jy, long jz) { return (R)s.emf[comp - 1][(jz * (ny + 1) + jy) * (nx + 1) + jx]; };
  if (nx > 1 && iy < ny && iz < nz) {
    long fi = face_index(s.gr, 0, ix, iy, iz), nf = s.nf[0];
    s.flb[0][B1 * nf + fi] = 0.0;
    s.flb[0][B2 * nf + fi] = (double)(R(0.5) * (E(3, ix, iy, iz) + E(3, ix, iy + 1, iz)));
    s.flb[0][B3 * nf + fi] = (double)(R(-0.5) * (E(2, ix, iy, iz) + E(2, ix, iy, iz + 1)));
  }
  if (ny > 1 && ix < nx && iz < nz) {
    long fi = face_index(s.gr, 1, ix, iy, iz), nf = s.nf[1];
    s.flb[1][B1 * nf + fi] = (double)(R(-0.5) * (E(3, ix, iy, iz) + E(3, ix + 1, iy, iz)));
    s.flb[1][B2 * nf + fi] = 0.0;
    s.flb[1][B3 * nf + fi] = (double)(R(0.5) * (E(1, ix, iy, iz) + E(1, ix, iy, iz + 1)));
  }
  if (nz > 1 && ix < nx && iy < ny) {
    long fi = face_index(s.gr, 2, ix, iy, iz), nf = s.nf[2];
    s.flb[2][B1 * nf + fi] = (double)(R(0.5) * (E(2, ix, iy, iz) + E(2, ix + 1, iy, iz)));
    s.flb[2][B2 * nf + fi] = (double)(R(-0.5) * (E(1, ix, iy, iz) + E(1, ix, iy + 1, iz)));
    s.flb[2][B3 * nf + fi] = 0.0;
  }
}

// ---- conserved update + metric source (sim.zig:1140,1542) --------------------
// 4 resident blocks (128 registers, small spills): measured 4% faster than 168
__global__ void __launch_bounds__(128, 4) k_update(DevState s, double gam, int dt_slot) {
  Range r = {0, 0, 0, s.gr.nx, s.gr.ny, s.gr.nz};
  long ix, iy, iz;
  if (!range_cell(r, ix, iy, iz)) return;
  long nc = s.gr.nc, c = cidx(s.gr, ix, iy, iz);
  const Grid& g = s.gr.g;
  double pp[NV];
  load_cell(s.p, nc, c, pp);
  Geom geo;
  geom_cell(s, ix, iy, iz, geo);
  double gdetu = geo.gdet;
  double ss[NV];
  for (int i = 0; i < NV; ++i) ss[i] = 0.0;
  double tij[4][4], tl[4][4], rup[4][4], rl[4][4];
  calc_tij(pp, geo, gam, tij);
  lower_second(tij, geo, tl);
  calc_rij(pp, geo, rup);
  lower_second(rup, geo, rl);
  const int rows[4] = {UU, VX, VY, VZ}, rrows[4] = {EE, FX, FY, FZ};
  for (int a = 0; a < 4; ++a)
    for (int l = 0; l < 4; ++l)
      for (int nu = 0; nu < 4; ++nu) {
        double k = s.kr[(long)(l * 10 + sym10(nu, a)) * nc + c];
        ss[rows[nu]] += gdetu * tl[a][l] * k;
        ss[rrows[nu]] += gdetu * rl[a][l] * k;
      }
  double dx = cell_size(g, ix, 0), dy = cell_size(g, iy, 1), dz = cell_size(g, iz, 2);
  double dt = s.coef[dt_slot];
  long fx0 = face_index(s.gr, 0, ix, iy, iz), fx1 = face_index(s.gr, 0, ix + 1, iy, iz);
  long fy0 = face_index(s.gr, 1, ix, iy, iz), fy1 = face_index(s.gr, 1, ix, iy + 1, iz);
  long fz0 = face_index(s.gr, 2, ix, iy, iz), fz1 = face_index(s.gr, 2, ix, iy, iz + 1);
  for (int iv = 0; iv < NV; ++iv) {
    double flxl = s.flb[0][iv * s.nf[0] + fx0], flxr = s.flb[0][iv * s.nf[0] + fx1];
    double flyl = s.flb[1][iv * s.nf[1] + fy0], flyr = s.flb[1][iv * s.nf[1] + fy1];
    double flzl = s.flb[2][iv * s.nf[2] + fz0], flzr = s.flb[2][iv * s.nf[2] + fz1];
    double du = -(flxr - flxl) * dt / dx - (flyr - flyl) * dt / dy - (flzr - flzl) * dt / dz;
    double uo = s.u[iv * nc + c];
    s.u[iv * nc + c] = uo + du + ss[iv] * dt;
  }
}

// ---- implicit operator (sim.zig:1715) ----------------------------------------
struct ImplArgs {
  double gam;
  int dt_slot;  // the pass's dt in DevState::coef
  int phi_fastest;  // thread -> cell order of the per-cell kernel: 1 = phi fastest, 0 = x fastest
  int y_fastest;    // without phi_fastest: theta (y) fastest instead of x (2D grids)
  RadParams rp;
  OpacParams op;
  ImplicitParams ip;
  int polar_nc;
};
// the learned-guess form and the training-pair harvest of the implicit pass
struct ImplExtra {
  const double* guess;  // [NV][nx ny nz] seeded starting states, or null (plain form)
  float* hx;            // harvest: features [cap][16], targets [cap][4], or null
  float* ht;
  unsigned long long* hcount;
  long hcap;
  unsigned long long* n_fallback;  // seeded ladders that failed and fell back to the plain path
  int hfilter;                     // harvest only cells whose pre-solve state must iterate
};
// Whether the no-bisection start (the cell's pre-solve state) would have to
// iterate: its first-rung residual against the Newton core's first exit
// (conv), as solve_implicit_lab_from evaluates it. Out of line, so that its
// locals do not enlarge the solve's call frame.
__device__ __noinline__ bool presolve_needs_newton(const double pp00[NV], const Geom& g, double dt, const ImplArgs& a) {
  double uu00[NV], pc[NV];
  p2u(pp00, uu00, g, a.gam);
  RadState st00;
  fill_rad_state(pp00, g, a.gam, a.op, true, st00);
  const double ehat = -calc_ff_rtt(pp00, g, nullptr);
  const int sw = (ehat < a.ip.threshold * pp00[UU]) ? PRIM_RAD : PRIM_MHD;
  const double e0 = implicit_start_residual(uu00, st00, pp00, g, dt, a.gam, a.rp, a.op, 1.0, a.ip, sw, pc);
  return !(e0 < a.ip.conv);
}
// FORM: IMPL_PLAIN is the reference path alone (the guess and harvest code is
// not compiled into it, so its registers and code size are those of the plain
// solve); IMPL_GUESS adds the learned start only; IMPL_FULL the learned start
// and the training-pair harvest.
// NT: threads per block, and one block per SM: the register budget follows
// (256 threads: 255 registers, 8 warps; 384: 168, 12 warps; 512: 128, 16 warps;
// an SM sub-partition holds 16 K registers, so no budget between these gives
// more warps). Every form runs in two block-synchronous phases: every thread's
// warm start (the 1-D bisection, or the learned start's pick), a block barrier,
// then every thread's ladder, so that all warps of the SM execute the same part
// of the solver's code at a time (the code is far larger than the instruction
// cache). Measured on the 192x180x64 wedge, implicit pass per step: one
// unsynchronised pass in blocks of 128 58.1 ms (255 registers, 2 blocks per SM);
// the two phases in blocks of 128 56.4; SM-wide blocks of 256 50.2, of 384 46.0,
// of 512 48.2; a third phase (the rung-0 first residual test) 52.9 at 256.
enum : int { IMPL_PLAIN = 0, IMPL_GUESS = 1, IMPL_FULL = 2 };
#ifndef KC_IMPLICIT_TPB
#define KC_IMPLICIT_TPB 384  // the default block: 12 warps, 168 registers
#endif
template <int FORM, int NT>
__global__ void __launch_bounds__(NT, 1) k_implicit(DevState s, DevScalars* sc, const __grid_constant__ ImplArgs a,
                                                        ImplExtra x) {
  const double dt = s.coef[a.dt_slot];
  long ix = 0, iy = 0, iz = 0;
  bool act;
  if (a.phi_fastest) {
    act = domain_cell_phi_fastest(s.gr, ix, iy, iz);
  } else if (a.y_fastest) {
    // 2D: neighbours in theta at one radius (measured 10% faster than x fastest
    // on the 384x360 grid; 8 x 4 tiles per warp were in between)
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    act = t < (long)s.gr.nx * s.gr.ny * s.gr.nz;
    if (act) {
      iy = t % s.gr.ny;
      long q = t / s.gr.ny;
      ix = q % s.gr.nx;
      iz = q / s.gr.nx;
    }
  } else {
    Range r = {0, 0, 0, s.gr.nx, s.gr.ny, s.gr.nz};
    act = range_cell(r, ix, iy, iz);
  }
  if (act && a.polar_nc > 0 && (iy < a.polar_nc || iy > s.gr.ny - a.polar_nc - 1)) act = false;
  long nc = s.gr.nc, c = act ? cidx(s.gr, ix, iy, iz) : 0;
  constexpr bool HARVEST = FORM == IMPL_FULL;
  const bool guessed = FORM != IMPL_PLAIN && x.guess != nullptr;
  // the cell's metric is read once and its state written once: evict-first in
  // L2 (which keeps L2 for the solver's call frames); the state loads stay plain
  // (their evict-first form costs the kernel registers and 200 bytes of spills)
  double uu[NV], pp[NV], pp00[NV];
  Geom g;
  ImplicitPre pre;
  int done = 0;  // the learned form's pre-solve state took the core's first exit
  if (act) {
    load_cell(s.u, nc, c, uu);
    load_cell(s.p, nc, c, pp);
    geom_cell<true>(s, ix, iy, iz, g);
    if (HARVEST)
      for (int i = 0; i < NV; ++i) pp00[i] = pp[i];
    if (guessed) {
      long nd = (long)s.gr.nx * s.gr.ny * s.gr.nz, td = ix + s.gr.nx * (iy + s.gr.ny * iz);
      double g0[NV];
      for (int i = 0; i < NV; ++i) g0[i] = x.guess[i * nd + td];
      done = implicit_prepare_from(uu, pp, g, dt, a.gam, a.rp, a.op, a.ip, g0, pre);
    } else {
      implicit_prepare(pp, g, dt, a.gam, a.op, a.ip, pre);
    }
  }
  __syncthreads();
  if (!act) return;
  ImplicitResult res;
  if (done) {
    res = implicit_first_exit_result(pre.startwith);
  } else {
    res = implicit_ladder(uu, pp, g, dt, a.gam, a.rp, a.op, a.ip, pre);
    if (guessed && !res.ok) {  // the seeded ladder failed: the plain solve
      atomicAdd(x.n_fallback, 1ULL);
      res = solve_implicit_lab(uu, pp, g, dt, a.gam, a.rp, a.op, a.ip);
    }
  }
  if (HARVEST && x.hx && res.ok && res.rung == 0 && (!x.hfilter || presolve_needs_newton(pp00, g, dt, a))) {
    unsigned long long k = atomicAdd(x.hcount, 1ULL);
    if ((long)k < x.hcap) {
      double ehat = -calc_ff_rtt(pp00, g, nullptr);
      int sw = (ehat < a.ip.threshold * pp00[UU]) ? PRIM_RAD : PRIM_MHD;
      mlp_features_raw(pp00, dt, g.gdet, g.alpha, sw, x.hx + k * MLP_IN);
      mlp_targets_raw(pp00, pp, sw, x.ht + k * MLP_OUT);
    }
  }
  if (res.ok) {
    store_cell<true>(s.u, nc, c, uu);
    store_cell<true>(s.p, nc, c, pp);
    s.flags[5 * nc + c] = 0;
    atomicAdd(&sc->n_iters, (unsigned long long)res.iters);
    atomicAdd(&sc->n_solves, 1ULL);
  } else {
    s.flags[5 * nc + c] = -1;
    atomicAdd(&sc->n_fail, 1ULL);
  }
}

// The split form of the implicit pass, bit-identical to k_implicit. Most cells
// of a torus step pass the Newton core's first residual test at their warm
// start, while the rest need one or more Newton iterations; in one kernel every
// warp holding a cell of the second kind runs at that cell's pace. The opening
// kernel runs the warm start and the rung-0 first residual for every cell,
// finishes the cells that pass, and appends the others (domain index and warm
// start) to a compact list; the ladder kernel runs the full ladder over the
// list only, so its warps hold only cells that iterate.
struct SplitList {
  unsigned long long* count;  // cells appended by the opening kernel
  int* cell;                  // domain index ix + nx (iy + ny iz)
  double* pp0;                // [NV][capacity] warm starts
  long cap;
};
__global__ void __launch_bounds__(128) k_implicit_open(DevState s, DevScalars* sc, const __grid_constant__ ImplArgs a,
                                                        SplitList L) {
  const double dt = s.coef[a.dt_slot];
  Range r = {0, 0, 0, s.gr.nx, s.gr.ny, s.gr.nz};
  long ix, iy, iz;
  if (!range_cell(r, ix, iy, iz)) return;
  if (a.polar_nc > 0 && (iy < a.polar_nc || iy > s.gr.ny - a.polar_nc - 1)) return;
  long nc = s.gr.nc, c = cidx(s.gr, ix, iy, iz);
  double uu[NV], pp[NV];
  load_cell(s.u, nc, c, uu);
  load_cell(s.p, nc, c, pp);
  Geom g;
  geom_cell(s, ix, iy, iz, g);
  ImplicitPre pre;
  implicit_prepare(pp, g, dt, a.gam, a.op, a.ip, pre);
  if (implicit_first_exit(uu, pp, g, dt, a.gam, a.rp, a.op, a.ip, pre)) {
    store_cell(s.u, nc, c, uu);
    store_cell(s.p, nc, c, pp);
    s.flags[5 * nc + c] = 0;
    atomicAdd(&sc->n_iters, 1ULL);
    atomicAdd(&sc->n_solves, 1ULL);
    return;
  }
  unsigned long long k = atomicAdd(L.count, 1ULL);
  if ((long)k >= L.cap) {  // cannot happen: the list holds every domain cell
    set_err(sc, KC_ERR_CUDA, c);
    return;
  }
  L.cell[k] = (int)(ix + s.gr.nx * (iy + s.gr.ny * iz));
  for (int i = 0; i < NV; ++i) L.pp0[(long)i * L.cap + (long)k] = pre.pp0[i];
}
__global__ void __launch_bounds__(128) k_implicit_ladder(DevState s, DevScalars* sc, const __grid_constant__ ImplArgs a,
                                                          SplitList L) {
  const double dt = s.coef[a.dt_slot];
  long n = (long)*L.count;
  if (n > L.cap) n = L.cap;
  for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
    long td = L.cell[k];
    long ix = td % s.gr.nx, iy = (td / s.gr.nx) % s.gr.ny, iz = td / ((long)s.gr.nx * s.gr.ny);
    long nc = s.gr.nc, c = cidx(s.gr, ix, iy, iz);
    double uu[NV], pp[NV];
    load_cell(s.u, nc, c, uu);
    load_cell(s.p, nc, c, pp);
    Geom g;
    geom_cell(s, ix, iy, iz, g);
    // implicit_prepare's state for this cell, with the warm start it computed
    ImplicitPre pre;
    p2u(pp, pre.uu00, g, a.gam);
    double ehat = -calc_ff_rtt(pp, g, nullptr);
    fill_rad_state(pp, g, a.gam, a.op, true, pre.state00);
    for (int i = 0; i < NV; ++i) pre.pp0[i] = L.pp0[(long)i * L.cap + k];
    pre.startwith = (ehat < a.ip.threshold * pp[UU]) ? PRIM_RAD : PRIM_MHD;
    ImplicitResult res = implicit_ladder(uu, pp, g, dt, a.gam, a.rp, a.op, a.ip, pre);
    if (res.ok) {
      store_cell(s.u, nc, c, uu);
      store_cell(s.p, nc, c, pp);
      s.flags[5 * nc + c] = 0;
      atomicAdd(&sc->n_iters, (unsigned long long)res.iters);
      atomicAdd(&sc->n_solves, 1ULL);
    } else {
      s.flags[5 * nc + c] = -1;
      atomicAdd(&sc->n_fail, 1ULL);
    }
  }
}

// The learned guess per domain cell: features of the pre-solve state,
// standardised, through the tensor-core network (one warp per 32 cells), and
// the seeded starting state written to guess [NV][nx ny nz].
__global__ void __launch_bounds__(128) k_mlp_guess(DevState s, MlpDev m, ImplArgs a, double* guess) {
  const double dt = s.coef[a.dt_slot];
  __shared__ float xs[4][32 * MLP_IN];
  __shared__ float ys[4][32 * MLP_OUT];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  long nx = s.gr.nx, ny = s.gr.ny, nd = nx * ny * s.gr.nz;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  bool valid = t < nd;
  double pp[NV];
  int sw = PRIM_MHD;
  float f[MLP_IN];
  for (int k = 0; k < MLP_IN; ++k) f[k] = 0.0f;
  if (valid) {
    long ix = t % nx, iy = (t / nx) % ny, iz = t / (nx * ny);
    long c = cidx(s.gr, ix, iy, iz);
    load_cell(s.p, s.gr.nc, c, pp);
    Geom g;
    geom_cell(s, ix, iy, iz, g);
    double ehat = -calc_ff_rtt(pp, g, nullptr);
    sw = (ehat < a.ip.threshold * pp[UU]) ? PRIM_RAD : PRIM_MHD;
    mlp_features_raw(pp, dt, g.gdet, g.alpha, sw, f);
    for (int k = 0; k < MLP_IN; ++k) f[k] = mlp_clip((f[k] - m.blob[MLP_OFF_IMEAN + k]) / m.blob[MLP_OFF_ISTD + k]);
  }
  for (int k = 0; k < MLP_IN; ++k) xs[warp][lane * MLP_IN + k] = f[k];
  __syncwarp();
  mlp_forward_warp(m, xs[warp], ys[warp]);
  if (!valid) return;
  float y[MLP_OUT];
  for (int o = 0; o < MLP_OUT; ++o)
    y[o] = mlp_clip(ys[warp][lane * MLP_OUT + o]) * m.blob[MLP_OFF_OSTD + o] + m.blob[MLP_OFF_OMEAN + o];
  double g0[NV];
  mlp_apply(pp, y, sw, g0);
  for (int i = 0; i < NV; ++i) guess[i * nd + t] = g0[i];
}
// standardised features through the tensor-core network, for kc_mlp_forward
__global__ void __launch_bounds__(128) k_mlp_forward(MlpDev m, long n, const float* X, float* Y) {
  __shared__ float xs[4][32 * MLP_IN];
  __shared__ float ys[4][32 * MLP_OUT];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  for (int k = 0; k < MLP_IN; ++k) xs[warp][lane * MLP_IN + k] = t < n ? X[t * MLP_IN + k] : 0.0f;
  __syncwarp();
  mlp_forward_warp(m, xs[warp], ys[warp]);
  if (t < n)
    for (int o = 0; o < MLP_OUT; ++o) Y[t * MLP_OUT + o] = ys[warp][lane * MLP_OUT + o];
}

// the same operator as a persistent, lane-refilling state machine (bit-identical)
__global__ void __launch_bounds__(128) k_implicit_persistent(DevState s, DevScalars* sc, const __grid_constant__ ImplArgs a,
                                                              long nwork) {
  const double dt = s.coef[a.dt_slot];
  long nyb = s.gr.ny - 2L * a.polar_nc;
  ImpStepSrc src{s, sc, dt, s.gr.nx, nyb, (long)a.polar_nc};
  ImpParams P{a.gam, a.rp, a.op, a.ip};
  imp_persistent(src, nwork, &sc->work_next, P);
}

// ---- radiative viscosity (koral/sim/rijvisc.zig:266) ---------------------------
struct ViscArgs {
  double gam, rhor, alpha;
  int dt_slot;
  OpacParams op;
};
__global__ void __launch_bounds__(128, KC_RIJVISC_MIN_BLOCKS) k_rijvisc(DevState s, const __grid_constant__ ViscArgs a) {
  const double dt = s.coef[a.dt_slot];
  long xl = s.gr.nx > 1, yl = s.gr.ny > 1, zl = s.gr.nz > 1;
  Range r = {-xl, -yl, -zl, s.gr.nx + 2 * xl, s.gr.ny + 2 * yl, s.gr.nz + 2 * zl};
  long ix, iy, iz;
  if (!range_cell(r, ix, iy, iz)) return;
  long nx = s.gr.nx, ny = s.gr.ny, nz = s.gr.nz;
  int nout = (ix < 0 || ix >= nx) + (iy < 0 || iy >= ny) + (iz < 0 || iz >= nz);
  if (nout >= 2) return;
  long nc = s.gr.nc, c = cidx(s.gr, ix, iy, iz);
  const Grid& g = s.gr.g;
  double pp[NV];
  load_cell(s.p, nc, c, pp);
  Geom geo;
  geom_cell(s, ix, iy, iz, geo);
  // C calc_shear_lab (rijvisc.zig:39), RAD branch
  double du[4][4], du2[4][4];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      du[i][j] = 0.0;
      du2[i][j] = 0.0;
    }
  double ucon[4], ucov[4];
  ucon_ucov_from_prims(pp[FX], pp[FY], pp[FZ], geo, ucon, ucov);
  long nd[3] = {nx, ny, nz};
  // unrolled: du, du2 indexed by constants stay in registers (no stack frame)
#pragma unroll
  for (int idim = 1; idim < 4; ++idim) {
    int dim = idim - 1;
    if (nd[dim] <= 1) continue;
    long cm[3] = {ix, iy, iz}, cp[3] = {ix, iy, iz};
    cm[dim] -= 1;
    cp[dim] += 1;
    long ccm = cidx(s.gr, cm[0], cm[1], cm[2]), ccp = cidx(s.gr, cp[0], cp[1], cp[2]);
    Geom gm, gp;
    geom_cell(s, cm[0], cm[1], cm[2], gm);
    geom_cell(s, cp[0], cp[1], cp[2], gp);
    double umc[4], umv[4], upc[4], upv[4];
    ucon_ucov_from_prims(s.p[FX * nc + ccm], s.p[FY * nc + ccm], s.p[FZ * nc + ccm], gm, umc, umv);
    ucon_ucov_from_prims(s.p[FX * nc + ccp], s.p[FY * nc + ccp], s.p[FZ * nc + ccp], gp, upc, upv);
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
  double k[64];
  kr_block(s, c, k);
  double sl[4][4], shear[4][4];
  shear_from_gradients(du, du2, ucon, ucov, geo, k, sl);
  raise_both(sl, geo, shear);
  double chi = calc_chi_slim(pp, geo, a.gam, a.op);
  double dx[3] = {cell_size(g, ix, 0) * kmath::sqrt(geo.gg[1][1]), cell_size(g, iy, 1) * kmath::sqrt(geo.gg[2][2]),
                  cell_size(g, iz, 2) * kmath::sqrt(geo.gg[3][3])};
  double mindx;
  if (ny == 1 && nz == 1) mindx = dx[0];
  else if (nz == 1) mindx = kmath::fmin(dx[0], dx[1]);
  else if (ny == 1) mindx = kmath::fmin(dx[0], dx[2]);
  else mindx = kmath::fmin(dx[0], kmath::fmin(dx[1], dx[2]));
  double nu = visc_coeff(chi, mindx, s.blg[26L * nc + c], a.rhor, a.alpha, dt);
  double rv[4][4];
  rij_visc(nu, pp[EE], shear, geo, rv);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) s.rijvisc[(long)(i * 4 + j) * nc + c] = rv[i][j];
}

// ---- mimic dynamo (koral/sim/dynamo.zig) --------------------------------------
// Per-radius scale height (dynamo.zig:158 calcScaleHeight). The fold over
// (iy, iz) of each x column keeps the reference's serial order (iy outer, iz
// inner). One block per column: its threads form SH_THREADS consecutive terms
// (rho gdet and rho gdet dtheta^2) at a time into shared memory, and thread 0
// folds them in order, so the sums are the serial ones; the terms of the next
// chunk are loaded while thread 0 folds the current one (two buffers), and the
// columns run in parallel across the SMs.
constexpr int SH_THREADS = 512;
__global__ void __launch_bounds__(SH_THREADS) k_scale_height(DevState s) {
  __shared__ double ta[2][SH_THREADS], tb[2][SH_THREADS];
  const long ix = blockIdx.x;
  const int t = threadIdx.x;
  const long nz = s.gr.nz, nsteps = (long)s.gr.ny * nz, nc = s.gr.nc;
  const long nch = (nsteps + SH_THREADS - 1) / SH_THREADS;
  auto term = [&](long k, double& a, double& b) {
    a = 0.0;
    b = 0.0;
    if (k < nsteps) {
      long c = cidx(s.gr, ix, k / nz, k % nz);
      double rho = s.p[RHO * nc + c], gd = s.cgc[10L * nc + c];
      double dth = KP_PI / 2.0 - s.blg[27L * nc + c];
      a = rho * gd;
      b = rho * gd * dth * dth;
    }
  };
  double a, b;
  term(t, a, b);
  ta[0][t] = a;
  tb[0][t] = b;
  __syncthreads();
  double sigma = 0.0, sth = 0.0;  // thread 0's
  for (long ch = 0; ch < nch; ++ch) {
    const int buf = (int)(ch & 1);
    const bool next = ch + 1 < nch;
    if (next) term((ch + 1) * SH_THREADS + t, a, b);  // in flight during the fold
    if (t == 0) {
      const long m = nsteps - ch * SH_THREADS < SH_THREADS ? nsteps - ch * SH_THREADS : SH_THREADS;
#pragma unroll 8
      for (int j = 0; j < m; ++j) {
        sigma += ta[buf][j];
        sth += tb[buf][j];
      }
    }
    if (next) {
      ta[buf ^ 1][t] = a;
      tb[buf ^ 1][t] = b;
    }
    __syncthreads();
  }
  if (t == 0) s.scaleth[ix] = (ix > 0) ? kmath::sqrt(sth / sigma) : sth;
}
struct DynArgs {
  double gam, a, rhor, risco;
  int dt_slot;
  DynamoParams dp;
};
__global__ void __launch_bounds__(128, KC_DYNAMO_MIN_BLOCKS) k_dynamo_delta_a(DevState s, DevScalars* sc, DynArgs a) {
  const double dt = s.coef[a.dt_slot];
  long xl = s.gr.nx > 1, yl = s.gr.ny > 1, zl = s.gr.nz > 1;
  Range r = {-xl, -yl, -zl, s.gr.nx + 2 * xl, s.gr.ny + 2 * yl, s.gr.nz + 2 * zl};
  long ix, iy, iz;
  if (!range_cell(r, ix, iy, iz)) return;
  long nc = s.gr.nc, c = cidx(s.gr, ix, iy, iz);
  s.dyn_a[c] = 0.0;
  Geom geo, gbl;
  geom_cell(s, ix, iy, iz, geo);
  geom_bl(s, c, gbl);
  double jac[4][4];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) jac[i][j] = s.jbl[(long)(i * 4 + j) * nc + c];
  double pp[NV];
  load_cell(s.p, nc, c, pp);
  double angle, bsq;
  int e = field_angle(geo, gbl, jac, pp, angle, bsq);
  if (e) {
    set_err(sc, e, c);
    return;
  }
  double rr = gbl.xx[1], th = gbl.xx[2];
  if (rr < 1.0001 * a.rhor) return;
  double prermhd = (a.gam - 1.0) * pp[UU];
  double ehat = -calc_ff_rtt(pp, geo, nullptr);
  prermhd += ehat / 3.0;
  long gix = ix < 0 ? 0 : (ix > s.gr.nx - 1 ? s.gr.nx - 1 : ix);
  DynamoOut o = dynamo_delta_a(a.dp, a.a, dt, a.rhor, a.risco, rr, th, pp[B3], bsq, angle, prermhd, geo.gg[3][3],
                               s.scaleth[gix]);
  s.dyn_a[c] = o.aphi;
  if (a.dp.dampbeta) s.p[B3 * nc + c] = o.bphi;
}
// corner-averaged A (ct.zig:224); src is a component-major [3][nc] field
// (for the dynamo only component 2 is stored, components 0/1 are zero)
__global__ void k_corner_avg_a(DevState s, const double* src, int comp_stride_zero) {
  long nx = s.gr.nx, ny = s.gr.ny, nz = s.gr.nz, nc = s.gr.nc;
  long mz = nz == 1 ? 1 : nz + 1, my = ny == 1 ? 1 : ny + 1;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (nx + 1) * my * mz) return;
  long ix = t % (nx + 1), q = t / (nx + 1), iy = q % my, iz = q / my;
  for (int cc = 0; cc < 3; ++cc) {
    auto S = [&](long jx, long jy, long jz) -> double {
      if (comp_stride_zero && cc < 2) return 0.0;
      long off = comp_stride_zero ? 0 : (long)cc * nc;
      return src[off + cidx(s.gr, jx, jy, jz)];
    };
    double a;
    if (ny == 1 && nz == 1) a = 1.0 / 2.0 * (S(ix, iy, iz) + S(ix - 1, iy, iz));
    else if (ny > 1 && nz == 1) a = 1.0 / 4.0 * (S(ix, iy, iz) + S(ix, iy - 1, iz) + S(ix - 1, iy, iz) + S(ix - 1, iy - 1, iz));
    else if (nz > 1 && ny == 1) a = 1.0 / 4.0 * (S(ix, iy, iz) + S(ix, iy, iz - 1) + S(ix - 1, iy, iz) + S(ix - 1, iy, iz - 1));
    else
      a = 1.0 / 8.0 *
          (S(ix, iy, iz) + S(ix, iy - 1, iz) + S(ix - 1, iy, iz) + S(ix - 1, iy - 1, iz) + S(ix, iy, iz - 1) +
           S(ix, iy - 1, iz - 1) + S(ix - 1, iy, iz - 1) + S(ix - 1, iy - 1, iz - 1));
    s.vecpot[(long)cc * nc + cidx(s.gr, ix, iy, iz)] = a;
  }
}
// curl of the corner A (ct.zig:282) into vecpot 3..5, then (mode 0) superpose on
// the domain B and refresh the magnetic conserveds (dynamo.zig:420), or
// (mode 1) overwrite B and all conserveds (calc_BfromA ifoverwrite, domain part)
__global__ void __launch_bounds__(128) k_curl_apply(DevState s, double gam, int mode) {
  Range r = {0, 0, 0, s.gr.nx, s.gr.ny, s.gr.nz};
  long ix, iy, iz;
  if (!range_cell(r, ix, iy, iz)) return;
  long nc = s.gr.nc, nz = s.gr.nz;
  const Grid& g = s.gr.g;
  auto V = [&](int cc, long jx, long jy, long jz) { return s.vecpot[(long)cc * nc + cidx(s.gr, jx, jy, jz)]; };
  double dA[4][4];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) dA[i][j] = 0.0;
  if (nz == 1) {
    for (int cc = 0; cc < 3; ++cc) {
      dA[cc + 1][2] = -(V(cc, ix, iy, iz) - V(cc, ix, iy + 1, iz) + V(cc, ix + 1, iy, iz) - V(cc, ix + 1, iy + 1, iz)) /
                      (2.0 * cell_size(g, iy, 1));
      dA[cc + 1][1] = -(V(cc, ix, iy, iz) + V(cc, ix, iy + 1, iz) - V(cc, ix + 1, iy, iz) - V(cc, ix + 1, iy + 1, iz)) /
                      (2.0 * cell_size(g, ix, 0));
      dA[cc + 1][3] = 0.0;
    }
  } else {
    for (int cc = 0; cc < 3; ++cc) {
      dA[cc + 1][1] = (V(cc, ix + 1, iy, iz) - V(cc, ix, iy, iz) + V(cc, ix + 1, iy + 1, iz) - V(cc, ix, iy + 1, iz) +
                       V(cc, ix + 1, iy, iz + 1) - V(cc, ix, iy, iz + 1) + V(cc, ix + 1, iy + 1, iz + 1) -
                       V(cc, ix, iy + 1, iz + 1)) /
                      (4.0 * cell_size(g, ix, 0));
      dA[cc + 1][2] = (V(cc, ix, iy + 1, iz) - V(cc, ix, iy, iz) + V(cc, ix + 1, iy + 1, iz) - V(cc, ix + 1, iy, iz) +
                       V(cc, ix, iy + 1, iz + 1) - V(cc, ix, iy, iz + 1) + V(cc, ix + 1, iy + 1, iz + 1) -
                       V(cc, ix + 1, iy, iz + 1)) /
                      (4.0 * cell_size(g, iy, 1));
      dA[cc + 1][3] = (V(cc, ix, iy, iz + 1) - V(cc, ix, iy, iz) + V(cc, ix + 1, iy, iz + 1) - V(cc, ix + 1, iy, iz) +
                       V(cc, ix, iy + 1, iz + 1) - V(cc, ix, iy + 1, iz) + V(cc, ix + 1, iy + 1, iz + 1) -
                       V(cc, ix + 1, iy + 1, iz)) /
                      (4.0 * cell_size(g, iz, 2));
    }
  }
  long c = cidx(s.gr, ix, iy, iz);
  double gdet = s.cgc[10L * nc + c];
  double b1 = (dA[2][3] - dA[3][2]) / gdet;
  double b2 = (dA[3][1] - dA[1][3]) / gdet;
  double b3 = (dA[1][2] - dA[2][1]) / gdet;
  double pp[NV];
  load_cell(s.p, nc, c, pp);
  if (mode == 0) {
    pp[B1] += b1;
    pp[B2] += b2;
    pp[B3] += b3;
  } else {
    pp[B1] = b1;
    pp[B2] = b2;
    pp[B3] = b3;
  }
  Geom geo;
  geom_cell(s, ix, iy, iz, geo);
  double uu[NV];
  p2u(pp, uu, geo, gam);
  s.p[B1 * nc + c] = pp[B1];
  s.p[B2 * nc + c] = pp[B2];
  s.p[B3 * nc + c] = pp[B3];
  if (mode == 0) {
    s.u[B1 * nc + c] = uu[B1];
    s.u[B2 * nc + c] = uu[B2];
    s.u[B3 * nc + c] = uu[B3];
  } else {
    store_cell(s.u, nc, c, uu);
  }
}

// ---- PUFFY init passes (puffy.zig:873 initAll) -------------------------------
// calc_BfromA's overwrite outside the domain (ct.zig:184): a ghost cell takes
// the curl scratch there, which the curl never writes and which holds zeros,
// and all its conserveds are refreshed.
__global__ void __launch_bounds__(128) k_init_ghost_b(DevState s, double gam) {
  long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long nc = s.gr.nc;
  if (c >= nc) return;
  long ix = c % s.gr.sx - s.gr.ngx, iy = (c / s.gr.sx) % s.gr.sy - s.gr.ngy, iz = c / (s.gr.sx * s.gr.sy) - s.gr.ngz;
  if (ix >= 0 && ix < s.gr.nx && iy >= 0 && iy < s.gr.ny && iz >= 0 && iz < s.gr.nz) return;
  double pp[NV], uu[NV];
  load_cell(s.p, nc, c, pp);
  pp[B1] = 0.0;
  pp[B2] = 0.0;
  pp[B3] = 0.0;
  Geom geo;
  geom_cell(s, ix, iy, iz, geo);
  p2u(pp, uu, geo, gam);
  store_cell(s.p, nc, c, pp);
  store_cell(s.u, nc, c, uu);
}
// postinit pass 1 (puffy.zig:939 betaMaxRows): the domain maximum of
// p_mag / p_tot with p_tot = p_gas + Ehat/3, as ordered bits of a positive
// double in sc->tsd_max_bits (the reference starts its max at 0, and a NaN
// never wins a `>` comparison).
__global__ void __launch_bounds__(128) k_init_beta_max(DevState s, DevScalars* sc, double gam) {
  Range r = {0, 0, 0, s.gr.nx, s.gr.ny, s.gr.nz};
  long ix, iy, iz;
  double v = 0.0;
  if (range_cell(r, ix, iy, iz)) {
    long nc = s.gr.nc, c = cidx(s.gr, ix, iy, iz);
    double pp[NV];
    load_cell(s.p, nc, c, pp);
    Geom geo;
    geom_cell(s, ix, iy, iz, geo);
    double ucon[4], ucov[4], bcon[4], bcov[4], bsq;
    ucon_ucov_from_prims(pp[VX], pp[VY], pp[VZ], geo, ucon, ucov);
    double B[3] = {pp[B1], pp[B2], pp[B3]};
    bcon_bcov_bsq(B, ucon, ucov, geo, bcon, bcov, bsq);
    double pmag = bsq / 2.0;
    double ptot = (gam - 1.0) * pp[UU];
    ptot += -calc_ff_rtt(pp, geo, nullptr) / 3.0;
    double q = pmag / ptot;
    if (q > 0.0) v = q;
  }
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffff, v, o));
  __shared__ double smax[32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) smax[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, smax[w]);
    if (m > 0.0) atomicMax(&sc->tsd_max_bits, dbits(m));
  }
}
// postinit pass 2 (puffy.zig:984 betaScaleRows): B *= fac and p2u, domain only
__global__ void __launch_bounds__(128) k_init_beta_scale(DevState s, double gam, double fac) {
  Range r = {0, 0, 0, s.gr.nx, s.gr.ny, s.gr.nz};
  long ix, iy, iz;
  if (!range_cell(r, ix, iy, iz)) return;
  long nc = s.gr.nc, c = cidx(s.gr, ix, iy, iz);
  double pp[NV], uu[NV];
  load_cell(s.p, nc, c, pp);
  pp[B1] *= fac;
  pp[B2] *= fac;
  pp[B3] *= fac;
  Geom geo;
  geom_cell(s, ix, iy, iz, geo);
  p2u(pp, uu, geo, gam);
  store_cell(s.p, nc, c, pp);
  store_cell(s.u, nc, c, uu);
}

// ---- scalar diagnostics (koral/io/scalars.zig, koral/io/dump.zig:358) ---------
// Each reduction writes its per-cell terms in the reference's serial loop order
// and k_fold_ordered adds them in that order, so the sums are the serial ones.

// per domain cell: the totalMass term (scalars.zig:78) at index
// ix + nx (iy + ny iz), and the collectDiag counts (non-finite cells, hd flags)
__global__ void __launch_bounds__(128) k_diag_cells(DevState s, double phifac, double* mass_terms,
                                                    unsigned long long* counts) {
  Range r = {0, 0, 0, s.gr.nx, s.gr.ny, s.gr.nz};
  long ix, iy, iz;
  if (!range_cell(r, ix, iy, iz)) return;
  long nc = s.gr.nc, c = cidx(s.gr, ix, iy, iz);
  const Grid& g = s.gr.g;
  double dx = cell_size(g, ix, 0), dy = cell_size(g, iy, 1), dz = cell_size(g, iz, 2) * phifac;
  mass_terms[ix + s.gr.nx * (iy + s.gr.ny * iz)] = s.p[RHO * nc + c] * dx * dy * dz * s.cgc[10L * nc + c];
  bool bad = false;
  for (int iv = 0; iv < NV; ++iv)
    if (!kmath::isfinite(s.p[iv * nc + c])) bad = true;
  if (bad) atomicAdd(&counts[0], 1ULL);
  if (s.flags[3 * nc + c] != 0) atomicAdd(&counts[1], 1ULL);
}
// the mdot terms through radial shell ix (scalars.zig:106), index iy + ny iz;
// dzfac = 0 selects the 2D dphi = 2 pi
__global__ void __launch_bounds__(128) k_diag_mdot(DevState s, DevScalars* sc, long ix, double dzfac, double* terms) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long ny = s.gr.ny;
  if (t >= ny * s.gr.nz) return;
  long iy = t % ny, iz = t / ny;
  long nc = s.gr.nc, c = cidx(s.gr, ix, iy, iz);
  Geom geo;
  geom_cell(s, ix, iy, iz, geo);
  double vcon[4] = {0.0, s.p[VX * nc + c], s.p[VY * nc + c], s.p[VZ * nc + c]}, ucon[4];
  int e = convert(vcon, VELR, VEL4, geo, RECOMPUTE_UT, ucon);
  if (e) {
    set_err(sc, e, c);
    terms[t] = 0.0;
    return;
  }
  double rhouconr = s.p[RHO * nc + c] * ucon[1];
  double dy = cell_size(s.gr.g, iy, 1);
  double dz = dzfac == 0.0 ? 2.0 * KP_PI : cell_size(s.gr.g, iz, 2) * dzfac;
  terms[t] = geo.gdet * rhouconr * dy * dz;
}
// the type-1 luminosity terms through radial shell ix in BL (scalars.zig:136):
// gbl, dth, dph are the shell's BL geometry and cell widths, index iy + ny iz
__global__ void __launch_bounds__(128) k_diag_lum(DevState s, DevScalars* sc, long ix, double gam, const Geom* gbl,
                                                  const double* dth, const double* dph, double* rad_terms,
                                                  double* tot_terms) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long ny = s.gr.ny;
  if (t >= ny * s.gr.nz) return;
  long iy = t % ny, iz = t / ny;
  long nc = s.gr.nc, c = cidx(s.gr, ix, iy, iz);
  double pp[NV];
  load_cell(s.p, nc, c, pp);
  Geom geo;
  geom_cell(s, ix, iy, iz, geo);
  const Geom& gb = gbl[t];
  double jac[4][4];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) jac[i][j] = s.jbl[(long)(i * 4 + j) * nc + c];
  int e = trans_pmhd_coco_j(pp, geo, gb, jac, pp);
  if (!e) e = trans_prad_coco_j(pp, geo, gb, jac, pp);
  double vcon[4] = {0.0, pp[VX], pp[VY], pp[VZ]}, ucon[4];
  if (!e) e = convert(vcon, VELR, VEL4, gb, RECOMPUTE_UT, ucon);
  if (e) {
    set_err(sc, e, c);
    rad_terms[t] = 0.0;
    tot_terms[t] = 0.0;
    return;
  }
  double rhour = pp[RHO] * ucon[1];
  double tup[4][4], tij[4][4], rup[4][4], rij[4][4];
  calc_tij(pp, gb, gam, tup);
  lower_second(tup, gb, tij);
  double trt = tij[1][0];
  calc_rij(pp, gb, rup);
  lower_second(rup, gb, rij);
  double rrt = -rij[1][0];
  if (rrt < 0.0) rrt = 0.0;
  rad_terms[t] = gb.gdet * rrt * dth[t] * dph[t];
  tot_terms[t] = gb.gdet * (rhour + trt + rrt) * dth[t] * dph[t];
}
// out[0] = ((0 + v[0]) + v[1]) + ... in index order: a block stages tiles in
// shared memory, thread 0 adds them in order
__global__ void __launch_bounds__(256) k_fold_ordered(const double* v, long n, double* out) {
  __shared__ double tile[2048];
  double acc = 0.0;
  for (long k0 = 0; k0 < n; k0 += 2048) {
    long m = n - k0 < 2048 ? n - k0 : 2048;
    for (long k = threadIdx.x; k < m; k += blockDim.x) tile[k] = v[k0 + k];
    __syncthreads();
    if (threadIdx.x == 0)
      for (long k = 0; k < m; ++k) acc += tile[k];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = acc;
}

}  // namespace kc
