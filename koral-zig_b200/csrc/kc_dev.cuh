// kc_dev.cuh — device-resident state of the engine and the geometry loaders.
//
// Layout in HBM: every per-cell field is structure-of-arrays, component-major,
// over the reference's padded cell index c = jx + jy*SX + jz*SX*SY
// (koral/grid.zig:110), so a warp reading one component of 32 consecutive x
// cells issues one coalesced 256-byte load. The metric cache is stored
// compactly: g_{mu nu} as its 10-entry upper triangle (bitwise symmetric),
// g^{mu nu} as all 16 entries (the cofactor inverse is not bitwise symmetric),
// Christoffels Gamma^l_{mn} as 4 x 10 lower-symmetric entries.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/koral/kvisc.h"

namespace kc {

using namespace kp;

// padded grid (koral/grid.zig)
struct DGrid {
  int nx, ny, nz, ng, ngx, ngy, ngz;
  long sx, sy, sz, nc;
  Grid g;  // extents and spacings for the coordinate helpers
};

// number of stored geometry components per point
enum : int { NGC = 11, NGCON = 17, NKR = 40, NBL = 28 };

// Device pointers of one engine instance. Passed to kernels by value.
struct DevState {
  DGrid gr;
  // metric cache
  const double* cgc;     // [NGC][nc]   gcov sym10 + gdet
  const double* cGc;     // [NGCON][nc] gcon 16 + gttpert
  const double* fgc[3];  // faces [NGC][nf_d]
  const double* fGc[3];  // faces [NGCON][nf_d]
  long nf[3];            // face count per direction
  const double* kr;      // [NKR][nc]
  const double* blg;     // [NBL][nc] BL gcov sym10, gcon 16, r, theta
  const double* jbl;     // [16][nc] MKS2->BL point Jacobian
  const double* jb2m;    // [16][ngx*sy*sz] BL->MKS2 Jacobian at the x-hi ghost cells
  // state
  double* p;       // [NV][nc]
  double* u;       // [NV][nc]
  int* flags;      // [6][nc]
  double* amax;    // [6][nc]: ahd max per dim, arad max per dim
  double* flb[3];  // face fluxes [NV][nf_d]
  double* emf[3];  // corner EMFs [(nx+1)(ny+1)(nz+1)]
  double* rijvisc; // [16][nc]
  double* dyn_a;   // [nc] (the phi slot; the other two slots are identically zero)
  double* vecpot;  // [6][nc]
  double* scaleth; // [nx]
  double* fix_p;   // [NV][nc] fixup staging
  double* fix_u;   // [NV][nc]
  // the step's dt-derived coefficients (dt, dt gamma_imex, ...), written once a
  // step from the host, so that a captured step graph reads each step's values
  const double* coef;
};

// Device-side scalars written by kernels (one block, read back once a step).
struct DevScalars {
  unsigned long long tsd_max_bits;  // ordered bits of the positive CFL maximum (0 = none)
  unsigned long long tsd_min_bits;
  unsigned long long n_fail, n_iters, n_solves, n_guard;
  unsigned long long work_next;  // next work item of a persistent kernel
  int any_hd;      // some cell requested an hd fixup in the last u2p pass
  int err;         // first error code
  long long err_cell;
};

// symmetric 4x4 upper-triangle slot of (i, j)
KC_HD int sym10(int i, int j) {
  if (i > j) {
    int t = i;
    i = j;
    j = t;
  }
  // (00,01,02,03,11,12,13,22,23,33)
  return i == 0 ? j : i == 1 ? 3 + j : i == 2 ? 5 + j : 9;
}

// A load of data read once per launch; with STREAM it is marked evict-first in
// L2 (ld.global.cs), so that it does not push out what the kernel reuses.
template <bool STREAM = false>
__device__ __forceinline__ double ld_once(const double* p) {
  if (STREAM) return __ldcs(p);
  return *p;
}
template <bool STREAM = false>
__device__ __forceinline__ void geom_load(const double* gc, const double* Gc, long stride, long c, double x1, double x2,
                                          double x3, Geom& g) {
  double sym[10];
  for (int k = 0; k < 10; ++k) sym[k] = ld_once<STREAM>(gc + (long)k * stride + c);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      g.gg[i][j] = sym[sym10(i, j)];
      g.GG[i][j] = ld_once<STREAM>(Gc + (long)(i * 4 + j) * stride + c);
    }
  g.gg[0][4] = 0.0;
  g.gg[1][4] = 0.0;
  g.gg[2][4] = 0.0;
  g.gg[3][4] = ld_once<STREAM>(gc + 10L * stride + c);
  g.GG[0][4] = 0.0;
  g.GG[1][4] = 0.0;
  g.GG[2][4] = 0.0;
  g.GG[3][4] = ld_once<STREAM>(Gc + 16L * stride + c);
  g.xx[0] = 0.0;
  g.xx[1] = x1;
  g.xx[2] = x2;
  g.xx[3] = x3;
  geom_finish(g);
}

__device__ __forceinline__ long cidx(const DGrid& gr, long ix, long iy, long iz) {
  return (ix + gr.ngx) + (iy + gr.ngy) * gr.sx + (iz + gr.ngz) * gr.sx * gr.sy;
}
__device__ __forceinline__ long face_index(const DGrid& gr, int dim, long ix, long iy, long iz) {
  long jx = ix + gr.ngx, jy = iy + gr.ngy, jz = iz + gr.ngz;
  if (dim == 0) return jx + jy * (gr.sx + 1) + jz * gr.sy * (gr.sx + 1);
  if (dim == 1) return jx + jy * gr.sx + jz * (gr.sy + 1) * gr.sx;
  return jx + jy * gr.sx + jz * gr.sy * gr.sx;
}
template <bool STREAM = false>
__device__ __forceinline__ void geom_cell(const DevState& s, long ix, long iy, long iz, Geom& g) {
  geom_load<STREAM>(s.cgc, s.cGc, s.gr.nc, cidx(s.gr, ix, iy, iz), grid_xc(s.gr.g, ix), grid_yc(s.gr.g, iy),
                    grid_zc(s.gr.g, iz), g);
}
__device__ __forceinline__ void geom_face(const DevState& s, long ix, long iy, long iz, int dim, Geom& g) {
  double x1 = dim == 0 ? grid_xl(s.gr.g, ix) : grid_xc(s.gr.g, ix);
  double x2 = dim == 1 ? grid_yl(s.gr.g, iy) : grid_yc(s.gr.g, iy);
  double x3 = dim == 2 ? grid_zl(s.gr.g, iz) : grid_zc(s.gr.g, iz);
  geom_load(s.fgc[dim], s.fGc[dim], s.nf[dim], face_index(s.gr, dim, ix, iy, iz), x1, x2, x3, g);
}
// BL geometry of a cell (its xx = BL position, as the reference's blGeom)
__device__ __forceinline__ void geom_bl(const DevState& s, long c, Geom& g) {
  long n = s.gr.nc;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      g.gg[i][j] = s.blg[(long)sym10(i, j) * n + c];
      g.GG[i][j] = s.blg[(long)(10 + i * 4 + j) * n + c];
    }
  for (int i = 0; i < 4; ++i) {
    g.gg[i][4] = 0.0;
    g.GG[i][4] = 0.0;
  }
  g.xx[0] = 0.0;
  g.xx[1] = s.blg[26L * n + c];
  g.xx[2] = s.blg[27L * n + c];
  g.xx[3] = 0.0;
  g.gdet = 0.0;
  g.gttpert = 0.0;
  g.alpha = kmath::sqrt(-1.0 / g.GG[0][0]);
}
template <bool STREAM = false>
__device__ __forceinline__ void load_cell(const double* f, long nc, long c, double v[NV]) {
#pragma unroll
  for (int i = 0; i < NV; ++i) v[i] = ld_once<STREAM>(f + i * nc + c);
}
template <bool STREAM = false>
__device__ __forceinline__ void store_cell(double* f, long nc, long c, const double v[NV]) {
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    if (STREAM) __stcs(f + i * nc + c, v[i]);
    else f[i * nc + c] = v[i];
  }
}
__device__ __forceinline__ void kr_block(const DevState& s, long c, double k[64]) {
  for (int l = 0; l < 4; ++l)
    for (int m = 0; m < 4; ++m)
      for (int n = 0; n < 4; ++n) k[l * 16 + m * 4 + n] = s.kr[(long)(l * 10 + sym10(m, n)) * s.gr.nc + c];
}

}  // namespace kc
